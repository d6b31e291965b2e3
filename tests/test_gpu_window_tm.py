"""N x M window observables and transfer-matrix eigenvalues on the GPU
against the oracle (Contract_RxC_iTPS_CTM, TransferMatrix::eigenvalues)."""
import numpy as np
import pytest

from oracle import tenes_oracle as O
from tests._helpers import SX, SZ, gpu_env, load_env, make_lattice, oracle_params, physical_tensors

pytestmark = pytest.mark.gpu


def _setup(is_complex, chi=6, D=2, sweeps=2):
    lat = make_lattice(2, 2, D)
    Tn = physical_tensors(lat, D, is_complex=is_complex)
    p = oracle_params(chi)
    oe = O.init_env(Tn, p, lat)
    for _ in range(sweeps):
        O.sweep(oe, Tn, p, lat)
    ge = gpu_env(lat, Tn, chi, is_complex)
    load_env(ge, oe)
    return lat, Tn, oe, ge


@pytest.mark.parametrize("is_complex", [False, True])
@pytest.mark.parametrize("shape", [(1, 2), (2, 1), (2, 2), (3, 2), (2, 3)])
def test_window_matches_oracle(is_complex, shape):
    lat, Tn, oe, ge = _setup(is_complex)
    nrow, ncol = shape
    rng = np.random.default_rng(nrow * 10 + ncol)
    for source in range(lat.N_UNIT):
        sr, sc = nrow - 1, 0
        idx, Cs, eTt, eTr, eTb, eTl, T = O._window(oe, Tn, lat, source, sc, sr, nrow, ncol)
        ops = {(0, ncol - 1): SZ, (nrow - 1, 0): SX + 0.3 * rng.standard_normal((2, 2))}
        opgrid = [[ops.get((r, c), np.eye(2)) for c in range(ncol)] for r in range(nrow)]
        o = O.contract_window(Cs, eTt, eTr, eTb, eTl, T, opgrid)
        g = ge.contract_window(source, nrow, ncol, sr, sc, ops)
        assert abs(g - o) <= 1e-10 * abs(o), (g, o)
        n_o = O.contract_window(Cs, eTt, eTr, eTb, eTl, T, [[np.eye(2)] * ncol for _ in range(nrow)])
        n_g = ge.contract_window(source, nrow, ncol, sr, sc)
        assert abs(n_g - n_o) <= 1e-10 * abs(n_o)


@pytest.mark.parametrize("is_complex", [False, True])
@pytest.mark.parametrize("chi", [8, 16])
def test_transfer_matrix_eigenvalues(is_complex, chi):
    """chi=8: N=64, dense eigensolver; chi=16: N=256 > 200, Arnoldi (maxdim 50, maxiter 1)."""
    lat, Tn, oe, ge = _setup(is_complex, chi=chi, sweeps=3)
    tp = O.TMParams()
    for direction in (0, 1):
        for fixed in range(2):
            o = O.tm_eigenvalues(oe, lat, direction, fixed, tp)
            g = ge.tm_eigenvalues(direction, fixed)
            L = 2
            xo, eo = O.correlation_length(o, L)
            xg, eg = O.correlation_length(g, L)
            np.testing.assert_allclose(np.abs(g), np.abs(o), rtol=1e-9 if chi == 8 else 1e-7)
            assert abs(xg - xo) <= (1e-9 if chi == 8 else 1e-7) * abs(xo)


@pytest.mark.parametrize("is_complex", [False, True])
def test_bond_rdm_reproduces_op12(is_complex):
    """tg_measure_bond_rdm: sum(op12 * rdm) equals Contract_two_sites_*_op12 of
    the oracle (source left / right / top / bottom), einsum('abab', rdm) its norm."""
    lat, Tn, oe, ge = _setup(is_complex)
    rng = np.random.default_rng(17)
    for source in range(lat.N_UNIT):
        for dx, dy in ((1, 0), (-1, 0), (0, 1), (0, -1)):
            op = rng.standard_normal((2, 2, 2, 2))
            if is_complex:
                op = op + 1j * rng.standard_normal((2, 2, 2, 2))
            rho = ge.contract_bond_rdm(source, dx, dy)
            assert rho.shape == (2, 2, 2, 2)
            g = ge.contract_bond_op12(source, dx, dy, op)
            assert abs(np.sum(op * rho) - g) <= 1e-11 * abs(g), (source, dx, dy)
            ident = np.einsum("ac,bd->abcd", np.eye(2), np.eye(2))
            n = ge.contract_bond_op12(source, dx, dy, ident)
            assert abs(np.einsum("abab->", rho) - n) <= 1e-11 * abs(n)
            # against the oracle directly
            target = lat.other(source, dx, dy)
            if dy == 0:
                left, right = (source, target) if dx > 0 else (target, source)
                o = op if left == source else op.transpose(1, 0, 3, 2)
                ref = O.contract_two_sites_horizontal_op12(
                    oe.C1[left], oe.C2[right], oe.C3[right], oe.C4[left], oe.eTt[left], oe.eTt[right],
                    oe.eTr[right], oe.eTb[right], oe.eTb[left], oe.eTl[left], Tn[left], Tn[right], o)
            else:
                top, bottom = (target, source) if dy > 0 else (source, target)
                o = op if top == source else op.transpose(1, 0, 3, 2)
                ref = O.contract_two_sites_vertical_op12(
                    oe.C1[top], oe.C2[top], oe.C3[bottom], oe.C4[bottom], oe.eTt[top], oe.eTr[top],
                    oe.eTr[bottom], oe.eTb[bottom], oe.eTl[bottom], oe.eTl[top], Tn[top], Tn[bottom], o)
            assert abs(np.sum(op * rho) - ref) <= 1e-10 * abs(ref), (source, dx, dy)
    ge.close()


@pytest.mark.parametrize("is_complex", [False, True])
def test_correlation_strip(is_complex):
    """tg_measure_correlation (StartCorrelation / Transfer / FinishCorrelation)
    against the oracle's strip for r = 1..5 in both directions, and against
    the GPU's own windows for r <= 3."""
    lat, Tn, oe, ge = _setup(is_complex)
    ops = [SZ, SX]
    for left in range(lat.N_UNIT):
        for vertical in (False, True):
            strip = ge.correlation_strip(left, vertical, 5, SZ, lambda s: ops)
            ref = O.correlation_strip(oe, Tn, lat, left, vertical, 5, SZ, lambda s: ops)
            np.testing.assert_allclose(strip, np.array(ref), rtol=1e-10, atol=1e-13)
            for r in range(1, 4):
                if vertical:
                    geo, pl, pr = (r + 1, 1, r, 0), (r, 0), (0, 0)
                else:
                    geo, pl, pr = (1, r + 1, 0, 0), (0, 0), (0, r)
                n = ge.contract_window(left, *geo)
                for k, op in enumerate(ops):
                    w = ge.contract_window(left, *geo, {pl: SZ, pr: op}) / n
                    assert abs(strip[r - 1][k] - w) <= 1e-10 * max(1.0, abs(w))
    ge.close()
