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
