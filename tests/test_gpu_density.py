"""iTPO (finite temperature, tg_params.density) on the GPU against the
oracle (oracle/tenes_density.py) and the reference's finite-temperature
golden runs: the single-layer CTMRG (corner and up/down projectors), the
density contractions (one site, nearest-neighbour op12 and its reduced
density matrix, windows of one-site operators, correlation strips, the
transfer matrix), the density simple update and the whole
finite-temperature driver."""
import os
import shutil

import numpy as np
import pytest

from oracle import tenes_density as D
from oracle import tenes_oracle as O
from tenes_b200.env import CTMParams, Environment
from tests._helpers import SX, SY, SZ, make_lattice

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def density_tensors(lat, seed, is_complex):
    """i.i.d. tensors with a decaying weight on every bond index, so that the
    corner spectra decay and no truncation falls between equal values."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(lat.N_UNIT):
        v = lat.virtual_dims[i]
        d = lat.physical_dims[i]
        sh = (v[0], v[1], v[2], v[3], d, d)
        T = rng.uniform(-1, 1, sh)
        if is_complex:
            T = T + 1j * rng.uniform(-1, 1, sh)
        for leg in range(4):
            w = 0.45 ** np.arange(v[leg])
            T = T * w.reshape([-1 if a == leg else 1 for a in range(6)])
        T[0, 0, 0, 0] += 2.0 * np.eye(d)  # a dominant identity part, as near infinite temperature
        out.append(T / np.max(np.abs(T)))
    return out


def gpu_density_env(lat, Tn, chi, is_complex, **kw):
    p = CTMParams(chi=chi, density=True, **kw)
    env = Environment(lat.LX, lat.LY, lat.physical_dims, lat.virtual_dims, p, is_complex, skew=lat.skew)
    for i, T in enumerate(Tn):
        env.set_site_tensor(i, T)
    return env


def close(g, o, tol, what):
    assert abs(g - o) <= tol * max(1.0, abs(o)), (what, g, o)


@pytest.mark.parametrize("corner", [True, False])
@pytest.mark.parametrize("is_complex", [False, True])
def test_density_ctm_and_observables_match_oracle(is_complex, corner):
    lat = make_lattice(2, 2, 3)
    Tn = density_tensors(lat, 5 + int(is_complex), is_complex)
    chi, iters = 8, 4
    p = O.Params(CHI=chi, Max_CTM_Iteration=iters, CTM_Projector_corner=corner)
    oe, ocnt, _, _ = D.calc_ctm_environment(Tn, p, lat, edge_bound=False)
    ge = gpu_density_env(lat, Tn, chi, is_complex, max_ctm_iteration=iters, projector_corner=corner)
    gcnt, _, _ = ge.calc_ctm_environment(True)
    assert gcnt == ocnt
    for w, name in enumerate(("C1", "C2", "C3", "C4")):
        for i in range(lat.N_UNIT):
            g = ge.corner_spectrum(w, i)
            o = O.corner_spectrum(getattr(oe, name)[i])
            np.testing.assert_allclose(g[:len(o)], o, rtol=1e-9, atol=1e-12, err_msg=f"{name}[{i}]")
            assert np.all(np.abs(g[len(o):]) < 1e-12)
    tol = 1e-9
    ops1 = (np.eye(2), SZ, SX, SY) if is_complex else (np.eye(2), SZ, SX)
    for i in range(lat.N_UNIT):
        for op in ops1:
            o = D.contract_one_site(oe.C1[i], oe.C2[i], oe.C3[i], oe.C4[i], oe.eTt[i], oe.eTr[i], oe.eTb[i],
                                    oe.eTl[i], Tn[i], op)
            close(ge.contract_one_site(i, op), o, tol, ("onesite", i))
    rng = np.random.default_rng(1)
    op12 = rng.standard_normal((2, 2, 2, 2)) + (1j * rng.standard_normal((2, 2, 2, 2)) if is_complex else 0)
    for s in range(lat.N_UNIT):
        for dx, dy in ((1, 0), (0, 1), (-1, 0), (0, -1)):
            o = D.contract_op12(oe, Tn, lat, s, dx, dy, op12)
            close(ge.contract_bond_op12(s, dx, dy, op12), o, tol, ("op12", s, dx, dy))
            rdm = ge.contract_bond_rdm(s, dx, dy)
            close(np.sum(op12 * rdm), o, tol, ("rdm", s, dx, dy))
    Y = SY if is_complex else SX @ SZ  # a real operator for real tensors
    for (nrow, ncol, sr, sc, ops) in ((1, 2, 0, 0, {(0, 0): SZ, (0, 1): SX}),
                                      (2, 1, 1, 0, {(1, 0): Y, (0, 0): SZ}),
                                      (2, 2, 1, 0, {(1, 0): SZ, (0, 1): SZ}),
                                      (3, 2, 2, 1, {(2, 1): SX, (0, 0): SZ, (1, 1): Y})):
        for s in range(lat.N_UNIT):
            o = D.window_value(oe, Tn, lat, s, nrow, ncol, sr, sc, ops)
            close(ge.contract_window(s, nrow, ncol, sr, sc, ops), o, tol, ("window", nrow, ncol, s))
    for left in range(lat.N_UNIT):
        for vertical in (False, True):
            o = np.array(D.correlation_strip(oe, Tn, lat, left, vertical, 4, SZ, lambda s: [SZ, SX]))
            g = ge.correlation_strip(left, vertical, 4, SZ, lambda s: [SZ, SX])
            np.testing.assert_allclose(g, o, rtol=1e-9, atol=1e-11)
    for direction in (0, 1):
        for fixed in range(2):
            o = D.tm_eigenvalues(oe, lat, direction, fixed, O.TMParams())
            g = ge.tm_eigenvalues(direction, fixed)
            np.testing.assert_allclose(np.abs(g), np.abs(o), rtol=1e-8)
    ge.close()


@pytest.mark.parametrize("is_complex", [False, True])
@pytest.mark.parametrize("leg", [0, 1, 2, 3])
def test_density_simple_update_matches_oracle(is_complex, leg):
    """One density bond step (kron(op, conj(op)) on the merged physical legs)
    and one one-site step, batched and single, against the oracle."""
    lat = make_lattice(2, 2, 3)
    Tn = density_tensors(lat, 11 + leg, is_complex)
    rng = np.random.default_rng(4)
    H = rng.standard_normal((4, 4)) + (1j * rng.standard_normal((4, 4)) if is_complex else 0)
    H = H + H.conj().T
    w, v = np.linalg.eigh(H)
    op = (v @ np.diag(np.exp(-0.1 * w)) @ v.conj().T).reshape(2, 2, 2, 2)
    h1 = rng.standard_normal((2, 2)) + (1j * rng.standard_normal((2, 2)) if is_complex else 0)
    lam = [[np.ones(3) for _ in range(4)] for _ in range(lat.N_UNIT)]

    class Up:
        def __init__(self, s, l, o):
            self.source_site, self.source_leg, self.op = s, l, o

        def is_onesite(self):
            return self.source_leg < 0
    src = 1
    tgt = lat.neighbor(src, leg)
    oT = [t.copy() for t in Tn]
    D.su_density(oT, lam, lat, Up(src, leg, op), O.Params())
    D.su_density(oT, lam, lat, Up(tgt, -1, h1), O.Params())
    for batched in (False, True):
        ge = gpu_density_env(lat, Tn, 4, is_complex)
        if batched:
            ge.simple_update_many([(src, leg, op), (tgt, -1, h1)])
        else:
            ge.simple_update(src, leg, op)
            ge.simple_update(tgt, -1, h1)
        np.testing.assert_allclose(ge.get_lambda(src, leg), lam[src][leg], rtol=1e-11)
        a, b = ge.get_site_tensor(src), ge.get_site_tensor(tgt)
        g = np.tensordot(a, b, ([leg], [(leg + 2) % 4]))
        o = np.tensordot(oT[src], oT[tgt], ([leg], [(leg + 2) % 4]))
        np.testing.assert_allclose(g, o, rtol=1e-10, atol=1e-12 * np.max(np.abs(o)))
        ge.close()


def test_density_init_is_the_identity():
    """tg_init_tensors on an iTPO: Tn[0,0,0,0,p,p] = 1 (tensors.cpp:190-202);
    its environment gives <1> = d per site and <S> = 0."""
    lat = make_lattice(2, 2, 3)
    ge = Environment(2, 2, lat.physical_dims, lat.virtual_dims, CTMParams(chi=6, density=True), True)
    ge.init_tensors(11, [[0.0]] * 4, [0.01] * 4)
    want = np.zeros((3, 3, 3, 3, 2, 2))
    want[0, 0, 0, 0] = np.eye(2)
    for i in range(4):
        np.testing.assert_array_equal(ge.get_site_tensor(i), want)
    ge.calc_ctm_environment(True)
    for i in range(4):
        n = ge.contract_one_site(i, np.eye(2))
        assert abs(ge.contract_one_site(i, SZ) / n) < 1e-14
    ge.close()


def _rows(path):
    out = []
    for line in open(path):
        line = line.split("#")[0].strip()
        if line:
            out.append([float(w) for w in line.split()])
    return out


@pytest.mark.parametrize("stem,tol,tol_xi", [("ft_tfi_square", 5e-5, 5e-4), ("ft_kitaev", 1e-9, 1e-4)])
def test_finite_temperature_golden_through_the_front_end(tmp_path, stem, tol, tol_xi):
    """The reference's FT_TFI_square and FT_Kitaev inputs through the GPU
    front end: every FT_*.dat row against the reference's own output at the
    oracle's distance to it (the reference checks rtol 1e-3 / atol 1e-4,
    test/fulltest.py.in:141-142)."""
    import tenes_b200.itps as itps
    from tests._ft import expected
    shutil.copyfile(os.path.join(GOLDEN, stem + "_input.toml"), tmp_path / "in.toml")
    itps.run(str(tmp_path / "in.toml"), print_level=0, outdir=str(tmp_path / "out"))
    exp = expected(stem)
    for name, key in [("FT_density.dat", "density"), ("FT_onesite_obs.dat", "onesite"),
                      ("FT_twosite_obs.dat", "twosite"), ("FT_correlation_length.dat", "correlation_length"),
                      ("FT_correlation.dat", "correlation")]:
        res = _rows(tmp_path / "out" / name)
        ref = exp[key]
        assert len(res) == len(ref), name
        t = tol_xi if key == "correlation_length" else tol
        for rs, rf in zip(res, ref):
            assert len(rs) == len(rf), name
            if int(rs[1]) == -1 and key in ("onesite", "twosite"):
                # a norm row: the single-layer network's norm carries the sign /
                # phase of its environment, which starts from all-ones boundary
                # vectors (ctm_single.cpp:752-960) and so follows the site
                # tensors' bond gauge (the simple update's singular-vector
                # signs); the observables divide it out
                rs, rf = rs[:-2] + [np.hypot(rs[-2], rs[-1]), 0.0], rf[:-2] + [np.hypot(rf[-2], rf[-1]), 0.0]
            np.testing.assert_allclose(rs, rf, rtol=t, atol=t, err_msg=name)
