"""CTMRG parity: the CUDA path against the FP64 oracle on the same seeded
tensors.  Gauge-invariant quantities are compared (|entries| after one move,
corner spectra, observables); the tolerance is 1e-10 relative."""
import numpy as np
import pytest

from oracle import tenes_oracle as O
from tests._helpers import (SX, SZ, gpu_env, load_env, make_lattice, oracle_params,
                            physical_tensors, random_tensors, rel)

pytestmark = pytest.mark.gpu
TOL = 1e-10


@pytest.mark.parametrize("is_complex", [False, True])
def test_init_env_matches_oracle(is_complex):
    lat = make_lattice(2, 2, 2)
    Tn = random_tensors(lat, 1, is_complex)
    chi = 6
    oe = O.init_env(Tn, oracle_params(chi), lat)
    ge = gpu_env(lat, Tn, chi, is_complex)
    ge.init_env()
    for w, name in enumerate(("C1", "C2", "C3", "C4", "eTt", "eTr", "eTb", "eTl")):
        for i in range(lat.N_UNIT):
            np.testing.assert_allclose(ge.get_env(w, i), getattr(oe, name)[i], rtol=0, atol=1e-13)


@pytest.mark.parametrize("direction", [0, 1, 2, 3])
@pytest.mark.parametrize("is_complex", [False, True])
def test_single_move_matches_oracle(direction, is_complex):
    lat = make_lattice(2, 2, 2)
    Tn = random_tensors(lat, 7, is_complex)
    chi = 8
    p = oracle_params(chi)
    oe = O.init_env(Tn, p, lat)
    O.sweep(oe, Tn, p, lat)  # a non-trivial environment
    ge = gpu_env(lat, Tn, chi, is_complex)
    load_env(ge, oe)
    move = (O.left_move, O.right_move, O.top_move, O.bottom_move)[direction]
    move(oe, Tn, 0, p, lat)
    ge.move(direction, 0)
    # sign / phase gauge of the SVD leaves |entries| unchanged
    for w, name in enumerate(("C1", "C2", "C3", "C4", "eTt", "eTr", "eTb", "eTl")):
        for i in range(lat.N_UNIT):
            g = np.abs(ge.get_env(w, i))
            o = np.abs(getattr(oe, name)[i])
            np.testing.assert_allclose(g, o, rtol=1e-9, atol=1e-11, err_msg=f"{name}[{i}]")


def _observables_oracle(oe, Tn, lat):
    out = []
    for i in range(lat.N_UNIT):
        nrm = O.contract_one_site(oe.C1[i], oe.C2[i], oe.C3[i], oe.C4[i], oe.eTt[i], oe.eTr[i],
                                  oe.eTb[i], oe.eTl[i], Tn[i], np.eye(2))
        for op in (SZ, SX):
            v = O.contract_one_site(oe.C1[i], oe.C2[i], oe.C3[i], oe.C4[i], oe.eTt[i], oe.eTr[i],
                                    oe.eTb[i], oe.eTl[i], Tn[i], op)
            out.append((v / nrm).real)
    return out


def _observables_gpu(ge, lat):
    out = []
    for i in range(lat.N_UNIT):
        nrm = ge.contract_one_site(i, np.eye(2))
        for op in (SZ, SX):
            out.append((ge.contract_one_site(i, op) / nrm).real)
    return out


@pytest.mark.parametrize("D,chi,iters,corner", [(2, 10, 10, True), (3, 12, 6, True), (2, 8, 5, False)])
def test_ctm_run_matches_oracle(D, chi, iters, corner):
    lat = make_lattice(2, 2, D)
    Tn = random_tensors(lat, 11 + D, False)
    p = oracle_params(chi, Max_CTM_Iteration=iters, CTM_Projector_corner=corner)
    oe, ocnt, oconv, osig = O.calc_ctm_environment(Tn, p, lat)
    ge = gpu_env(lat, Tn, chi, False, max_ctm_iteration=iters, projector_corner=corner)
    gcnt, gconv, gsig = ge.calc_ctm_environment(True)
    assert gcnt == ocnt and gconv == oconv
    assert rel(gsig, osig) < 1e-6 or abs(gsig - osig) < 1e-12
    for w, name in enumerate(("C1", "C2", "C3", "C4")):
        for i in range(lat.N_UNIT):
            np.testing.assert_allclose(ge.corner_spectrum(w, i), O.corner_spectrum(getattr(oe, name)[i]),
                                       rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(_observables_gpu(ge, lat), _observables_oracle(oe, Tn, lat), rtol=TOL, atol=1e-12)
    # nearest-neighbour <SzSz> through the op12 contractions
    op12 = np.einsum("ac,bd->abcd", SZ, SZ)
    for i in range(lat.N_UNIT):
        for dx, dy in ((1, 0), (0, 1)):
            g = ge.contract_bond_op12(i, dx, dy, op12) / ge.contract_bond_op12(i, dx, dy, np.einsum(
                "ac,bd->abcd", np.eye(2), np.eye(2)))
            if dy == 0:
                j = lat.right(i)
                args = (oe.C1[i], oe.C2[j], oe.C3[j], oe.C4[i], oe.eTt[i], oe.eTt[j], oe.eTr[j],
                        oe.eTb[j], oe.eTb[i], oe.eTl[i], Tn[i], Tn[j])
                f = O.contract_two_sites_horizontal_op12
            else:
                j = lat.top(i)
                args = (oe.C1[j], oe.C2[j], oe.C3[i], oe.C4[i], oe.eTt[j], oe.eTr[j], oe.eTr[i],
                        oe.eTb[i], oe.eTl[i], oe.eTl[j], Tn[j], Tn[i])
                f = O.contract_two_sites_vertical_op12
            o = f(*args, op12) / f(*args, np.einsum("ac,bd->abcd", np.eye(2), np.eye(2)))
            assert rel(g.real, o.real) < TOL or abs(g.real - o.real) < 1e-12


def test_complex_ctm_run_matches_oracle():
    lat = make_lattice(2, 2, 2)
    Tn = random_tensors(lat, 5, True)
    chi = 8
    p = oracle_params(chi, Max_CTM_Iteration=4)
    oe, ocnt, _, _ = O.calc_ctm_environment(Tn, p, lat)
    ge = gpu_env(lat, Tn, chi, True, max_ctm_iteration=4)
    gcnt, _, _ = ge.calc_ctm_environment(True)
    assert gcnt == ocnt
    np.testing.assert_allclose(_observables_gpu(ge, lat), _observables_oracle(oe, Tn, lat), rtol=TOL, atol=1e-12)


@pytest.mark.parametrize("is_complex", [False, True])
@pytest.mark.parametrize("oversample", [-1, 4])
def test_rsvd_ctm_run_matches_oracle(is_complex, oversample):
    """rSVD projectors (ctm.cpp:231-266) with the shared counter-based test
    matrix: the GPU rSVD and the oracle's see identical random inputs, so the
    environments agree to rounding.  Physical (simple-update) tensors: with
    i.i.d. random tensors the spectrum is flat at the sketch size and the rSVD
    iteration amplifies rounding differences."""
    lat = make_lattice(2, 2, 2)
    Tn = physical_tensors(lat, 2, is_complex=is_complex)
    chi, iters = 8, 4
    kw = dict(Use_RSVD=True, Max_CTM_Iteration=iters, rsvd_power_iters=2)
    if oversample >= 0:
        kw["rsvd_oversample_abs"] = oversample
    oe, ocnt, _, _ = O.calc_ctm_environment(Tn, oracle_params(chi, **kw), lat)
    ge = gpu_env(lat, Tn, chi, is_complex, max_ctm_iteration=iters, use_rsvd=True,
                 rsvd_oversample_abs=oversample, rsvd_power_iters=2)
    gcnt, _, _ = ge.calc_ctm_environment(True)
    assert gcnt == ocnt
    for w, name in enumerate(("C1", "C2", "C3", "C4")):
        for i in range(lat.N_UNIT):
            np.testing.assert_allclose(ge.corner_spectrum(w, i), O.corner_spectrum(getattr(oe, name)[i]),
                                       rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(_observables_gpu(ge, lat), _observables_oracle(oe, Tn, lat), rtol=TOL, atol=1e-12)


@pytest.mark.parametrize("is_complex", [False, True])
def test_rsvd_single_move_matches_oracle(is_complex):
    """One Left_move with rSVD projectors from a full-rank environment."""
    lat = make_lattice(2, 2, 2)
    Tn = random_tensors(lat, 31, is_complex)
    chi = 8
    p_full = oracle_params(chi)
    oe = O.init_env(Tn, p_full, lat)
    for _ in range(2):
        O.sweep(oe, Tn, p_full, lat)
    p = oracle_params(chi, Use_RSVD=True, rsvd_power_iters=2, rsvd_oversample_abs=4)
    ge = gpu_env(lat, Tn, chi, is_complex, use_rsvd=True, rsvd_oversample_abs=4, rsvd_power_iters=2)
    load_env(ge, oe)
    O.left_move(oe, Tn, 0, p, lat)
    ge.move(0, 0)
    for w, name in enumerate(("C1", "C2", "C3", "C4", "eTt", "eTr", "eTb", "eTl")):
        for i in range(lat.N_UNIT):
            np.testing.assert_allclose(np.abs(ge.get_env(w, i)), np.abs(getattr(oe, name)[i]), rtol=1e-8,
                                       atol=1e-10, err_msg=f"{name}[{i}]")


@pytest.mark.parametrize("direction", [0, 1, 2, 3])
@pytest.mark.parametrize("is_complex", [False, True])
def test_updown_rsvd_single_move_matches_oracle(direction, is_complex):
    """One move with the rSVD branch of the up/down projectors
    (ctm.cpp:401-439; projector_corner = false), from a full-rank environment:
    the GPU applies M = RT^T LT LB RB as four products per panel, the oracle
    forms R1 R2^T; both draw the same counter-based test matrix."""
    lat = make_lattice(2, 2, 2)
    Tn = random_tensors(lat, 31, is_complex)
    chi = 8
    p_full = oracle_params(chi, CTM_Projector_corner=False)
    oe = O.init_env(Tn, p_full, lat)
    for _ in range(2):
        O.sweep(oe, Tn, p_full, lat)
    p = oracle_params(chi, Use_RSVD=True, CTM_Projector_corner=False, rsvd_power_iters=2, rsvd_oversample_abs=4)
    ge = gpu_env(lat, Tn, chi, is_complex, use_rsvd=True, projector_corner=False, rsvd_oversample_abs=4,
                 rsvd_power_iters=2)
    load_env(ge, oe)
    move = (O.left_move, O.right_move, O.top_move, O.bottom_move)[direction]
    move(oe, Tn, 0, p, lat)
    ge.move(direction, 0)
    for w, name in enumerate(("C1", "C2", "C3", "C4", "eTt", "eTr", "eTb", "eTl")):
        for i in range(lat.N_UNIT):
            np.testing.assert_allclose(np.abs(ge.get_env(w, i)), np.abs(getattr(oe, name)[i]), rtol=1e-8,
                                       atol=1e-10, err_msg=f"{name}[{i}]")


@pytest.mark.parametrize("is_complex", [False, True])
def test_updown_rsvd_ctm_run_matches_oracle(is_complex):
    """Whole CTMRG runs with up/down rSVD projectors and the reference's
    default multiplicative oversampling (k = 2 cut)."""
    lat = make_lattice(2, 2, 2)
    Tn = physical_tensors(lat, 2, is_complex=is_complex)
    chi, iters = 8, 4
    oe, ocnt, _, _ = O.calc_ctm_environment(
        Tn, oracle_params(chi, Use_RSVD=True, CTM_Projector_corner=False, Max_CTM_Iteration=iters,
                          rsvd_power_iters=2), lat)
    ge = gpu_env(lat, Tn, chi, is_complex, max_ctm_iteration=iters, use_rsvd=True, projector_corner=False,
                 rsvd_power_iters=2)
    gcnt, _, _ = ge.calc_ctm_environment(True)
    assert gcnt == ocnt
    for w, name in enumerate(("C1", "C2", "C3", "C4")):
        for i in range(lat.N_UNIT):
            # the reference shrinks a leg to the cut when s_i/s_0 <= 1e-12 cuts
            # below chi; the GPU keeps chi with exact zeros there
            o = O.corner_spectrum(getattr(oe, name)[i])
            g = ge.corner_spectrum(w, i)
            np.testing.assert_allclose(g[:len(o)], o, rtol=1e-9, atol=1e-12)
            assert np.all(g[len(o):] == 0.0)
    np.testing.assert_allclose(_observables_gpu(ge, lat), _observables_oracle(oe, Tn, lat), rtol=TOL, atol=1e-12)


@pytest.mark.parametrize("is_complex", [False, True])
def test_graph_sweeps_equal_eager_sweeps(is_complex):
    """Sweeps replayed from the captured CUDA graph give the same environment as
    sweeps launched kernel by kernel, re-capture after the site tensors change,
    and count the same kernels."""
    from tenes_b200.env import kernel_launch_count
    lat = make_lattice(2, 2, 2)
    Tn = physical_tensors(lat, 2, is_complex=is_complex)
    kw = dict(use_rsvd=True, rsvd_oversample_abs=4, rsvd_power_iters=2, max_ctm_iteration=5,
              ctm_convergence_epsilon=1e-30)
    envs = {g: gpu_env(lat, Tn, 8, is_complex, cuda_graph=g, **kw) for g in (False, True)}
    counts = {}
    for g, e in envs.items():
        e.init_env()
        n0 = kernel_launch_count()
        for _ in range(5):
            e.sweep()
        counts[g] = kernel_launch_count() - n0
    assert counts[True] == counts[False] > 0
    for rnd in range(2):
        for w in range(8):
            for i in range(lat.N_UNIT):
                a, b = envs[False].get_env(w, i), envs[True].get_env(w, i)
                np.testing.assert_allclose(b, a, rtol=0, atol=1e-13 * np.abs(a).max())
        if rnd == 0:
            for e in envs.values():
                e.set_site_tensor(0, Tn[1] if Tn[1].shape == Tn[0].shape else Tn[0])
                for _ in range(3):
                    e.sweep()


@pytest.mark.parametrize("LX,LY,skew", [(2, 1, 1), (3, 2, 1), (2, 2, 1)])
@pytest.mark.parametrize("is_complex", [False, True])
def test_skewed_cell_ctm_run_matches_oracle(LX, LY, skew, is_complex):
    """Skewed unit cells, where a move's current and next lines share sites
    (the second pass must read the corners and edges as they were before it,
    the reference's C1_bak / eTl_bak, ctm.cpp:595-601): a whole run against the
    oracle, corner spectra, one-site values and both transfer-matrix
    spectra, whose sub-leading eigenvalues see every edge tensor."""
    lat = make_lattice(LX, LY, 2, skew=skew)
    Tn = random_tensors(lat, 7 + LX + LY, is_complex)
    chi, iters = 8, 4
    oe, ocnt, _, _ = O.calc_ctm_environment(Tn, oracle_params(chi, Max_CTM_Iteration=iters), lat)
    ge = gpu_env(lat, Tn, chi, is_complex, max_ctm_iteration=iters)
    gcnt, _, _ = ge.calc_ctm_environment(True)
    assert gcnt == ocnt
    for w, name in enumerate(("C1", "C2", "C3", "C4")):
        for i in range(lat.N_UNIT):
            np.testing.assert_allclose(ge.corner_spectrum(w, i), O.corner_spectrum(getattr(oe, name)[i]),
                                       rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(_observables_gpu(ge, lat), _observables_oracle(oe, Tn, lat), rtol=TOL, atol=1e-12)
    # The vertical transfer matrix of a skewed cell continues at column
    # x + skew after the top row (transfer_matrix.cpp:281, 302), while the
    # site above that row is in column x - skew (SquareLattice.cpp:95-100);
    # unless the two coincide (2 skew = 0 mod LX) it chains edge tensors that
    # share no bond, and its spectrum depends on the projectors' singular-
    # vector phases -- in the reference as much as here -- so only the
    # well-defined cases are compared.
    dirs = (0, 1) if (2 * skew) % LX == 0 else (0,)
    for d in dirs:
        fixed = 0
        o = O.tm_eigenvalues(oe, lat, d, fixed, O.TMParams())
        g = ge.tm_eigenvalues(d, fixed)
        np.testing.assert_allclose(np.abs(g), np.abs(o), rtol=1e-8, atol=1e-14)
    ge.close()
