"""Parity at the workload configurations: the CUDA path against the FP64
oracle on the same seeded inputs, at the sizes the workloads name.

* c1: transverse-field Ising, 2x2, D=2, chi=10: 1000 simple-update steps at
  tau=0.01 (bond -SzSz, field -Sx as one-site operators), then exactly 10
  CTMRG iterations; energy per site, <Sz>, <Sx>, corner spectra.
* c2: Heisenberg, 2x2, D=4, chi=32, Neel + noise 1e-2 through
  iTPS::initialize_tensors (seed 11): 200 simple-update steps, then CTMRG
  (at most 30 iterations, reference convergence check); energy per site,
  staggered magnetisation, the 4 leading row transfer-matrix eigenvalues and
  the correlation length.
* c3: Heisenberg, 2x2, D=6, chi=72: one FP64 full-SVD Left_move from a
  non-trivial environment (gauge-invariant outputs after the move).
* initialize_tensors: the library's mt19937 draws equal the oracle's bit for
  bit (src/iTPS/tensors.cpp:83-128).

Tolerance: 1e-10 relative on gauge-invariant outputs (1e-12 absolute floor for
quantities that vanish); a normalised corner spectrum is compared as one
vector, 1e-10 in relative 2-norm."""
import numpy as np
import pytest

from oracle import tenes_oracle as O
from tenes_b200.env import CTMParams, Environment
from tenes_b200.std_ops import (evolution_onesite, evolution_twosite, heisenberg_bond, ising_bond,
                                real_if_close, spin_ops, two_site)
from tests._helpers import SX, SZ, gpu_env, load_env, make_lattice, rel

pytestmark = pytest.mark.gpu
TOL = 1e-10
TAU = 0.01
BONDS = [(s, 2) for s in range(4)] + [(s, 1) for s in range(4)]


def _neel(lat):
    lat.initial_dirs = [[1.0, 0.0] if ((i % lat.LX) + (i // lat.LX)) % 2 == 0 else [0.0, 1.0]
                        for i in range(lat.N_UNIT)]
    return lat.initial_dirs


def _oracle_su(lat, Tn, steps, bond_op, site_op=None):
    Tn = [t.copy() for t in Tn]
    lam = [[np.ones(lat.virtual_dims[i][l]) for l in range(4)] for i in range(lat.N_UNIT)]
    p = O.Params()
    for _ in range(steps):
        for s, leg in BONDS:
            tg = lat.neighbor(s, leg)
            a, b, lc = O.simple_update_bond(Tn[s], Tn[tg], lam[s], lam[tg], bond_op, leg, p)
            lam[s][leg] = lc
            lam[tg][(leg + 2) % 4] = lc
            Tn[s], Tn[tg] = a, b
        if site_op is not None:
            for s in range(lat.N_UNIT):
                # iTPS::simple_update, one-site: tensordot(Tn, op, Axes(4), Axes(0)) (simple_update.cpp:27-30)
                Tn[s] = np.tensordot(Tn[s], site_op, ([4], [0]))
    return Tn, lam


def _gpu_su(env, steps, bond_op, site_op=None):
    for _ in range(steps):
        for s, leg in BONDS:
            env.simple_update(s, leg, bond_op)
        if site_op is not None:
            for s in range(env.N):
                env.simple_update(s, -1, site_op)


def _oracle_bond(oe, Tn, lat, i, dx, op12):
    """Contract_two_sites_{horizontal,vertical}_op12 of the bond (i, right) or (i, top)."""
    if dx:
        j = lat.right(i)
        args = (oe.C1[i], oe.C2[j], oe.C3[j], oe.C4[i], oe.eTt[i], oe.eTt[j], oe.eTr[j],
                oe.eTb[j], oe.eTb[i], oe.eTl[i], Tn[i], Tn[j])
        f = O.contract_two_sites_horizontal_op12
    else:
        j = lat.top(i)
        args = (oe.C1[j], oe.C2[j], oe.C3[i], oe.C4[i], oe.eTt[j], oe.eTr[j], oe.eTr[i],
                oe.eTb[i], oe.eTl[i], oe.eTl[j], Tn[j], Tn[i])
        f = O.contract_two_sites_vertical_op12
    one = np.einsum("ac,bd->abcd", np.eye(2), np.eye(2))
    return (f(*args, op12) / f(*args, one)).real


def _gpu_bond(ge, i, dx, op12):
    rho = ge.contract_bond_rdm(i, dx, 1 - dx)
    return (np.sum(op12 * rho) / np.einsum("abab->", rho)).real


def _oracle_site(oe, Tn, i, op):
    a = (oe.C1[i], oe.C2[i], oe.C3[i], oe.C4[i], oe.eTt[i], oe.eTr[i], oe.eTb[i], oe.eTl[i], Tn[i])
    return (O.contract_one_site(*a, op) / O.contract_one_site(*a, np.eye(2))).real


def _gpu_site(ge, i, op):
    return (ge.contract_one_site(i, op) / ge.contract_one_site(i, np.eye(2))).real


def _close(g, o, what, tol=TOL, floor=1e-12):
    g, o = np.asarray(g, dtype=float), np.asarray(o, dtype=float)
    err = np.abs(g - o)
    ok = np.all(err <= tol * np.abs(o) + floor)
    assert ok, f"{what}: max abs err {err.max():.3e}, values {g} vs {o}"


def _spectrum_close(g, o, what, tol=TOL):
    """A normalised corner spectrum as one vector: ||g - o||_2 <= tol ||o||_2
    (its small tail values carry the absolute error of the whole vector)."""
    g, o = np.asarray(g, dtype=float), np.asarray(o, dtype=float)
    err = np.linalg.norm(g - o) / np.linalg.norm(o)
    assert err <= tol, f"{what}: relative 2-norm error {err:.3e}"


@pytest.mark.parametrize("is_complex", [False, True])
def test_init_tensors_bit_exact(is_complex):
    """tg_init_tensors (host std::mt19937 + uniform_real_distribution, uploaded)
    equals O.initialize_tensors bit for bit: uneven virtual dimensions, one
    site with a zero initial state (random direction drawn from the stream)."""
    lat = O.Lattice(2, 2)
    lat.physical_dims = [2, 3, 2, 3]
    lat.virtual_dims = [[2, 3, 4, 3], [4, 2, 2, 3], [2, 3, 4, 3], [4, 3, 2, 2]]
    dirs = [[1.0, 0.0], [0.0, 0.0, 0.0], [0.3, -0.7], [0.0, 1.0, 0.0]]
    noises = [0.1, 0.02, 1.0, 0.5]
    lat.initial_dirs, lat.noises = dirs, noises
    for seed in (11, 12345):
        want = O.initialize_tensors(lat, seed, not is_complex)
        env = Environment(2, 2, lat.physical_dims, lat.virtual_dims, CTMParams(chi=4), is_complex)
        env.init_tensors(seed, dirs, noises)
        for i in range(4):
            got = env.get_site_tensor(i)
            assert got.shape == want[i].shape
            assert np.array_equal(got, want[i]), f"site {i}, seed {seed}"
        env.close()


def test_c1_tfi_pipeline():
    """c1 end to end: the same seeded start, 1000 simple-update steps and 10
    CTMRG iterations on each side; then the oracle's CTMRG from the GPU's
    simple-update tensors, so that the CTMRG comparison holds the inputs
    fixed."""
    D, chi, hx = 2, 10, 1.0
    lat = make_lattice(2, 2, D)
    rng = np.random.default_rng(11)
    T0 = []
    for _ in range(4):
        t = rng.uniform(-1.0, 1.0, (D, D, D, D, 2))
        T0.append(t / np.abs(t).max())
    Sz, Sx, _ = spin_ops(0.5)
    bond = real_if_close(evolution_twosite(ising_bond(1.0), TAU))
    site = real_if_close(evolution_onesite(-hx * Sx, TAU))
    To, lam_o = _oracle_su(lat, T0, 1000, bond, site)
    ge = gpu_env(lat, T0, chi, False, max_ctm_iteration=10, ctm_convergence_epsilon=1e-30)
    _gpu_su(ge, 1000, bond, site)
    for s in range(4):
        for leg in range(4):
            _close(ge.get_lambda(s, leg), lam_o[s][leg], f"lambda[{s}][{leg}]")
    Tg = [ge.get_site_tensor(i) for i in range(4)]
    p = O.Params(CHI=chi, Max_CTM_Iteration=10, CTM_Convergence_Epsilon=1e-30)
    hb = real_if_close(ising_bond(1.0))
    gcnt, _, _ = ge.calc_ctm_environment(True)
    assert gcnt == 10

    def energy(site_val, bond_val):
        return (sum(bond_val(i, dx, hb) for i in range(4) for dx in (1, 0))
                - hx * sum(site_val(i, SX) for i in range(4))) / 4

    e_g = energy(lambda i, op: _gpu_site(ge, i, op), lambda i, dx, h: _gpu_bond(ge, i, dx, h))
    sz_g = [_gpu_site(ge, i, SZ) for i in range(4)]
    sx_g = [_gpu_site(ge, i, SX) for i in range(4)]
    spec_g = [[ge.corner_spectrum(w, i) for i in range(4)] for w in range(4)]
    for Ttag, Tset in (("oracle tensors", To), ("GPU tensors", Tg)):
        oe, ocnt, _, _ = O.calc_ctm_environment(Tset, p, lat)
        assert ocnt == 10
        e_o = energy(lambda i, op: _oracle_site(oe, Tset, i, op),
                     lambda i, dx, h: _oracle_bond(oe, Tset, lat, i, dx, h))
        _close(e_g, e_o, f"E/site ({Ttag})")
        _close(sz_g, [_oracle_site(oe, Tset, i, SZ) for i in range(4)], f"<Sz> ({Ttag})")
        _close(sx_g, [_oracle_site(oe, Tset, i, SX) for i in range(4)], f"<Sx> ({Ttag})")
        for w, name in enumerate(("C1", "C2", "C3", "C4")):
            for i in range(4):
                _spectrum_close(spec_g[w][i], O.corner_spectrum(getattr(oe, name)[i]),
                                f"{name}[{i}] spectrum ({Ttag})")
    ge.close()


def test_c2_afh_pipeline():
    """c2 end to end: Neel + noise 1e-2 through initialize_tensors (seed 11),
    200 simple-update steps, CTMRG with the reference's convergence check (at
    most 30 iterations), then energy, staggered magnetisation and the row
    transfer matrix's leading eigenvalues: the GPU's restarted Arnoldi run to
    convergence against the oracle's dense eigensolver of the same 1024 x 1024
    matrix, and the reference's default Arnoldi (one pass) on both sides."""
    D, chi = 4, 32
    lat = make_lattice(2, 2, D)
    dirs = _neel(lat)
    lat.noises = [1e-2] * 4
    T0 = O.initialize_tensors(lat, 11, True)
    bond = real_if_close(evolution_twosite(heisenberg_bond(1.0), TAU))
    To, lam_o = _oracle_su(lat, T0, 200, bond)
    ge = Environment(2, 2, lat.physical_dims, lat.virtual_dims, CTMParams(chi=chi, max_ctm_iteration=30), False)
    ge.init_tensors(11, dirs, lat.noises)
    for i in range(4):
        assert np.array_equal(ge.get_site_tensor(i), T0[i])
    _gpu_su(ge, 200, bond)
    for s in range(4):
        for leg in range(4):
            _close(ge.get_lambda(s, leg), lam_o[s][leg], f"lambda[{s}][{leg}]")
    Tg = [ge.get_site_tensor(i) for i in range(4)]
    gcnt, gconv, _ = ge.calc_ctm_environment(True)
    oe, ocnt, oconv, _ = O.calc_ctm_environment(Tg, O.Params(CHI=chi, Max_CTM_Iteration=30), lat)
    assert (gcnt, gconv) == (ocnt, oconv)
    h = real_if_close(heisenberg_bond(1.0))
    e_g = sum(_gpu_bond(ge, i, dx, h) for i in range(4) for dx in (1, 0)) / 4
    e_o = sum(_oracle_bond(oe, Tg, lat, i, dx, h) for i in range(4) for dx in (1, 0)) / 4
    _close(e_g, e_o, "E/site")
    sign = [1.0 if ((i % 2) + (i // 2)) % 2 == 0 else -1.0 for i in range(4)]
    m_g = sum(sign[i] * _gpu_site(ge, i, SZ) for i in range(4)) / 4
    m_o = sum(sign[i] * _oracle_site(oe, Tg, i, SZ) for i in range(4)) / 4
    _close(m_g, m_o, "staggered m")
    for w, name in enumerate(("C1", "C2", "C3", "C4")):
        for i in range(4):
            _spectrum_close(ge.corner_spectrum(w, i), O.corner_spectrum(getattr(oe, name)[i]), f"{name}[{i}] spectrum")
    # row transfer matrix at y = 0: N = chi^2 = 1024 > 200 -> Arnoldi
    N = chi * chi
    M = np.stack([O.tm_matvec_horizontal(oe, lat, 0, e) for e in np.eye(N)], axis=1)
    dense = O._sorted_eigvals(M, 4)
    conv = ge.tm_eigenvalues(0, 0, 4, arnoldi_maxiter=200, arnoldi_rtol=1e-14)
    _close(np.abs(conv), np.abs(dense), "|lambda_i| (converged Arnoldi vs dense)")
    xi_g, _ = O.correlation_length(conv, 2)
    xi_o, _ = O.correlation_length(dense, 2)
    _close(xi_g, xi_o, "correlation length")
    # the reference's defaults (maxdim 50, restart 20, one pass): the same
    # Krylov process on both sides; one pass converges the leading pair
    # (which sets the correlation length), not every requested eigenvalue, so
    # only those two are compared
    g1 = ge.tm_eigenvalues(0, 0, 4)
    o1 = O.tm_eigenvalues(oe, lat, 0, 0, O.TMParams())
    np.testing.assert_allclose(np.abs(g1[:2]), np.abs(o1[:2]), rtol=1e-8)
    np.testing.assert_allclose(np.abs(o1[:2]), np.abs(dense[:2]), rtol=1e-8)
    ge.close()


def test_c3_full_svd_left_move():
    """c3 shapes (D=6, chi=72): one FP64 Left_move with full-SVD corner
    projectors (ctm.cpp:562-616, 267-302) from the environment of three rSVD
    sweeps, on the GPU and in the oracle; the moved corners' spectra and the
    one-site observables are compared (gauge invariant)."""
    D, chi = 6, 72
    lat = make_lattice(2, 2, D)
    dirs = _neel(lat)
    lat.noises = [1e-2] * 4
    bond = real_if_close(evolution_twosite(heisenberg_bond(1.0), TAU))
    prep = Environment(2, 2, lat.physical_dims, lat.virtual_dims,
                       CTMParams(chi=chi, max_ctm_iteration=1, use_rsvd=True, rsvd_oversample_abs=10), False)
    prep.init_tensors(11, dirs, lat.noises)
    _gpu_su(prep, 300, bond)
    Tn = [prep.get_site_tensor(i) for i in range(4)]
    prep.init_env()
    for _ in range(3):
        prep.sweep()
    oe = O.Env(*[[prep.get_env(w, i) for i in range(4)] for w in range(8)])
    prep.close()
    ge = gpu_env(lat, Tn, chi, False)
    load_env(ge, oe)
    O.left_move(oe, Tn, 0, O.Params(CHI=chi), lat)
    ge.move(0, 0)
    for w, name in enumerate(("C1", "C2", "C3", "C4")):
        for i in range(4):
            _spectrum_close(ge.corner_spectrum(w, i), O.corner_spectrum(getattr(oe, name)[i]), f"{name}[{i}] spectrum")
    for op, nm in ((SZ, "Sz"), (SX, "Sx")):
        _close([_gpu_site(ge, i, op) for i in range(4)], [_oracle_site(oe, Tn, i, op) for i in range(4)],
               f"<{nm}>")
    ge.close()
