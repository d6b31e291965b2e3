"""CPU checks of the CTMRG energy gradient.

* the closed-form SVD adjoint of the FP64 host reference against torch's own
  SVD autograd;
* the host reference's forward against the numpy oracle, its backward
  against central finite differences;
* the library's adjoint (tenes_b200/csrc/adjoint.hpp, instantiated on host
  tensors by tests/ad_host_check.cpp) against the host reference: energy,
  gradient, independence of the checkpoint interval, uneven bond dimensions
  (non-square projector matrices).
"""

import os
import shutil
import subprocess

import numpy as np
import pytest
import torch

from oracle import ctm_autograd as R
from oracle import tenes_oracle as O
from tenes_b200.grad import j1j2_terms, two_site_terms, window_geometry

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def lattice(LX, LY, vd, pd=2):
    lat = O.Lattice(LX, LY)
    lat.physical_dims = [pd] * lat.N_UNIT
    lat.virtual_dims = vd
    return lat


def uniform_dims(N, D):
    return [[D] * 4 for _ in range(N)]


def uneven_dims(lat, rng, choices=(2, 3)):
    """Per-bond dimensions, consistent between neighbours."""
    N = lat.N_UNIT
    h = [int(rng.choice(choices)) for _ in range(N)]  # bond between i and right(i)
    v = [int(rng.choice(choices)) for _ in range(N)]  # bond between i and top(i)
    return [[h[lat.left(i)], v[i], h[i], v[lat.bottom(i)]] for i in range(N)]


def random_tensors(lat, rng):
    return [rng.standard_normal(tuple(lat.virtual_dims[i]) + (lat.physical_dims[i],))
            for i in range(lat.N_UNIT)]


# ------------------------------------------------------------- SVD adjoint
@pytest.mark.parametrize("m,n", [(6, 6), (7, 5), (5, 7)])
def test_svd_backward_matches_torch_autograd(m, n):
    g = torch.Generator().manual_seed(m * 10 + n)
    M = torch.randn(m, n, dtype=torch.float64, generator=g)
    k = min(m, n)
    W1 = torch.randn(m, 3, dtype=torch.float64, generator=g)
    w = torch.randn(3, dtype=torch.float64, generator=g)
    W2 = torch.randn(3, n, dtype=torch.float64, generator=g)

    def loss(U, s, Vh):
        return (W1 * U[:, :3]).sum() + (w * s[:3]).sum() + (W2 * Vh[:3]).sum()

    A = M.clone().requires_grad_(True)
    U, s, Vh = torch.linalg.svd(A, full_matrices=False)
    (gt,) = torch.autograd.grad(loss(U, s, Vh), A)
    B = M.clone().requires_grad_(True)
    U2, s2, Vh2 = R.TruncSVD.apply(B, 0.0)
    (gm,) = torch.autograd.grad(loss(U2, s2, Vh2), B)
    assert k == s.numel()
    np.testing.assert_allclose(gm.numpy(), gt.numpy(), rtol=1e-9, atol=1e-11)


# --------------------------------------------------------- energy terms
def test_two_site_terms_reproduce_the_operator():
    from tenes_b200.std_ops import heisenberg_bond, real_if_close
    h = real_if_close(heisenberg_bond(1.0))
    terms = two_site_terms(0, 1, 0, h, 1.0)
    assert len(terms) == 3
    acc = np.zeros_like(h)
    for t in terms:
        (a, b) = [t["ops"][k] for k in sorted(t["ops"])]
        acc += np.einsum("ac,bd->abcd", a, b)
    np.testing.assert_allclose(acc, h, atol=1e-14)
    assert window_geometry(1, 0) == (1, 2, 0, 0, 0, 1)
    assert window_geometry(0, 1) == (2, 1, 1, 0, 0, 0)
    assert window_geometry(1, -1) == (2, 2, 0, 0, 1, 1)
    assert window_geometry(-1, 1) == (2, 2, 1, 1, 0, 0)


def _oracle_energy(Tn, terms, chi, iters, lat, corner=True):
    p = O.Params(CHI=chi, CTM_Projector_corner=corner)
    env = O.init_env(Tn, p, lat)
    for _ in range(iters):
        O.sweep(env, Tn, p, lat)
    norms = {}
    E = 0.0
    for t in terms:
        key = (t["source"], t["nrow"], t["ncol"], t["source_row"], t["source_col"])

        def val(ops):
            idx, C, eTt, eTr, eTb, eTl, T = O._window(env, Tn, lat, t["source"], t["source_col"],
                                                     t["source_row"], t["nrow"], t["ncol"])
            op = [[ops.get((r, c), np.eye(lat.physical_dims[idx[r][c]])) for c in range(t["ncol"])]
                  for r in range(t["nrow"])]
            return O.contract_window(C, eTt, eTr, eTb, eTl, T, op).real
        if key not in norms:
            norms[key] = val({})
        E += t["coeff"] * val(t["ops"]) / norms[key]
    return E


@pytest.mark.parametrize("corner", [True, False])
def test_reference_forward_matches_oracle(corner):
    rng = np.random.default_rng(3)
    lat = lattice(2, 2, uniform_dims(4, 2))
    Tn = random_tensors(lat, rng)
    terms = j1j2_terms(4, 1.0, 0.5)
    E0 = _oracle_energy(Tn, terms, 4, 2, lat, corner)
    with torch.no_grad():
        E1 = float(R.energy([torch.tensor(t) for t in Tn], terms, 4, 2, lat, corner=corner))
    assert abs(E1 - E0) <= 1e-11 * abs(E0)


@pytest.mark.parametrize("corner,chi", [(True, 4), (False, 4), (True, 8), (False, 8)])
def test_reference_gradient_matches_finite_differences(corner, chi):
    """chi = 8 > D^2: zero-padded first environments and, for the up/down
    projectors, matrices M = R1 R2 of small norm whose kept singular values
    span six decades -- the case an absolute Lorentzian broadening got wrong
    by up to 1.5% and the pair-relative one gets right."""
    rng = np.random.default_rng(5)
    lat = lattice(2, 2, uniform_dims(4, 2))
    Tn = random_tensors(lat, rng)
    terms = j1j2_terms(4, 1.0, 0.5)
    E, g = R.energy_and_grad(Tn, terms, chi, 2, lat, corner=corner)
    h = 1e-5
    for site, idx in [(0, (0, 1, 0, 1, 0)), (1, (1, 1, 1, 0, 1)), (2, (0, 0, 1, 1, 1)), (3, (1, 0, 0, 0, 0))]:
        def f(delta):
            T = [t.copy() for t in Tn]
            T[site][idx] += delta
            with torch.no_grad():
                return float(R.energy([torch.tensor(t) for t in T], terms, chi, 2, lat, corner=corner))
        fd = (f(h) - f(-h)) / (2 * h)
        assert abs(fd - g[site][idx]) <= 1e-6 * max(abs(fd), 1e-3), (site, idx, fd, g[site][idx])


# ------------------------------------------ the library adjoint on the host
@pytest.fixture(scope="module")
def host_adjoint(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    from tenes_b200.build import cuda_home
    out = str(tmp_path_factory.mktemp("adhost") / "ad_host_check")
    subprocess.check_call([gxx, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                           "-I", os.path.join(ROOT, "tenes_b200", "csrc"), "-I", os.path.join(ROOT, "tests"),
                           "-I", os.path.join(cuda_home(), "include"),
                           os.path.join(ROOT, "tests", "ad_host_check.cpp"), "-o", out])
    return out


def run_host(exe, lat, Tn, terms, chi, iters, ckpt, cutoff=1e-12, eps=1e-12, zero_null=False, corner=True):
    lines = [f"{lat.LX} {lat.LY} 0 {chi} {iters} {ckpt}", f"{cutoff!r} {eps!r}"]
    for i in range(lat.N_UNIT):
        lines.append(" ".join(str(x) for x in [lat.physical_dims[i]] + list(lat.virtual_dims[i])))
    for t in Tn:
        lines.append(" ".join(repr(float(x)) for x in t.reshape(-1)))
    lines.append(str(len(terms)))
    for t in terms:
        keys = sorted(t["ops"])
        lines.append(f"{t['source']} {t['nrow']} {t['ncol']} {t['source_row']} {t['source_col']} "
                     f"{t['coeff']!r} {len(keys)}")
        for k in keys:
            op = np.asarray(t["ops"][k], dtype=np.float64)
            lines.append(f"{k[0]} {k[1]} {op.shape[0]} " + " ".join(repr(float(x)) for x in op.reshape(-1)))
    res = subprocess.run([exe] + (["zero-null"] if zero_null else []) + ([] if corner else ["updown"]),
                         input="\n".join(lines) + "\n",
                         capture_output=True, text=True, check=True)
    out = res.stdout.splitlines()
    E = float(out[0].split()[1])
    g = [np.array([float(x) for x in ln.split()[1:]]).reshape(Tn[i].shape) for i, ln in enumerate(out[1:])]
    return E, g


def _rel(a, b):
    a = np.concatenate([x.reshape(-1) for x in a])
    b = np.concatenate([x.reshape(-1) for x in b])
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("corner", [True, False])
@pytest.mark.parametrize("uneven", [False, True])
def test_host_adjoint_matches_reference(host_adjoint, uneven, corner):
    rng = np.random.default_rng(11 if uneven else 7)
    lat = lattice(2, 2, uniform_dims(4, 2))
    if uneven:
        lat.virtual_dims = uneven_dims(lat, rng)
    Tn = random_tensors(lat, rng)
    terms = j1j2_terms(4, 1.0, 0.5)
    chi, iters = 5, 3
    E_ref, g_ref = R.energy_and_grad(Tn, terms, chi, iters, lat, corner=corner)
    E, g = run_host(host_adjoint, lat, Tn, terms, chi, iters, ckpt=2, corner=corner)
    assert abs(E - E_ref) <= 1e-10 * abs(E_ref)
    assert _rel(g, g_ref) <= 1e-8, _rel(g, g_ref)


def test_host_adjoint_checkpoint_interval_is_invisible(host_adjoint):
    rng = np.random.default_rng(9)
    lat = lattice(2, 2, uniform_dims(4, 2))
    Tn = random_tensors(lat, rng)
    terms = j1j2_terms(4, 1.0, 0.0)
    E1, g1 = run_host(host_adjoint, lat, Tn, terms, 4, 4, ckpt=1)
    E4, g4 = run_host(host_adjoint, lat, Tn, terms, 4, 4, ckpt=4)
    E3, g3 = run_host(host_adjoint, lat, Tn, terms, 4, 4, ckpt=3)
    assert E1 == E4 == E3
    for a, b, c in zip(g1, g4, g3):
        np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-15)
        np.testing.assert_allclose(a, c, rtol=1e-12, atol=1e-15)


def test_host_adjoint_does_not_use_null_space_vectors(host_adjoint):
    """chi > D^2 pads the first environments with zeros, so the projector
    matrices have exactly vanishing singular values; the adjoint must not
    depend on how the SVD completes their singular vectors."""
    rng = np.random.default_rng(13)
    lat = lattice(2, 2, uniform_dims(4, 2))
    Tn = random_tensors(lat, rng)
    terms = j1j2_terms(4, 1.0, 0.5)
    E1, g1 = run_host(host_adjoint, lat, Tn, terms, 6, 2, ckpt=1)
    E2, g2 = run_host(host_adjoint, lat, Tn, terms, 6, 2, ckpt=1, zero_null=True)
    assert abs(E1 - E2) <= 1e-12 * abs(E1)
    assert _rel(g2, g1) <= 1e-9, _rel(g2, g1)
