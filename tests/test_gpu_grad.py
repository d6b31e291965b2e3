"""GPU checks of the CTMRG energy gradient (tg_energy_grad).

* its forward energy equals the library's own sweep + window measurement;
* its gradient equals the FP64 host autograd reference (oracle/ctm_autograd.py)
  at small sizes, with uniform and uneven bond dimensions, with the
  environment zero-padded to chi, for corner and up/down projectors;
* the checkpoint interval changes nothing;
* central finite differences at the J1-J2 gradient workload's shapes
  (D = 3, chi = 36, 2 x 2, J2 = 0.5, normal(0,1) tensors);
* the 3xTF32 (mixed) gradient against the FP64 one;
* a few L-BFGS steps through the torch.autograd.Function lower the energy.
"""

import numpy as np
import pytest
import torch

from oracle import ctm_autograd as R
from tests.test_grad import lattice, random_tensors, uneven_dims, uniform_dims, _rel
from tenes_b200.env import CTMParams, Environment
from tenes_b200.grad import CTMEnergy, j1j2_terms, optimize_lbfgs

pytestmark = pytest.mark.gpu


def make(lat, Tn, chi, mixed=False, corner=True):
    env = Environment(lat.LX, lat.LY, lat.physical_dims, lat.virtual_dims,
                      CTMParams(chi=chi, max_ctm_iteration=1, mixed=mixed, projector_corner=corner), False)
    for i, t in enumerate(Tn):
        env.set_site_tensor(i, t)
    return env


def window_energy(env, terms):
    norms, E = {}, 0.0
    for t in terms:
        key = (t["source"], t["nrow"], t["ncol"], t["source_row"], t["source_col"])
        if key not in norms:
            norms[key] = env.contract_window(t["source"], t["nrow"], t["ncol"], t["source_row"],
                                             t["source_col"], {}).real
        E += t["coeff"] * env.contract_window(t["source"], t["nrow"], t["ncol"], t["source_row"],
                                              t["source_col"], t["ops"]).real / norms[key]
    return E


@pytest.mark.parametrize("corner", [True, False])
def test_energy_equals_sweeps_and_measurement(corner):
    rng = np.random.default_rng(1)
    lat = lattice(2, 2, uniform_dims(4, 3))
    Tn = random_tensors(lat, rng)
    terms = j1j2_terms(4, 1.0, 0.5)
    env = make(lat, Tn, 12, corner=corner)
    E, g = env.energy_grad(terms, 3, grad=False)
    assert g is None
    env.init_env()
    for _ in range(3):
        env.sweep()
    E2 = window_energy(env, terms)
    env.close()
    assert abs(E - E2) <= 1e-10 * abs(E2), (E, E2)


@pytest.mark.parametrize("uneven,chi,corner", [(False, 4, True), (False, 5, True), (True, 5, True),
                                               (False, 5, False), (True, 5, False)])
def test_gradient_matches_host_reference(uneven, chi, corner):
    """corner=False: the up/down projectors (ctm.cpp:320-491, full SVD)."""
    rng = np.random.default_rng(21 + chi + 7 * uneven)
    lat = lattice(2, 2, uniform_dims(4, 2))
    if uneven:
        lat.virtual_dims = uneven_dims(lat, rng)
    Tn = random_tensors(lat, rng)
    terms = j1j2_terms(4, 1.0, 0.5)
    iters = 3
    E_ref, g_ref = R.energy_and_grad(Tn, terms, chi, iters, lat, corner=corner)
    env = make(lat, Tn, chi, corner=corner)
    E, g = env.energy_grad(terms, iters, checkpoint_every=2)
    env.close()
    assert abs(E - E_ref) <= 1e-10 * abs(E_ref)
    assert _rel(g, g_ref) <= 1e-8, _rel(g, g_ref)


def test_checkpoint_interval_is_invisible():
    rng = np.random.default_rng(4)
    lat = lattice(2, 2, uniform_dims(4, 3))
    Tn = random_tensors(lat, rng)
    terms = j1j2_terms(4, 1.0, 0.5)
    env = make(lat, Tn, 10)
    res = [env.energy_grad(terms, 5, checkpoint_every=c) for c in (1, 2, 5, 100)]
    env.close()
    for E, g in res[1:]:
        assert abs(E - res[0][0]) <= 1e-13 * abs(E)
        assert _rel(g, res[0][1]) <= 1e-12


def _c4_problem(iters):
    rng = np.random.default_rng(2024)
    lat = lattice(2, 2, uniform_dims(4, 3))
    Tn = random_tensors(lat, rng)
    return lat, Tn, j1j2_terms(4, 1.0, 0.5)


def test_updown_gradient_matches_finite_differences():
    """The up/down projectors' adjoint against central differences (step
    1e-5) on 6 seeded entries: D = 2, chi = 8, 4 sweeps."""
    iters = 4
    rng = np.random.default_rng(77)
    lat = lattice(2, 2, uniform_dims(4, 2))
    Tn = random_tensors(lat, rng)
    terms = j1j2_terms(4, 1.0, 0.5)
    env = make(lat, Tn, 8, corner=False)
    E, g = env.energy_grad(terms, iters, checkpoint_every=2)
    gmax = max(np.abs(x).max() for x in g)
    h = 1e-5
    for _ in range(6):
        site = int(rng.integers(4))
        idx = tuple(int(rng.integers(n)) for n in Tn[site].shape)
        vals = []
        for s in (+1, -1):
            T = [t.copy() for t in Tn]
            T[site][idx] += s * h
            for i, t in enumerate(T):
                env.set_site_tensor(i, t)
            vals.append(env.energy_grad(terms, iters, grad=False)[0])
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - g[site][idx]) <= 1e-6 * max(abs(fd), abs(g[site][idx]), 1e-3 * gmax), \
            (site, idx, fd, g[site][idx])
    env.close()


def test_finite_differences_at_the_gradient_workload_shapes():
    """D = 3, chi = 36, J2 = 0.5; central differences, step 1e-5, on 8
    seeded entries; relative error 1e-6 (on the larger of the two values and
    a floor of 1e-3 of the gradient's largest entry)."""
    iters = 6
    lat, Tn, terms = _c4_problem(iters)
    env = make(lat, Tn, 36)
    E, g = env.energy_grad(terms, iters, checkpoint_every=3)
    gmax = max(np.abs(x).max() for x in g)
    rng = np.random.default_rng(7)
    h = 1e-5
    for _ in range(8):
        site = int(rng.integers(4))
        idx = tuple(int(rng.integers(n)) for n in Tn[site].shape)
        vals = []
        for s in (+1, -1):
            T = [t.copy() for t in Tn]
            T[site][idx] += s * h
            for i, t in enumerate(T):
                env.set_site_tensor(i, t)
            vals.append(env.energy_grad(terms, iters, grad=False)[0])
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - g[site][idx]) <= 1e-6 * max(abs(fd), abs(g[site][idx]), 1e-3 * gmax), \
            (site, idx, fd, g[site][idx])
    env.close()


def test_mixed_gradient_close_to_fp64():
    iters = 4
    lat, Tn, terms = _c4_problem(iters)
    env = make(lat, Tn, 36)
    E, g = env.energy_grad(terms, iters)
    env.close()
    envm = make(lat, Tn, 36, mixed=True)
    Em, gm = envm.energy_grad(terms, iters)
    envm.close()
    assert abs(Em - E) <= 1e-7  # |dE/site|, the mixed form's energy tolerance
    assert _rel(gm, g) <= 5e-3, _rel(gm, g)


def test_autograd_function_and_lbfgs_lower_the_energy():
    rng = np.random.default_rng(3)
    lat = lattice(2, 2, uniform_dims(4, 2))
    Tn = random_tensors(lat, rng)
    terms = j1j2_terms(4, 1.0, 0.5)
    env = make(lat, Tn, 8)
    params = [torch.tensor(t, requires_grad=True) for t in Tn]
    E = CTMEnergy.apply(env, terms, 3, 5, 1e-12, *params)
    E.backward()
    E_ref, g_ref = env.energy_grad(terms, 3)
    assert abs(float(E) - E_ref) <= 1e-13 * abs(E_ref)
    assert _rel([p.grad.numpy() for p in params], g_ref) <= 1e-13
    _, energies = optimize_lbfgs(env, Tn, terms, iterations=3, steps=4)
    env.close()
    assert energies[-1] < float(E) - 1e-3, (float(E), energies)
