"""Simple update on the GPU against the reference KAT and the oracle, and the
TE_TFI golden (simple update + CTMRG + observables, complex) end to end."""
import json
import os

import numpy as np
import pytest

from oracle import tenes_oracle as O
from tests._helpers import gpu_env, make_lattice, random_tensors
from tests._te_tfi import GOLDEN, expected, oracle_setup

pytestmark = pytest.mark.gpu


def test_su_known_answer_on_gpu():
    kat = json.load(open(os.path.join(GOLDEN, "simple_update_kat.json")))
    D, d = kat["D"], kat["ldof"]
    lat = make_lattice(2, 1, D, d)
    T = np.ones((D, D, D, D, d))
    env = gpu_env(lat, [T, T], 4)
    op = np.zeros((d, d, d, d))
    for i in range(d):
        op[i, i, i, i] = 1.0
    env.simple_update(0, kat["connect"], op)
    np.testing.assert_allclose(env.get_lambda(0, 2), kat["lambda"], rtol=kat["tol"])
    np.testing.assert_allclose(env.get_lambda(1, 0), kat["lambda"], rtol=kat["tol"])
    for site, key in ((0, "T1"), (1, "T2")):
        new = env.get_site_tensor(site)
        ans = np.array(kat[key]).reshape(D, D, D, D, d)
        for idx in np.ndindex(D, D, D, D):
            sign = 0
            for m in range(d):
                r, a = new[idx + (m,)], ans[idx + (m,)]
                if sign == 0 and r != 0.0:
                    sign = 1 if a * r > 0 else -1
                assert abs(r * sign - a) <= kat["tol"] * abs(a) + 1e-12


@pytest.mark.parametrize("is_complex", [False, True])
@pytest.mark.parametrize("leg", [0, 1, 2, 3])
def test_su_bond_matches_oracle(is_complex, leg):
    lat = make_lattice(2, 2, 3)
    Tn = random_tensors(lat, 3 + leg, is_complex)
    rng = np.random.default_rng(9)
    lam = [[rng.uniform(0.2, 1.0, 3) for _ in range(4)] for _ in range(lat.N_UNIT)]
    H = rng.standard_normal((4, 4))
    if is_complex:
        H = H + 1j * rng.standard_normal((4, 4))
    H = H + H.conj().T
    w, v = np.linalg.eigh(H)
    op = (v @ np.diag(np.exp(-0.1 * w)) @ v.conj().T).reshape(2, 2, 2, 2)
    env = gpu_env(lat, Tn, 4, is_complex)
    for i in range(lat.N_UNIT):
        for l in range(4):
            env.set_lambda(i, l, lam[i][l])
    src = 0
    tgt = lat.neighbor(src, leg)
    a, b, lc = O.simple_update_bond(Tn[src], Tn[tgt], lam[src], lam[tgt], op, leg, O.Params())
    env.simple_update(src, leg, op)
    np.testing.assert_allclose(env.get_lambda(src, leg), lc, rtol=1e-11)
    # contracting the updated bond removes its gauge freedom
    ga, gb = env.get_site_tensor(src), env.get_site_tensor(tgt)
    g = np.tensordot(ga, gb, ([leg], [(leg + 2) % 4]))
    o = np.tensordot(a, b, ([leg], [(leg + 2) % 4]))
    np.testing.assert_allclose(g, o, rtol=1e-10, atol=1e-12 * np.max(np.abs(o)))


def test_te_tfi_golden_on_gpu():
    """Full TE_TFI flow through the C ABI: the reference golden at 1e-10."""
    inp, lat, p, one, two, multi = oracle_setup(os.path.join(GOLDEN, "te_tfi_input.toml"))
    exp = expected()
    Tn = O.initialize_tensors(lat, inp.params.seed, inp.is_real)
    env = gpu_env(lat, Tn, inp.params.CHI, not inp.is_real, max_ctm_iteration=inp.params.Max_CTM_Iteration)
    sz = [o for o in one if o.name == "Sz"]

    def measure(t):
        env.calc_ctm_environment(True)
        for o in sz:
            nrm = env.contract_one_site(o.site, np.eye(2))
            v = (env.contract_one_site(o.site, o.op) / nrm).real
            ref = [r for r in exp["onesite"] if abs(r[0] - t) < 1e-9 and int(r[1]) == o.group
                   and int(r[2]) == o.site][0]
            assert abs(v - ref[3]) < 1e-10 * max(1, abs(ref[3]))
        E = 0.0
        for o in two:
            if o.name != "bond_hamiltonian":
                continue
            ident = np.einsum("ac,bd->abcd", np.eye(2), np.eye(2))
            E += (env.contract_bond_op12(o.source, o.dx, o.dy, o.op)
                  / env.contract_bond_op12(o.source, o.dx, o.dy, ident)).real
        E /= lat.N_UNIT
        ref = [r for r in exp["density"] if abs(r[0] - t) < 1e-9 and int(r[1]) == 0][0]
        assert abs(E - ref[2]) < 1e-10

    measure(0.0)
    t = 0.0
    for step in range(1, inp.params.num_simple_step[0] + 1):
        for up in inp.simple_updates:
            env.simple_update(up.source_site, up.source_leg, up.op)
        t += inp.params.tau_simple_step[0]
        if step % inp.params.measure_interval[0] == 0:
            measure(t)


@pytest.mark.parametrize("is_complex", [False, True])
def test_batched_steps_equal_single_steps(is_complex):
    """tg_su_bonds (runs of site-disjoint bond steps as one launch) gives the
    same tensors and weights, bit for bit, as the same steps one call at a
    time, one-site operators in between included; a 2x2 and a 4x2 cell."""
    from tenes_b200.std_ops import evolution_onesite, evolution_twosite, heisenberg_bond, spin_ops
    _, Sx, _ = spin_ops(0.5)
    bond = evolution_twosite(heisenberg_bond(1.0), 0.05)
    site = evolution_onesite(-0.3 * Sx, 0.05)
    if not is_complex:
        bond, site = bond.real, site.real
    for LX, LY in ((2, 2), (4, 2)):
        lat = make_lattice(LX, LY, 3)
        Tn = random_tensors(lat, 21, is_complex)
        steps = [(s, 2, bond) for s in range(lat.N_UNIT)] + [(s, 1, bond) for s in range(lat.N_UNIT)]
        steps += [(s, -1, site) for s in range(lat.N_UNIT)]
        one, many = gpu_env(lat, Tn, 4, is_complex), gpu_env(lat, Tn, 4, is_complex)
        for _ in range(3):
            for s, leg, op in steps:
                one.simple_update(s, leg, op)
            many.simple_update_many(steps)
        for i in range(lat.N_UNIT):
            assert np.array_equal(one.get_site_tensor(i), many.get_site_tensor(i)), i
            for leg in range(4):
                assert np.array_equal(one.get_lambda(i, leg), many.get_lambda(i, leg)), (i, leg)
        one.close()
        many.close()
