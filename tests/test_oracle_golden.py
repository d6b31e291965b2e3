"""Pin the CPU oracle against the reference's own golden vectors.

* mt19937 draws from the C++ standard library (oracle/mt19937_draws.cpp).
* test/data/simple_update.dat: known answer of Simple_update_bond
  (test/simple_update.cpp:28-160, tol 1e-8 with the per-fibre sign gauge).
* test/data/full_update.dat: known answer of Full_update_bond
  (test/full_update.cpp:28-140, tol 1e-8 with the per-index sign gauge).
* test/data/output_TE_TFI: simple update + CTMRG + observables + correlation
  length.  The reference test compares at rtol 1e-3 / atol 1e-4
  (test/fulltest.py.in:141-142); the restatement reproduces it to 1e-10.
"""
import json
import math
import os

import numpy as np
import pytest

from oracle import tenes_oracle as O
from tests._te_tfi import GOLDEN, expected, oracle_setup, su_step


def test_mt19937_matches_libstdcxx():
    ref = json.load(open(os.path.join(GOLDEN, "mt19937_seed11.json")))["uniform_pm1"]
    g = O.MT19937(11)
    got = [O.uniform_pm1(g) for _ in range(len(ref))]
    assert got == ref


def test_simple_update_known_answer():
    kat = json.load(open(os.path.join(GOLDEN, "simple_update_kat.json")))
    D, d = kat["D"], kat["ldof"]
    T = np.ones((D, D, D, D, d))
    lam = [np.ones(D) for _ in range(4)]
    op = np.zeros((d, d, d, d))
    for i in range(d):
        op[i, i, i, i] = 1.0
    T1, T2, lc = O.simple_update_bond(T, T.copy(), lam, [l.copy() for l in lam], op,
                                      kat["connect"], O.Params())
    tol = kat["tol"]
    for new, ans in ((T1, kat["T1"]), (T2, kat["T2"])):
        ans = np.array(ans).reshape(D, D, D, D, d)
        for idx in np.ndindex(D, D, D, D):
            sign = 0
            for m in range(d):
                r, a = new[idx + (m,)], ans[idx + (m,)]
                if sign == 0 and r != 0.0:
                    sign = 1 if a * r > 0 else -1
                assert r * sign == pytest.approx(a, rel=tol, abs=1e-14)
    np.testing.assert_allclose(lc, kat["lambda"], rtol=tol)


def test_full_update_known_answer():
    """test/full_update.cpp:28-140: all-ones tensors and environment (the
    corners non-zero on their D x D block only), op12 = delta_{iiii},
    horizontal bond; the reference's check fixes one sign per physical index
    and tensor from the first non-zero entry."""
    kat = json.load(open(os.path.join(GOLDEN, "full_update_kat.json")))
    D, d, chi = kat["D"], kat["ldof"], kat["chi"]
    T = np.ones((D, D, D, D, d))
    C = []
    for _ in range(4):
        c = np.zeros((chi, chi))
        c[:D, :D] = 1.0
        C.append(c)
    E = [np.ones((chi, chi, D, D)) for _ in range(6)]
    op = np.zeros((d, d, d, d))
    for i in range(d):
        op[i, i, i, i] = 1.0
    T1, T2 = O.full_update_bond(*C, *E, T, T.copy(), op, kat["connect"], O.Params())
    for new, ans in ((T1, kat["T1"]), (T2, kat["T2"])):
        ans = np.array(ans).reshape(D, D, D, D, d)
        sign = np.zeros(d)
        for idx in np.ndindex(new.shape):
            m = idx[4]
            if sign[m] == 0 and new[idx] != 0.0:
                sign[m] = 1 if ans[idx] * new[idx] > 0 else -1
            assert new[idx] * sign[m] == pytest.approx(ans[idx], rel=kat["tol"], abs=1e-14)


def _match(t, rows, key_fn, val_fn, tol=1e-10):
    n = 0
    for r in rows:
        if abs(r[0] - t) > 1e-9:
            continue
        v = val_fn(r)
        assert abs(v.real - r[key_fn]) <= tol * max(1.0, abs(r[key_fn])), (t, r, v)
        n += 1
    return n


def test_te_tfi_golden():
    inp, lat, p, one, two, multi = oracle_setup(os.path.join(GOLDEN, "te_tfi_input.toml"))
    exp = expected()
    Tn = O.initialize_tensors(lat, inp.params.seed, inp.is_real)
    lam = [[np.ones(lat.virtual_dims[i][l]) for l in range(4)] for i in range(lat.N_UNIT)]
    n1 = max(o.group for o in one) + 1
    n2 = max(o.group for o in two) + 1
    n3 = max(o.group for o in multi) + 1
    bond_groups = [o.group for o in two if o.name == "bond_hamiltonian"]

    def measure(t):
        env, cnt, conv, sig = O.calc_ctm_environment(Tn, p, lat)
        v1, norm = O.measure_onesite(env, Tn, lat, one, n1)
        v2, _ = O.measure_twosite(env, Tn, lat, two, one, n2)
        v3 = O.measure_multisite(env, Tn, lat, multi, one, n3)
        E = sum(sum(v2[g].values()).real for g in set(bond_groups)) / lat.N_UNIT
        rows = [r for r in exp["density"] if abs(r[0] - t) < 1e-9 and int(r[1]) == 0]
        assert abs(E - rows[0][2]) < 1e-12
        n = _match(t, exp["onesite"], 3,
                   lambda r: norm[int(r[2])] if int(r[1]) == -1 else v1[int(r[1])][int(r[2])])
        n += _match(t, [r for r in exp["twosite"] if int(r[1]) >= 0], 5,
                    lambda r: v2[int(r[1])][(int(r[2]), int(r[3]), int(r[4]))])
        n += _match(t, exp["multisite"], 9,
                    lambda r: v3[int(r[1])][(int(r[2]), (int(r[3]), int(r[5]), int(r[7])),
                                             (int(r[4]), int(r[6]), int(r[8])))])
        assert n > 40
        if t > 0.99:
            for r in exp["correlation_length"]:
                if abs(r[0] - t) > 1e-9:
                    continue
                ev = O.tm_eigenvalues(env, lat, int(r[1]), int(r[2]), O.TMParams())
                L = lat.LX_noskew if int(r[1]) == 0 else lat.LY_noskew
                xi, es = O.correlation_length(ev, L)
                assert xi == pytest.approx(r[3], rel=1e-10)
                np.testing.assert_allclose(es, r[4:], rtol=1e-10)

    measure(0.0)
    t = 0.0
    for step in range(1, inp.params.num_simple_step[0] + 1):
        su_step(inp, lat, p, Tn, lam)
        t += inp.params.tau_simple_step[0]
        if step % inp.params.measure_interval[0] == 0:
            measure(t)


# observed deviation from the golden files: 1.4e-14 (afh_real), 1.5e-14
# (afh_complex), 1.2e-12 (honeycomb), 2.3e-6 (j1j2_afh, whose full-update
# gates change a site's physical dimension 2 -> 8 -> 2 along the sequence),
# 2.4e-5 (honeycomb_skew, the one skewed cell), 7e-15 (rsvd: rSVD up/down
# projectors at chi = 5, where k = 2 chi covers the rank of the projected
# matrices, so the random test matrix does not show); all inside the
# reference's own check (rtol 1e-3, atol 1e-4)
FU_GOLDEN_TOL = {"afh_real": 1e-11, "afh_complex": 1e-11, "honeycomb": 1e-10, "j1j2_afh": 1e-5,
                 "honeycomb_skew": 1e-4, "rsvd": 1e-11}


@pytest.mark.parametrize("stem", sorted(FU_GOLDEN_TOL))
def test_full_update_pipeline_golden(stem):
    """test/data/{AntiferroHeisenberg_real, J1J2_AFH, Honeycomb,
    Honeycomb_skew, AntiferroHeisenberg_complex, RSVD}: simple-update steps,
    full-update steps (fast full update: single moves after every bond,
    src/iTPS/full_update.cpp:30-186, preceded by a full CTMRG), then CTMRG
    and the observables (onesite_obs, twosite_obs, multisite_obs_4 and the
    energy of density.dat).  The reference checks at rtol 1e-3 / atol 1e-4."""
    with open(os.path.join(GOLDEN, stem + "_expected.json")) as f:
        exp = json.load(f)
    inp, lat, p, one, two, multi = oracle_setup(os.path.join(GOLDEN, stem + "_input.toml"))
    Tn = O.initialize_tensors(lat, inp.params.seed, inp.is_real)
    lam = [[np.ones(lat.virtual_dims[i][l]) for l in range(4)] for i in range(lat.N_UNIT)]
    for _ in range(inp.params.num_simple_step[0]):
        su_step(inp, lat, p, Tn, lam)
    env, _, _, _ = O.calc_ctm_environment(Tn, p, lat)
    for _ in range(inp.params.num_full_step[0]):
        for up in inp.full_updates:
            if up.group == 0:
                O.full_update_op(env, Tn, up.source_site, -1 if up.is_onesite() else up.source_leg, up.op, p, lat)
    env, _, _, _ = O.calc_ctm_environment(Tn, p, lat)
    n1 = max(o.group for o in one) + 1
    n2 = max(o.group for o in two) + 1
    v1, norm = O.measure_onesite(env, Tn, lat, one, n1)
    v2, _ = O.measure_twosite(env, Tn, lat, two, one, n2)
    v3 = O.measure_multisite(env, Tn, lat, multi, one, max(o.group for o in multi) + 1) if multi else None
    tol = FU_GOLDEN_TOL[stem]
    n = 0
    for r in exp["onesite"]:
        v = norm[int(r[1])] if int(r[0]) == -1 else v1[int(r[0])][int(r[1])]
        assert abs(v.real - r[2]) <= tol * max(1.0, abs(r[2])), (r, v)
        n += 1
    for r in exp["twosite"]:
        if int(r[0]) < 0:
            continue
        v = v2[int(r[0])][(int(r[1]), int(r[2]), int(r[3]))]
        assert abs(v.real - r[4]) <= tol * max(1.0, abs(r[4])), (r, v)
        n += 1
    for r in exp.get("multisite", []):
        v = v3[int(r[0])][(int(r[1]), (int(r[2]), int(r[4]), int(r[6])), (int(r[3]), int(r[5]), int(r[7])))]
        assert abs(v.real - r[8]) <= tol * max(1.0, abs(r[8])), (r, v)
        n += 1
    assert n > 10
