"""Shared driver: run a finite-temperature golden case through the oracle
(iTPS::finite_temperature, src/iTPS/finite_temperature.cpp:22-86, with
measure_density, measure.cpp:110-144) and compare each measurement with the
reference's output rows."""
import json
import os

import numpy as np

from oracle import tenes_density as D
from oracle import tenes_oracle as O
from tests._te_tfi import GOLDEN, oracle_setup


def expected(stem):
    with open(os.path.join(GOLDEN, stem + "_expected.json")) as f:
        return json.load(f)


def fix_gauge_density(Tn, lam, lat, p, maxiter, eps):
    """fix_local_gauge_density (simple_update.cpp:180-256): the pure-state
    gauge fixing on the tensors with their physical legs merged."""
    flat = [t.reshape(t.shape[:4] + (t.shape[4] * t.shape[5],)) for t in Tn]
    O.fix_local_gauge(flat, lam, lat, p, maxiter, eps)
    for i, t in enumerate(flat):
        Tn[i] = t.reshape(Tn[i].shape)


def measure(inp, lat, p, one, two, multi, Tn):
    """One measure_density: the environment from scratch, then the one-site,
    two-site and multisite values, norms and correlations."""
    env, cnt, conv, sig = D.calc_ctm_environment(Tn, p, lat)
    n1 = max(o.group for o in one) + 1
    v1, norm = D.measure_onesite(env, Tn, lat, one, n1)
    n2 = max(o.group for o in two) + 1 if two else 0
    v2, norms2 = D.measure_twosite(env, Tn, lat, two, one, n2) if two else ([], {})
    v3 = D.measure_multisite(env, Tn, lat, multi, one, max(o.group for o in multi) + 1) if multi else []
    return env, v1, norm, v2, norms2, v3


def correlations(inp, lat, env, Tn, one):
    """measure_correlation_ctm rows (left_op, left_site, right_op, dx, dy) ->
    value, for the input's [correlation] block."""
    cp = inp.corparam
    out = {}
    ops = {}
    for o in one:
        ops[(o.site, o.group)] = o.op
    r_ops = {}
    for a, b in cp.operators:
        r_ops.setdefault(a, []).append(b)
    for left in range(lat.N_UNIT):
        for lop, rlist in r_ops.items():
            if (left, lop) not in ops:
                continue
            for vertical in (False, True):
                res = D.correlation_strip(env, Tn, lat, left, vertical, cp.r_max, ops[(left, lop)],
                                          lambda s, rl=rlist: [ops[(s, r)] for r in rl])
                for r in range(cp.r_max):
                    for k, rop in enumerate(rlist):
                        key = (lop, left, rop, 0 if vertical else r + 1, r + 1 if vertical else 0)
                        out[key] = res[r][k]
    return out


def run(stem, on_measure, steps=None):
    """Run the case; on_measure(beta, inp, lat, p, one, two, multi, Tn) at
    every measurement.  `steps` truncates the Trotter steps of group 0."""
    inp, lat, p, one, two, multi = oracle_setup(os.path.join(GOLDEN, stem + "_input.toml"))
    Tn = D.initial_density(lat, inp.is_real)
    lam = [[np.ones(lat.virtual_dims[i][l]) for l in range(4)] for i in range(lat.N_UNIT)]
    beta = 0.0
    on_measure(beta, inp, lat, p, one, two, multi, Tn)
    groups = max(up.group for up in inp.simple_updates) + 1
    intervals = list(inp.params.measure_interval)
    while len(intervals) < groups:
        intervals.append(intervals[-1])
    for g in range(groups):
        nsteps = inp.params.num_simple_step[g]
        if steps is not None:
            nsteps = min(nsteps, steps)
        dt = inp.params.tau_simple_step[g]
        iv = intervals[g]
        for k in range(nsteps):
            for up in inp.simple_updates:
                if up.group == g:
                    D.su_density(Tn, lam, lat, up, p)
            beta += 2.0 * dt
            if inp.params.Simple_Gauge_Fix:
                fix_gauge_density(Tn, lam, lat, p, inp.params.Simple_Gauge_maxiter,
                                  inp.params.Simple_Gauge_Convergence_Epsilon)
            if (k + 1) % iv == 0:
                on_measure(beta, inp, lat, p, one, two, multi, Tn)
        if iv == 0 or nsteps % iv != 0:
            on_measure(beta, inp, lat, p, one, two, multi, Tn)
    return Tn, lam
