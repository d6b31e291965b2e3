"""Shared driver: run the TE_TFI golden case through the oracle."""
import json
import os

import numpy as np

from oracle import tenes_oracle as O
from tenes_b200.input import load_input

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def oracle_setup(path):
    inp = load_input(path)
    ls = inp.lattice
    lat = O.Lattice(ls.LX, ls.LY, ls.skew)
    lat.physical_dims = ls.physical_dims
    lat.virtual_dims = ls.virtual_dims
    lat.initial_dirs = ls.initial_dirs
    lat.noises = ls.noises
    p = O.Params(CHI=inp.params.CHI, Max_CTM_Iteration=inp.params.Max_CTM_Iteration,
                 CTM_Convergence_Epsilon=inp.params.CTM_Convergence_Epsilon,
                 CTM_Projector_corner=inp.params.CTM_Projector_corner,
                 Use_RSVD=inp.params.Use_RSVD, seed=inp.params.seed)
    one = [O.OneSiteOp(o.name, o.group, o.source_site, o.op, o.coeff) for o in inp.onesite]
    two = [O.TwoSiteOp(o.name, o.group, o.source_site, o.dx[0], o.dy[0], o.op,
                       tuple(o.ops_indices), o.coeff) for o in inp.twosite]
    multi = [O.MultiSiteOp(o.name, o.group, o.source_site, tuple(o.dx), tuple(o.dy),
                           tuple(o.ops_indices), o.coeff) for o in inp.multisite]
    return inp, lat, p, one, two, multi


def su_step(inp, lat, p, Tn, lam, group=0):
    """One Trotter step: every evolution op of the group in input order
    (src/iTPS/simple_update.cpp:113-119, 25-46)."""
    for up in inp.simple_updates:
        if up.group != group:
            continue
        if up.is_onesite():
            Tn[up.source_site] = np.tensordot(Tn[up.source_site], up.op, ([4], [0]))
        else:
            s, leg = up.source_site, up.source_leg
            tg = lat.neighbor(s, leg)
            a, b, lc = O.simple_update_bond(Tn[s], Tn[tg], lam[s], lam[tg], up.op, leg, p)
            lam[s][leg] = lc
            lam[tg][(leg + 2) % 4] = lc
            Tn[s], Tn[tg] = a, b


def expected():
    with open(os.path.join(GOLDEN, "te_tfi_expected.json")) as f:
        return json.load(f)
