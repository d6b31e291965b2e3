"""Shared fixtures for the GPU parity tests."""
import numpy as np

from oracle import tenes_oracle as O
from tenes_b200.env import CTMParams, Environment

SZ = np.diag([0.5, -0.5])
SX = np.array([[0.0, 0.5], [0.5, 0.0]])
SY = np.array([[0.0, -0.5j], [0.5j, 0.0]])


def random_tensors(lat, seed, is_complex=False, dist="uniform"):
    rng = np.random.default_rng(seed)
    Tn = []
    for i in range(lat.N_UNIT):
        v = lat.virtual_dims[i]
        sh = (v[0], v[1], v[2], v[3], lat.physical_dims[i])
        if dist == "uniform":
            T = rng.uniform(-1, 1, sh)
            if is_complex:
                T = T + 1j * rng.uniform(-1, 1, sh)
        else:
            T = rng.standard_normal(sh)
            if is_complex:
                T = T + 1j * rng.standard_normal(sh)
        Tn.append(T / np.max(np.abs(T)))
    return Tn


def make_lattice(LX, LY, D, d=2, skew=0):
    lat = O.Lattice(LX, LY, skew)
    lat.physical_dims = [d] * lat.N_UNIT
    lat.virtual_dims = [[D] * 4 for _ in range(lat.N_UNIT)]
    return lat


def gpu_env(lat, Tn, chi, is_complex=False, **kw):
    p = CTMParams(chi=chi, **kw)
    env = Environment(lat.LX, lat.LY, lat.physical_dims, lat.virtual_dims, p, is_complex, skew=lat.skew)
    for i, T in enumerate(Tn):
        env.set_site_tensor(i, T)
    return env


def oracle_params(chi, **kw):
    return O.Params(CHI=chi, **kw)


def load_env(genv, oenv):
    for w, name in enumerate(("C1", "C2", "C3", "C4", "eTt", "eTr", "eTb", "eTl")):
        for i, t in enumerate(getattr(oenv, name)):
            genv.set_env(w, i, t)


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


def physical_tensors(lat, D, steps=40, tau=0.05, seed=3, is_complex=False):
    """Site tensors from `steps` simple-update steps of the spin-1/2 Heisenberg
    model (oracle), from a seeded random start: spectra decay like a physical
    state's, unlike i.i.d. random tensors."""
    from tenes_b200.std_ops import evolution_twosite, heisenberg_bond
    op = evolution_twosite(heisenberg_bond(1.0), tau)
    op = op if is_complex else op.real
    Tn = random_tensors(lat, seed, is_complex)
    lam = [[np.ones(D) for _ in range(4)] for _ in range(lat.N_UNIT)]
    p = O.Params()
    for _ in range(steps):
        for s in range(lat.N_UNIT):
            for leg in (2, 1):
                tg = lat.neighbor(s, leg)
                a, b, lc = O.simple_update_bond(Tn[s], Tn[tg], lam[s], lam[tg], op, leg, p)
                lam[s][leg] = lc
                lam[tg][(leg + 2) % 4] = lc
                Tn[s], Tn[tg] = a, b
    return [T / np.max(np.abs(T)) for T in Tn]
