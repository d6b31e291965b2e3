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
