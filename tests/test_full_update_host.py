"""The library's full-update bond step (tenes_b200/csrc/full_update.hpp),
instantiated on host tensors by tests/fu_host_check.cpp (g++), against the
oracle's restatement (pinned to the reference's full_update.dat and the
AntiferroHeisenberg_real golden in test_oracle_golden.py).

The host backend's SVD and eigensolver may pick other signs and bases than
LAPACK; those change the new tensors only by a gauge on the updated bond, so
the comparison is on the bond-contracted pair Tn1_new . Tn2_new, and on the
number of least-squares iterations."""

import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import tenes_oracle as O
from tenes_b200.std_ops import evolution_twosite, heisenberg_bond

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# bond legs (Tn1 leg, Tn2 leg) for connect1 = 0..3
BOND = {0: (0, 2), 1: (1, 3), 2: (2, 0), 3: (3, 1)}


@pytest.fixture(scope="module")
def fu_exe(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    from tenes_b200.build import cuda_home
    out = str(tmp_path_factory.mktemp("fuhost") / "fu_host_check")
    subprocess.check_call([gxx, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                           "-I", os.path.join(ROOT, "tenes_b200", "csrc"), "-I", os.path.join(ROOT, "tests"),
                           "-I", os.path.join(cuda_home(), "include"),
                           os.path.join(ROOT, "tests", "fu_host_check.cpp"), "-o", out])
    return out


def run_host(exe, tensors, connect):
    cplx = any(np.iscomplexobj(t) for t in tensors)
    parts = ["complex" if cplx else "real"]
    for t in tensors:
        t = np.asarray(t, dtype=np.complex128 if cplx else np.float64)
        if cplx:
            vals = " ".join(f"{float(x.real)!r} {float(x.imag)!r}" for x in t.reshape(-1))
        else:
            vals = " ".join(repr(float(x)) for x in t.reshape(-1))
        parts.append(f"{t.ndim} " + " ".join(str(d) for d in t.shape) + " " + vals)
    parts.append(str(connect))
    out = subprocess.run([exe], input="\n".join(parts) + "\n", capture_output=True, text=True,
                         check=True).stdout.splitlines()
    st = out[0].split()
    res = []
    for ln in out[1:3]:
        w = ln.split()
        r = int(w[1])
        shape = tuple(int(x) for x in w[2:2 + r])
        v = np.array([float(x) for x in w[2 + r:]])
        res.append((v[0::2] + 1j * v[1::2] if cplx else v).reshape(shape))
    return int(st[1]), bool(int(st[2])), res[0], res[1]


def pair(a, b, connect):
    la, lb = BOND[connect]
    return np.tensordot(a, b, ([la], [lb]))


def test_known_answer_inputs(fu_exe):
    D, d, chi = 2, 2, 4
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
    ra, rb = O.full_update_bond(*C, *E, T, T.copy(), op, 2, O.Params())
    it, conv, a, b = run_host(fu_exe, C + E + [T, T, op], 2)
    np.testing.assert_allclose(pair(a, b, 2), pair(ra, rb, 2), rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("is_complex", [False, True])
@pytest.mark.parametrize("leg", [0, 1, 2, 3])
def test_bond_in_a_ctm_environment(fu_exe, leg, is_complex):
    """Each bond direction of a 2x2 cell in the environment of a few CTMRG
    sweeps (random D = 2 tensors, chi = 4), with exp(-0.1 H) of the
    Heisenberg bond; real and complex tensors."""
    rng = np.random.default_rng(31 + leg + 10 * is_complex)
    lat = O.Lattice(2, 2)
    lat.physical_dims = [2] * 4
    lat.virtual_dims = [[2] * 4 for _ in range(4)]
    Tn = [rng.standard_normal((2, 2, 2, 2, 2)) for _ in range(4)]
    if is_complex:
        Tn = [t + 1j * rng.standard_normal(t.shape) for t in Tn]
    p = O.Params(CHI=4)
    env = O.init_env(Tn, p, lat)
    for _ in range(3):
        O.sweep(env, Tn, p, lat)
    op = evolution_twosite(heisenberg_bond(1.0), 0.1)
    op = op if is_complex else op.real
    source = 1
    tgt = lat.neighbor(source, leg)
    args = O.full_update_env_args(env, source, leg, lat)
    ref = O.full_update_bond_horizontal  # iteration count of the oracle
    r = O._FU_ROT[leg]
    _, _, it_ref, conv_ref = ref(*args, Tn[source].transpose(r), Tn[tgt].transpose(r), op, p)
    ra, rb = O.full_update_bond(*args, Tn[source], Tn[tgt], op, leg, p)
    it, conv, a, b = run_host(fu_exe, list(args) + [Tn[source], Tn[tgt], op], leg)
    assert a.shape == ra.shape and b.shape == rb.shape
    assert (it, conv) == (it_ref, conv_ref)
    np.testing.assert_allclose(pair(a, b, leg), pair(ra, rb, leg), rtol=1e-8, atol=1e-12)
