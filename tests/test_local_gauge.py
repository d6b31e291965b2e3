"""Local gauge fixing of the simple update (core::fix_local_gauge,
src/iTPS/core/local_gauge.cpp:44-224; iTPS::fix_local_gauge,
src/iTPS/simple_update.cpp:49-101).

The reference's tests hold no fixture for it and its source needs mptensor,
so the oracle's restatement is checked through the properties that define the
transform: one bond step leaves the state unchanged up to a positive scale
(the bond-contracted pair Tn1_new . Tn2_new is proportional to Tn1 . Tn2, the
weights being absorbed in the site tensors as the simple update leaves them;
the scale comes from renormalising the new weights), and the sweeps drive every
boundary tensor to the identity.  The library's template
(tenes_b200/csrc/local_gauge.hpp), instantiated on host tensors by
tests/gauge_host_check.cpp, is compared with the oracle: sweep count, score
and bond weights, which the SVD and eigensolver sign choices leave alone."""

import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import tenes_oracle as O
from tenes_b200.std_ops import evolution_twosite, heisenberg_bond

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def su_state(is_complex, D=3, steps=20, seed=0):
    """A 2 x 2 cell after simple-update steps of exp(-0.1 H), Heisenberg."""
    rng = np.random.default_rng(seed)
    lat = O.Lattice(2, 2)
    lat.physical_dims = [2] * 4
    lat.virtual_dims = [[D] * 4 for _ in range(4)]
    Tn = [rng.standard_normal((D, D, D, D, 2)) for _ in range(4)]
    if is_complex:
        Tn = [t + 1j * rng.standard_normal(t.shape) for t in Tn]
    lam = [[np.ones(D) for _ in range(4)] for _ in range(4)]
    p = O.Params()
    op = evolution_twosite(heisenberg_bond(1.0), 0.1)
    op = op if is_complex else op.real
    for _ in range(steps):
        for s in range(4):
            for leg in (2, 1):
                t = lat.neighbor(s, leg)
                a, b, lc = O.simple_update_bond(Tn[s], Tn[t], lam[s], lam[t], op, leg, p)
                Tn[s], Tn[t] = a, b
                lam[s][leg] = lc
                lam[t][(leg + 2) % 4] = lc
    return lat, Tn, lam, p


@pytest.mark.parametrize("is_complex", [False, True])
@pytest.mark.parametrize("leg", [0, 1, 2, 3])
def test_bond_step_keeps_the_state(is_complex, leg):
    lat, Tn, lam, p = su_state(is_complex)
    s = 1
    t = lat.neighbor(s, leg)
    c2 = (leg + 2) % 4
    a, b, lc = O.local_gauge_bond(Tn[s], Tn[t], lam[s], lam[t], leg, p)
    new, old = np.tensordot(a, b, ([leg], [c2])), np.tensordot(Tn[s], Tn[t], ([leg], [c2]))
    # the same state up to the positive scale of renormalising lambda_c
    np.testing.assert_allclose(new / np.linalg.norm(new), old / np.linalg.norm(old), rtol=1e-9, atol=1e-12)
    assert abs(np.sum(lc ** 4) - 1.0) < 1e-12  # lambda_c = sqrt(s / |s|)


@pytest.mark.parametrize("is_complex,eps", [(False, 1e-9), (True, 1e-4)])
def test_sweeps_reach_identity_boundaries(is_complex, eps):
    """Each bond step makes its two boundary tensors the identity; the sweeps
    converge on all bonds together (the complex state here starts further
    from the fixed point and converges linearly, about 0.92 per sweep)."""
    lat, Tn, lam, p = su_state(is_complex)
    before = O.gauge_score(Tn, lam, lat, p)
    sweeps, score = O.fix_local_gauge(Tn, lam, lat, p, maxiter=100, eps=eps)
    assert before > 1e-3 and score < eps and sweeps < 100


@pytest.fixture(scope="module")
def gauge_exe(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    from tenes_b200.build import cuda_home
    out = str(tmp_path_factory.mktemp("gaugehost") / "gauge_host_check")
    subprocess.check_call([gxx, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                           "-I", os.path.join(ROOT, "tenes_b200", "csrc"), "-I", os.path.join(ROOT, "tests"),
                           "-I", os.path.join(cuda_home(), "include"),
                           os.path.join(ROOT, "tests", "gauge_host_check.cpp"), "-o", out])
    return out


def run_host(exe, lat, Tn, lam, cut, maxiter, eps):
    cplx = any(np.iscomplexobj(t) for t in Tn)
    parts = ["complex" if cplx else "real", str(lat.N_UNIT)]
    for i in range(lat.N_UNIT):
        parts.append(f"{lat.parity(i)} " + " ".join(str(lat.neighbor(i, l)) for l in range(4)))
    for t in Tn:
        t = np.asarray(t, dtype=np.complex128 if cplx else np.float64)
        vals = " ".join(f"{float(x.real)!r} {float(x.imag)!r}" for x in t.reshape(-1)) if cplx else \
            " ".join(repr(float(x)) for x in t.reshape(-1))
        parts.append(f"{t.ndim} " + " ".join(str(d) for d in t.shape) + " " + vals)
    for w in lam:
        for v in w:
            parts.append(" ".join(repr(float(x)) for x in v))
    parts.append(f"{cut!r} {maxiter} {eps!r}")
    out = subprocess.run([exe], input="\n".join(parts) + "\n", capture_output=True, text=True,
                         check=True).stdout.splitlines()
    st = out[0].split()
    lams = [np.array([float(x) for x in ln.split()[1:]]) for ln in out[1 + lat.N_UNIT:]]
    return int(st[1]), float(st[2]), [lams[4 * i:4 * i + 4] for i in range(lat.N_UNIT)]


@pytest.mark.parametrize("is_complex", [False, True])
@pytest.mark.parametrize("maxiter,eps", [(1, 1e-2), (100, 1e-8)])
def test_host_template_matches_oracle(gauge_exe, is_complex, maxiter, eps):
    lat, Tn, lam, p = su_state(is_complex, seed=3)
    h_sweeps, h_score, h_lam = run_host(gauge_exe, lat, Tn, lam, p.Inverse_lambda_cut, maxiter, eps)
    sweeps, score = O.fix_local_gauge(Tn, lam, lat, p, maxiter=maxiter, eps=eps)
    assert h_sweeps == sweeps
    assert abs(h_score - score) <= 1e-8 * max(1.0, score)
    for i in range(lat.N_UNIT):
        for leg in range(4):
            np.testing.assert_allclose(h_lam[i][leg], lam[i][leg], rtol=1e-9, atol=1e-12)


def test_front_end_fixes_the_gauge_after_each_step(tmp_path, monkeypatch):
    """simple_update.gauge_fix = true through the front end (over the
    oracle-backed environment): every simple-update step ends with the gauge
    sweeps (simple_update.cpp:121-124), so the final state's boundary tensors
    are within gauge_convergence_epsilon of the identity."""
    import re

    import tenes_b200.itps as itps
    from tests._oracle_env import OracleEnvironment
    monkeypatch.setattr(itps, "Environment", OracleEnvironment)
    txt = open(os.path.join(ROOT, "tests", "golden", "te_tfi_input.toml")).read()
    txt = txt.replace("mode = 'time'", "mode = 'ground state'")
    txt = re.sub(r"\[parameter.simple_update\]\nnum_step = \d+",
                 "[parameter.simple_update]\nnum_step = 5\ngauge_fix = true\ngauge_convergence_epsilon = 1e-6",
                 txt)
    txt = txt.replace("dimension = 10", "dimension = 4").replace("iteration_max = 10", "iteration_max = 2")
    txt = txt.replace("noise = 0.0", "noise = 0.05")
    txt = re.sub(r"\[correlation\].*?(?=\[observable\])", "", txt, flags=re.S)
    (tmp_path / "in.toml").write_text(txt)
    it = itps.run(str(tmp_path / "in.toml"), print_level=0, outdir=str(tmp_path / "out"))
    assert it.p.Simple_Gauge_Fix and it.p.Simple_Gauge_Convergence_Epsilon == 1e-6
    env = it.env
    assert O.gauge_score(env.Tn, env.lam, env.lat, env.p) < 1e-6
