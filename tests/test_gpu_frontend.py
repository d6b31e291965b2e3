"""End-to-end run of the reference's TE_TFI test input through
``python -m tenes_b200`` on the GPU, checked the way the reference checks its
own runs (test/fulltest.py.in:55-88, rtol 1e-3, atol 1e-4) against the
committed TE_* output fixtures."""
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest

from tests._te_tfi import GOLDEN, expected

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _env():
    """The child runs the repository's package from any directory."""
    e = dict(os.environ)
    e["PYTHONPATH"] = REPO + os.pathsep + e.get("PYTHONPATH", "")
    return e


def _read(path):
    rows = []
    with open(path) as f:
        for line in f:
            line = line.split("#")[0].strip()
            if line:
                rows.append([float(w) for w in line.split()])
    return rows


@pytest.fixture(scope="module")
def te_tfi_run(tmp_path_factory):
    out = tmp_path_factory.mktemp("te_tfi")
    r = subprocess.run([sys.executable, "-m", "tenes_b200", os.path.join(GOLDEN, "te_tfi_input.toml"),
                        "--outdir", str(out), "--quiet"], cwd=REPO, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    return out


@pytest.mark.parametrize("name,key", [("TE_density.dat", "density"), ("TE_onesite_obs.dat", "onesite"),
                                      ("TE_twosite_obs.dat", "twosite"),
                                      ("TE_multisite_obs_4.dat", "multisite"),
                                      ("TE_correlation_length.dat", "correlation_length"),
                                      ("TE_correlation.dat", "correlation")])
def test_te_tfi_outputs(te_tfi_run, name, key):
    exp = expected()
    tol = exp["tolerance"]
    res = _read(os.path.join(te_tfi_run, name))
    ref = exp[key]
    assert len(res) == len(ref), (name, len(res), len(ref))
    bad = []
    for i, (rs, rf) in enumerate(zip(res, ref)):
        if not all(np.isclose(s, f, rtol=tol["rtol"], atol=tol["atol"]) for s, f in zip(rs, rf)):
            bad.append((i, rs, rf))
    assert not bad, bad[:5]


def test_te_tfi_time_dat(te_tfi_run):
    lines = open(os.path.join(te_tfi_run, "time.dat")).read().splitlines()
    assert [l.split("=")[0].strip() for l in lines] == [
        "time all", "time simple update", "time full update", "time environment", "time observable"]


def _density(path):
    out = []
    for line in open(path):
        w = line.split()
        out.append(complex(float(w[2]), float(w[3])))
    return out


def test_restart_from_saved_tensors(tmp_path):
    """The reference's restart test (test/restart.py.in) on the GPU front end:
    restart_0 runs 10 simple-update steps and saves the tensors and weights,
    restart_1 loads them and runs 10 more.  Both inputs write into
    output_restart_0 (the reference's test then compares that directory with
    itself), so the first run's output is moved aside; the continued run must
    reproduce one uninterrupted run of 20 steps from the same start, and its
    observables must have moved away from the first run's."""
    for k in (0, 1):
        shutil.copyfile(os.path.join(GOLDEN, f"restart_{k}_input.toml"), tmp_path / f"restart_{k}.toml")
    txt = open(os.path.join(GOLDEN, "restart_0_input.toml")).read()
    assert "num_step = 10" in txt and "tensor_save = 'tensor'" in txt
    txt = txt.replace("num_step = 10", "num_step = 20", 1).replace("tensor_save = 'tensor'", "")
    (tmp_path / "twenty.toml").write_text(txt.replace("output = 'output_restart_0'", "output = 'output_twenty'"))

    def run(name):
        r = subprocess.run([sys.executable, "-m", "tenes_b200", name, "--quiet"], cwd=tmp_path,
                           capture_output=True, text=True, timeout=900, env=_env())
        assert r.returncode == 0, r.stderr[-3000:]
    run("restart_0.toml")
    assert (tmp_path / "tensor" / "params.dat").exists()
    shutil.move(str(tmp_path / "output_restart_0"), str(tmp_path / "first"))
    run("restart_1.toml")
    run("twenty.toml")
    res, ref, first = tmp_path / "output_restart_0", tmp_path / "output_twenty", tmp_path / "first"
    a, b = _density(res / "density.dat"), _density(ref / "density.dat")
    assert len(a) == len(b)
    np.testing.assert_allclose(a, b, rtol=1e-9, atol=1e-12)
    assert np.max(np.abs(np.array(a) - np.array(_density(first / "density.dat")))) > 1e-6
    for name in ("onesite_obs.dat", "twosite_obs.dat"):
        x, y = _read(res / name), _read(ref / name)
        assert len(x) == len(y), name
        np.testing.assert_allclose(np.array(x), np.array(y), rtol=1e-9, atol=1e-12, err_msg=name)
