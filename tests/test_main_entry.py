"""tenes_gpu_main, the process-level C entry point (the counterpart of
tenes_itps_main, src/iTPS/main.hpp:26-28), called from a C program that has
no Python of its own (tests/main_host.c, built with the system cc).

CPU: the embedded front end starts, and input errors come back as
TG_E_INPUT with a message, nothing raised -- no GPU is touched before the
input is accepted.  GPU: the reference's TE_TFI and AntiferroHeisenberg_real
inputs run through the C call, and every output file is checked against the
reference's own (test/fulltest.py.in:55-88 tolerances; parameters.dat byte
for byte but for its start time)."""
import json
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")
LIB = os.path.join(REPO, "tenes_b200", "libtenes_gpu.so")
TG_E_INPUT = 1


@pytest.fixture(scope="module")
def host(tmp_path_factory):
    if not os.path.exists(LIB):
        pytest.skip("libtenes_gpu.so is not built")
    exe = str(tmp_path_factory.mktemp("host") / "main_host")
    subprocess.check_call(["cc", "-O1", "-o", exe, os.path.join(REPO, "tests", "main_host.c"), "-ldl"])
    return exe


def _run(host, cwd, *inputs, print_level=0, timeout=900):
    env = dict(os.environ)
    env.pop("PYTHONPATH", None)
    return subprocess.run([host, LIB, str(print_level), *inputs], cwd=cwd, capture_output=True, text=True,
                          timeout=timeout, env=env)


def test_missing_and_bad_inputs_are_input_errors(host, tmp_path):
    bad = tmp_path / "mf.toml"
    text = open(os.path.join(GOLDEN, "te_tfi_input.toml")).read().replace("meanfield_env = false",
                                                                          "meanfield_env = true")
    assert "meanfield_env = true" in text
    bad.write_text(text)
    r = _run(host, tmp_path, str(tmp_path / "absent.toml"), str(bad), "")
    statuses = [int(x) for x in re.findall(r"^status (\d+)$", r.stdout, re.M)]
    assert statuses == [TG_E_INPUT] * 3, r.stdout + r.stderr
    msgs = re.findall(r"^message (.*)$", r.stdout, re.M)
    assert "absent.toml" in msgs[0]
    assert "mean-field" in msgs[1]
    assert "empty" in msgs[2]
    assert r.returncode == TG_E_INPUT


def _rows(path):
    out = []
    for line in open(path):
        line = line.split("#")[0].strip()
        if line:
            out.append([float(w) for w in line.split()])
    return out


def _check_parameters_dat(outdir, stem):
    want = json.load(open(os.path.join(GOLDEN, "parameters_dat.json")))["files"][stem]
    lines = open(os.path.join(outdir, "parameters.dat")).read().splitlines(keepends=True)
    assert lines[-1].startswith("start_datetime =  ")
    assert "".join(lines[:-1]) == want


@pytest.mark.gpu
def test_te_tfi_and_afh_real_through_the_c_entry_point(host, tmp_path):
    for stem in ("te_tfi", "afh_real"):
        shutil.copyfile(os.path.join(GOLDEN, f"{stem}_input.toml"), tmp_path / f"{stem}.toml")
    # two runs in one process: the interpreter is brought up once and reused
    r = _run(host, tmp_path, "te_tfi.toml", "afh_real.toml")
    assert re.findall(r"^status (\d+)$", r.stdout, re.M) == ["0", "0"], r.stdout + r.stderr[-3000:]
    # TE_TFI: time evolution, TE_* files
    out = tmp_path / "output_TE_TFI"
    exp = json.load(open(os.path.join(GOLDEN, "te_tfi_expected.json")))
    tol = exp["tolerance"]
    for name, key in (("TE_density.dat", "density"), ("TE_onesite_obs.dat", "onesite"),
                      ("TE_twosite_obs.dat", "twosite"), ("TE_multisite_obs_4.dat", "multisite"),
                      ("TE_correlation.dat", "correlation")):
        res, ref = _rows(out / name), exp[key]
        assert len(res) == len(ref), name
        np.testing.assert_allclose(np.array(res), np.array(ref), rtol=tol["rtol"], atol=tol["atol"], err_msg=name)
    # the common leading columns of the correlation lengths (test/fulltest.py.in:77)
    res, ref = _rows(out / "TE_correlation_length.dat"), exp["correlation_length"]
    assert len(res) == len(ref)
    for a, b in zip(res, ref):
        n = min(len(a), len(b))
        np.testing.assert_allclose(a[:n], b[:n], rtol=tol["rtol"], atol=tol["atol"])
    _check_parameters_dat(out, "te_tfi")
    assert (out / "time.dat").exists()
    # AntiferroHeisenberg_real: simple update + one full-update step + CTMRG
    out = tmp_path / "output_AntiferroHeisenberg_real"
    exp = json.load(open(os.path.join(GOLDEN, "afh_real_expected.json")))
    dens = {}
    for line in open(out / "density.dat"):
        if "=" in line:
            k, v = line.split("=")
            dens[k.strip()] = [float(x) for x in v.split()]
    assert set(dens) == set(exp["density"])
    for k, v in exp["density"].items():
        np.testing.assert_allclose(dens[k], v, rtol=tol["rtol"], atol=tol["atol"], err_msg=k)
    for name, key in (("onesite_obs.dat", "onesite"), ("twosite_obs.dat", "twosite"),
                      ("multisite_obs_4.dat", "multisite"), ("correlation.dat", "correlation"),
                      ("correlation_length.dat", "correlation_length")):
        res, ref = _rows(out / name), exp[key]
        assert len(res) == len(ref), name
        for a, b in zip(res, ref):
            n = min(len(a), len(b))
            np.testing.assert_allclose(a[:n], b[:n], rtol=tol["rtol"], atol=tol["atol"], err_msg=name)
    _check_parameters_dat(out, "afh_real")
