"""Full-update time evolution through the front end (time_evolution.cpp:21-90:
full-update steps when simple_update.num_step = 0, tau read from the
simple_update table as load_toml.cpp:373 does), over the oracle-backed
stand-in of the environment.

The reference ships no golden run of this mode, so the test uses what the
driver guarantees: with a measure interval longer than the run, a
time evolution is one measurement (a full CTMRG), the full-update steps, and a
final measurement; the ground-state driver with the same steps is a full
CTMRG (full_update.cpp:151-160) and the same steps.  The two end in the same
state, so the last TE_ rows equal the ground-state observables, and the TE_
files hold the rows of t = 0 and t = num_step * tau."""

import os
import re

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NSTEP, TAU = 3, 0.01


def _input(tmp_path, name, mode):
    txt = open(os.path.join(GOLDEN, "te_tfi_input.toml")).read()
    txt = txt.replace("mode = 'time'", f"mode = '{mode}'")
    txt = re.sub(r"\[parameter.simple_update\]\nnum_step = \d+", "[parameter.simple_update]\nnum_step = 0", txt)
    txt = re.sub(r"\[parameter.full_update\]\nnum_step = \d+", f"[parameter.full_update]\nnum_step = {NSTEP}", txt)
    txt = txt.replace("tau = 0.01", f"tau = {TAU}")
    txt = txt.replace("dimension = 10", "dimension = 6").replace("iteration_max = 10", "iteration_max = 4")
    txt = txt.replace("noise = 0.0", "noise = 0.05")
    txt = re.sub(r"\[correlation\].*?(?=\[observable\])", "", txt, flags=re.S)
    txt = txt.replace("[[evolution.simple]]", "[[evolution.full]]")
    p = tmp_path / name
    p.write_text(txt)
    return str(p)


def _rows(path):
    out = []
    for line in open(path):
        line = line.split("#")[0].strip()
        if line:
            out.append([float(w) for w in line.split()])
    return np.array(out)


def _run(path, outdir, monkeypatch):
    import tenes_b200.itps as itps
    from tests._oracle_env import OracleEnvironment
    monkeypatch.setattr(itps, "Environment", OracleEnvironment)
    return itps.run(path, print_level=0, outdir=str(outdir))


def test_full_update_time_evolution_matches_ground_state_steps(tmp_path, monkeypatch):
    te = _run(_input(tmp_path, "te.toml", "time"), tmp_path / "te", monkeypatch)
    gs = _run(_input(tmp_path, "gs.toml", "ground state"), tmp_path / "gs", monkeypatch)
    assert te.t_fu > 0.0 and te.t_su == 0.0
    one_te, one_gs = _rows(tmp_path / "te" / "TE_onesite_obs.dat"), _rows(tmp_path / "gs" / "onesite_obs.dat")
    times = sorted(set(one_te[:, 0]))
    np.testing.assert_allclose(times, [0.0, NSTEP * TAU], rtol=0, atol=1e-15)
    last = one_te[one_te[:, 0] == times[-1]][:, 1:]
    np.testing.assert_allclose(last, one_gs, rtol=0, atol=1e-13)
    two_te, two_gs = _rows(tmp_path / "te" / "TE_twosite_obs.dat"), _rows(tmp_path / "gs" / "twosite_obs.dat")
    np.testing.assert_allclose(two_te[two_te[:, 0] == times[-1]][:, 1:], two_gs, rtol=0, atol=1e-13)
    for i in range(4):
        np.testing.assert_array_equal(te.env.Tn[i], gs.env.Tn[i])
    # the steps changed the state
    first = one_te[one_te[:, 0] == 0.0][:, 1:]
    assert np.abs(first[:, 2:] - last[:, 2:]).max() > 1e-6


def test_both_update_kinds_in_time_evolution_is_an_input_error(tmp_path, monkeypatch):
    from tenes_b200.input import InputError
    txt = open(_input(tmp_path, "x.toml", "time")).read()
    txt = re.sub(r"\[parameter.simple_update\]\nnum_step = \d+", "[parameter.simple_update]\nnum_step = 2", txt)
    (tmp_path / "y.toml").write_text(txt)
    with pytest.raises(InputError, match="simple update and full update are both required"):
        _run(str(tmp_path / "y.toml"), tmp_path / "y", monkeypatch)
