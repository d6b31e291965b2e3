"""Tensor checkpoints (iTPS::save_tensors / load_tensors, saveload_tensors.cpp;
resize_tensor, tensor.cpp:114-149) through the front end, on the CPU with the
oracle-backed stand-in of the environment.

The reference's own restart test (test/restart.py.in) runs a ground-state
calculation that saves its tensors, then one that loads them, and compares
the observables; here the second run does no simple-update steps, so the
loaded state must reproduce the first run's observables exactly."""

import os
import re

import numpy as np
import pytest

from tenes_b200 import saveload as S

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _input(tmp_path, name, general, su_steps, D=2, chi=6):
    """A ground-state variant of the TE_TFI expert input (2 x 2, TFI terms)."""
    txt = open(os.path.join(GOLDEN, "te_tfi_input.toml")).read()
    txt = txt.replace("mode = 'time'", "mode = 'ground state'\n" + general)
    txt = re.sub(r"\[parameter.simple_update\]\nnum_step = \d+",
                 f"[parameter.simple_update]\nnum_step = {su_steps}", txt)
    txt = txt.replace("dimension = 10", f"dimension = {chi}").replace("iteration_max = 10", "iteration_max = 4")
    txt = txt.replace("virtual_dim = [2, 2, 2, 2]", f"virtual_dim = [{D}, {D}, {D}, {D}]")
    txt = txt.replace("noise = 0.0", "noise = 0.05")
    # the correlation section is skipped by the front end anyway
    txt = re.sub(r"\[correlation\].*?(?=\[observable\])", "", txt, flags=re.S)
    p = tmp_path / name
    p.write_text(txt)
    return str(p)


def _run(path, outdir, monkeypatch):
    import tenes_b200.itps as itps
    from tests._oracle_env import OracleEnvironment
    monkeypatch.setattr(itps, "Environment", OracleEnvironment)
    return itps.run(path, print_level=0, outdir=str(outdir))


def _obs(outdir):
    rows = []
    for line in open(os.path.join(outdir, "onesite_obs.dat")):
        line = line.split("#")[0].strip()
        if line:
            rows.append([float(w) for w in line.split()])
    return np.array(rows)


def test_tensor_file_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    for a in (rng.standard_normal((2, 3, 1, 4)), rng.standard_normal((3, 2)) + 1j * rng.standard_normal((3, 2)),
              np.array(2.5)):
        S.write_tensor(str(tmp_path / "x.dat"), a)
        b = S.read_tensor(str(tmp_path / "x.dat"))
        assert b.shape == a.shape and b.dtype == a.dtype
        assert np.array_equal(a, b)


def test_resize_tensor_extends_with_zeros_and_slices():
    a = np.arange(12.0).reshape(3, 4)
    b = S.resize_tensor(a, (5, 2))
    assert b.shape == (5, 2)
    np.testing.assert_array_equal(b[:3], a[:, :2])
    assert not b[3:].any()
    with pytest.raises(S.LoadError):
        S.resize_tensor(a, (3, 4, 1))


def test_foreign_tensor_file_is_a_load_error(tmp_path):
    p = tmp_path / "T_0.dat"
    p.write_bytes(b"\x00\x01binary")
    with pytest.raises(S.LoadError, match="not a tenes_b200 tensor file"):
        S.read_tensor(str(p))


def test_save_then_load_reproduces_the_state(tmp_path, monkeypatch):
    save = tmp_path / "ckpt"
    a = _run(_input(tmp_path, "a.toml", f"tensor_save = '{save}'", 20), tmp_path / "out_a", monkeypatch)
    # params.dat in the reference's layout (saveload_tensors.cpp:45-58)
    lines = open(save / "params.dat").read().splitlines()
    assert lines[0] == "1 # Format_Version" and lines[1] == "4 # N_UNIT" and lines[2] == "6 # CHI"
    assert lines[3] == "2 2 2 2 2 # Shape of Tn[0]"
    names = {f"{s}_{i}.dat" for s in ("T", "Et", "Er", "Eb", "El", "C1", "C2", "C3", "C4", "lambda")
             for i in range(4)}
    assert names <= set(os.listdir(save))
    for i in range(4):
        np.testing.assert_array_equal(S.read_tensor(str(save / f"T_{i}.dat")), a.env.Tn[i])
    b = _run(_input(tmp_path, "b.toml", f"tensor_load = '{save}'", 0), tmp_path / "out_b", monkeypatch)
    for i in range(4):
        np.testing.assert_array_equal(b.env.Tn[i], a.env.Tn[i])
        for leg in range(4):
            np.testing.assert_array_equal(b.env.lam[i][leg], a.env.lam[i][leg])
    np.testing.assert_allclose(_obs(tmp_path / "out_b"), _obs(tmp_path / "out_a"), rtol=0, atol=0)


def test_load_resizes_to_the_new_dimensions(tmp_path, monkeypatch, capsys):
    save = tmp_path / "ckpt"
    a = _run(_input(tmp_path, "a.toml", f"tensor_save = '{save}'", 10), tmp_path / "out_a", monkeypatch)
    import tenes_b200.itps as itps
    from tenes_b200.input import load_input
    from tests._oracle_env import OracleEnvironment
    monkeypatch.setattr(itps, "Environment", OracleEnvironment)
    inp = load_input(_input(tmp_path, "b.toml", f"tensor_load = '{save}'", 0, D=3, chi=8))
    inp.params.outdir = str(tmp_path / "out_b")
    b = itps.ITPS(inp, print_level=1)
    out = capsys.readouterr().out
    assert "WARNING: parameters.ctm.dimension is 8 but loaded tensors have CHI = 6" in out
    assert "WARNING: virtual dimension of the leg 0 of the tensor 0 is 3 but loaded tensor has 2" in out
    for i in range(4):
        T = b.env.Tn[i]
        assert T.shape == (3, 3, 3, 3, 2)
        np.testing.assert_array_equal(T[:2, :2, :2, :2], a.env.Tn[i])
        assert not T[2:].any() and not T[:, 2:].any()
        for leg in range(4):
            lam = b.env.lam[i][leg]
            np.testing.assert_array_equal(lam[:2], a.env.lam[i][leg])
            assert lam[2] == 0.0
        assert b.env.get_env(0, i).shape == (8, 8)
        assert b.env.get_env(4, i).shape == (8, 8, 3, 3)


def test_incompatible_checkpoints_are_load_errors(tmp_path, monkeypatch):
    save = tmp_path / "ckpt"
    _run(_input(tmp_path, "a.toml", f"tensor_save = '{save}'", 2), tmp_path / "out_a", monkeypatch)
    with pytest.raises(S.LoadError, match="does not exists"):
        _run(_input(tmp_path, "b.toml", f"tensor_load = '{tmp_path / 'nope'}'", 0), tmp_path / "o1", monkeypatch)
    txt = (save / "params.dat").read_text().replace("4 # N_UNIT", "9 # N_UNIT")
    (save / "params.dat").write_text(txt)
    with pytest.raises(S.LoadError, match="N_UNIT"):
        _run(_input(tmp_path, "c.toml", f"tensor_load = '{save}'", 0), tmp_path / "o2", monkeypatch)
    txt = txt.replace("9 # N_UNIT", "4 # N_UNIT").replace("2 2 2 2 2 # Shape of Tn[1]", "2 2 2 2 3 # Shape of Tn[1]")
    (save / "params.dat").write_text(txt)
    with pytest.raises(S.LoadError, match="physical bond of the tensor 1"):
        _run(_input(tmp_path, "d.toml", f"tensor_load = '{save}'", 0), tmp_path / "o3", monkeypatch)
