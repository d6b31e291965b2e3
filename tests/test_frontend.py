"""CPU checks of the tenes-compatible front-end: lattice walks, group names and
the byte layout of the output files (src/iTPS/onesite_obs.cpp:125-200,
twosite_obs.cpp:288-361, density.cpp:30-228, correlation_length.cpp:57-125)."""
import os

import numpy as np
import pytest

from oracle import tenes_oracle as O
from tenes_b200.input import InputError, load_input
from tenes_b200.itps import ITPS

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("LX,LY,skew", [(2, 2, 0), (3, 2, 1), (2, 1, -1), (4, 3, 2), (1, 1, 0)])
def test_lattice_other_matches_oracle(LX, LY, skew):
    inp = load_input(os.path.join(GOLDEN, "te_tfi_input.toml"))
    ls = inp.lattice
    ls.LX, ls.LY, ls.skew = LX, LY, skew
    lat = O.Lattice(LX, LY, skew)
    assert ls.neighbors() == [[lat.neighbor(i, d) for d in range(4)] for i in range(LX * LY)]
    for i in range(LX * LY):
        for dx in range(-3, 4):
            for dy in range(-3, 4):
                assert ls.other(i, dx, dy) == lat.other(i, dx, dy)


def _fake(tmp_path, calcmode="ground_state"):
    """An ITPS front-end without a device context (writers only)."""
    inp = load_input(os.path.join(GOLDEN, "te_tfi_input.toml"))
    inp.params.calcmode = calcmode
    it = object.__new__(ITPS)
    it.inp, it.p = inp, inp.params
    it.LX, it.LY, it.N = inp.lattice.LX, inp.lattice.LY, inp.lattice.LX * inp.lattice.LY
    it.outdir = str(tmp_path)
    it.print_level = 0
    n1 = ITPS._names(inp.onesite, "onesite", False)
    n2 = ITPS._names(inp.twosite, "twosite", False)
    nm = ITPS._names(inp.multisite, "multisite", True)
    w = max([len("Energy")] + [len(s) for s in n1 + n2 + nm])
    it.names1, it.names2, it.namesm = ([s.ljust(w) for s in n] for n in (n1, n2, nm))
    it._first = {}
    return it


def test_group_names_padded_to_common_width(tmp_path):
    it = _fake(tmp_path)
    widths = {len(s) for s in it.names1 + it.names2 + it.namesm}
    assert len(widths) == 1
    assert it.names1[0].rstrip() == "Sz"


def test_group_with_two_names_is_an_error():
    inp = load_input(os.path.join(GOLDEN, "te_tfi_input.toml"))
    ops = list(inp.onesite)
    ops[1] = type(ops[1])("other", ops[0].group, ops[1].source_site, [], [], ops[1].op, [], 1.0)
    with pytest.raises(InputError):
        ITPS._names(ops, "onesite", False)


def test_onesite_and_density_layout(tmp_path):
    it = _fake(tmp_path)
    ng = len(it.names1)
    vals = [[complex(0.25 * g - 0.1 * i, 0.0) for i in range(it.N)] for g in range(ng)]
    norm = [1.0 + 0j] * it.N
    it.save_onesite(vals, norm, None, "")
    text = open(tmp_path / "onesite_obs.dat").read().splitlines()
    assert text[0] == "# The meaning of each column is the following: "
    assert text[1:5] == ["# $1: op_group", "# $2: site_index", "# $3: real", "# $4: imag"]
    assert text[5] == "# The names of op_group are the following: "
    assert text[6 + ng] == "# -1: norm" and text[7 + ng] == ""
    rows = text[8 + ng:]
    assert rows[0] == f"0 0 {0.0:.17e} {0.0:.17e}"
    assert rows[1] == f"0 1 {-0.1:.17e} {0.0:.17e}"
    assert len(rows) == (ng + 1) * it.N
    two = [dict() for _ in it.names2]
    it.save_density(vals, two, [dict() for _ in it.namesm], None, "")
    dens = open(tmp_path / "density.dat").read().splitlines()
    w = len(it.names1[0])
    assert dens[0].startswith("Energy".ljust(w) + " = ")
    mean = sum(vals[0], 0j).real / it.N
    assert dens[1] == f"{it.names1[0]} = {mean:.17e}  {0.0:.17e}"


def test_time_evolution_headers_and_rows(tmp_path):
    it = _fake(tmp_path, "time_evolution")
    ng = len(it.names1)
    vals = [[complex(1.0, 0.0)] * it.N for _ in range(ng)]
    for t in (0.0, 0.2):
        it.save_onesite(vals, [1.0 + 0j] * it.N, t, "TE_")
        it.save_density(vals, [dict() for _ in it.names2], [dict() for _ in it.namesm], t, "TE_")
    text = open(tmp_path / "TE_onesite_obs.dat").read().splitlines()
    assert text[1] == "# $1: time"
    data = [l for l in text if l and not l.startswith("#")]
    assert len(data) == 2 * (ng + 1) * it.N
    assert data[-1].startswith(f"{0.2:.17e} -1 {it.N - 1} ")
    dens = [l for l in open(tmp_path / "TE_density.dat").read().splitlines() if l and not l.startswith("#")]
    assert dens[0].split()[:2] == [f"{0.0:.17e}", "0"]
    assert len(dens) == 2 * (1 + ng + len(it.names2) + len(it.namesm))


def test_correlation_length_layout(tmp_path):
    it = _fake(tmp_path)
    res = [(0, 0, np.array([2.0, 1.0, 0.5, 0.0])), (1, 1, np.array([3.0]))]
    it.save_correlation_length(res, None, "")
    rows = [l for l in open(tmp_path / "correlation_length.dat").read().splitlines()
            if l and not l.startswith("#")]
    L = it.LX
    w = rows[0].split()
    assert w[:2] == ["0", "0"]
    assert float(w[2]) == pytest.approx(-L / np.log(0.5))
    assert float(w[3]) == pytest.approx(np.log(2.0) / L) and w[5] == "inf"
    assert rows[1] == f"1 1 {0.0:.17e}"


def _rows(path):
    out = []
    with open(path) as f:
        for line in f:
            line = line.split("#")[0].strip()
            if line:
                out.append([float(w) for w in line.split()])
    return out


def test_te_tfi_driver_on_oracle(tmp_path, monkeypatch):
    """The whole front-end (time-evolution loop, measurements, writers) over the
    oracle-backed stand-in reproduces the reference's TE_TFI output files."""
    import tenes_b200.itps as itps
    from tests._oracle_env import OracleEnvironment
    from tests._te_tfi import expected

    monkeypatch.setattr(itps, "Environment", OracleEnvironment)
    itps.run(os.path.join(GOLDEN, "te_tfi_input.toml"), print_level=0, outdir=str(tmp_path))
    exp = expected()
    for name, key in [("TE_density.dat", "density"), ("TE_onesite_obs.dat", "onesite"),
                      ("TE_twosite_obs.dat", "twosite"), ("TE_multisite_obs_4.dat", "multisite"),
                      ("TE_correlation_length.dat", "correlation_length"), ("TE_correlation.dat", "correlation")]:
        res = _rows(tmp_path / name)
        ref = exp[key]
        assert len(res) == len(ref), name
        for rs, rf in zip(res, ref):
            if len(rs) != len(rf):
                # the product state at t = 0 has one-dimensional boundary legs, so its
                # transfer matrix is 1 x 1 and only "dir x 0.0" is written
                # (transfer_matrix.cpp:90-93, correlation_length.cpp:99-106); the stored
                # file lists zero eigenvalues there, and the reference's own check
                # compares the common leading columns (test/fulltest.py.in:77)
                assert name == "TE_correlation_length.dat" and len(rs) == 4 and rs[3] == 0.0
                assert all(np.isinf(rf[4:])), rf
            n = min(len(rs), len(rf))
            np.testing.assert_allclose(rs[:n], rf[:n], rtol=1e-9, atol=1e-11, err_msg=name)


@pytest.mark.parametrize("stem,tol,tol_xi", [("ft_tfi_square", 5e-5, 5e-4), ("ft_kitaev", 1e-10, 1e-4)])
def test_finite_temperature_driver_on_oracle(tmp_path, monkeypatch, stem, tol, tol_xi):
    """The finite-temperature front end (iTPS::finite_temperature: beta
    stepping, measure_density with the transfer matrix skipped at beta = 0,
    the FT_ writers) over the oracle-backed stand-in reproduces the
    reference's FT_TFI_square and FT_Kitaev output files; the tolerance is
    the oracle's own distance to them (tests/test_oracle_density.py)."""
    import tenes_b200.itps as itps
    from tests._oracle_env import OracleEnvironment
    from tests._ft import expected

    monkeypatch.setattr(itps, "Environment", OracleEnvironment)
    itps.run(os.path.join(GOLDEN, stem + "_input.toml"), print_level=0, outdir=str(tmp_path))
    exp = expected(stem)
    for name, key in [("FT_density.dat", "density"), ("FT_onesite_obs.dat", "onesite"),
                      ("FT_twosite_obs.dat", "twosite"), ("FT_correlation_length.dat", "correlation_length"),
                      ("FT_correlation.dat", "correlation")]:
        res = _rows(tmp_path / name)
        ref = exp[key]
        assert len(res) == len(ref), name
        for rs, rf in zip(res, ref):
            assert len(rs) == len(rf), name
            t = tol_xi if key == "correlation_length" else tol
            np.testing.assert_allclose(rs, rf, rtol=t, atol=t, err_msg=name)
    head = open(tmp_path / "FT_density.dat").read().splitlines()
    assert head[1] == "# $1: inverse temperature"
