"""parameters.dat (PEPS_Parameters::save, PEPS_Parameters.cpp:220-300;
SquareLattice::save, SquareLattice.cpp:139-150; iTPS.cpp:145-150): the front
end's writer reproduces the reference's own files of the golden runs byte for
byte, the run-dependent start_datetime value aside."""
import json
import os
import re

import pytest

from tenes_b200.input import load_input
from tenes_b200.itps import write_parameters

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FILES = json.load(open(os.path.join(GOLDEN, "parameters_dat.json")))["files"]


@pytest.mark.parametrize("stem", sorted(FILES))
def test_parameters_dat_matches_reference(tmp_path, stem):
    inp = load_input(os.path.join(GOLDEN, f"{stem}_input.toml"))
    path = tmp_path / "parameters.dat"
    write_parameters(str(path), inp.params, inp.lattice)
    text = path.read_text()
    lines = text.splitlines(keepends=True)
    assert re.fullmatch(r"start_datetime =  \d{4}-\d\d-\d\dT\d\d:\d\d:\d\d[+-]\d\d:\d\d\n", lines[-1])
    got = "".join(lines[:-1])
    want = FILES[stem]
    if "\nmode = " not in want:
        # written by an earlier TeNeS, before PEPS_Parameters::save gained the
        # calculation-mode block (PEPS_Parameters.cpp:280-291 in v2.1.2)
        got = re.sub(r"mode = [^\n]*\n(finite temperature\n)?simple\n", "", got)
    assert got == want
