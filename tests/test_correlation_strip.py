"""Long-range correlations along a strip (StartCorrelation / Transfer /
FinishCorrelation_iTPS_CTM, contract_itps_ctm/correlation.cpp) in the oracle
and through the front end's strip path."""

import json
import os
import re

import numpy as np
import pytest

from oracle import tenes_oracle as O
from tests._helpers import make_lattice, oracle_params, physical_tensors

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SZ = np.diag([0.5, -0.5])
SX = np.array([[0.0, 0.5], [0.5, 0.0]])


@pytest.mark.parametrize("is_complex", [False, True])
@pytest.mark.parametrize("vertical", [False, True])
def test_strip_equals_windows(is_complex, vertical):
    lat = make_lattice(2, 2, 2)
    Tn = physical_tensors(lat, 2, is_complex=is_complex)
    p = oracle_params(6)
    env = O.init_env(Tn, p, lat)
    for _ in range(3):
        O.sweep(env, Tn, p, lat)
    for left in range(4):
        res = O.correlation_strip(env, Tn, lat, left, vertical, 4, SZ, lambda s: [SZ, SX])
        for r in range(1, 5):
            if vertical:
                nrow, ncol, sr, sc, pl, pr = r + 1, 1, r, 0, (r, 0), (0, 0)
            else:
                nrow, ncol, sr, sc, pl, pr = 1, r + 1, 0, 0, (0, 0), (0, r)
            idx, C, eTt, eTr, eTb, eTl, T = O._window(env, Tn, lat, left, sc, sr, nrow, ncol)

            def w(ops):
                g = [[ops.get((a, b), np.eye(2)) for b in range(ncol)] for a in range(nrow)]
                return O.contract_window(C, eTt, eTr, eTb, eTl, T, g)
            nrm = w({})
            for k, op in enumerate([SZ, SX]):
                ref = w({pl: SZ, pr: op}) / nrm
                assert abs(res[r - 1][k] - ref) <= 1e-12 * max(1.0, abs(ref))


def test_front_end_strip_path_reproduces_the_golden(tmp_path, monkeypatch):
    """r_max = 5 takes the strip path; its r <= 3 rows are the golden's."""
    import tenes_b200.itps as itps
    from tests._oracle_env import OracleEnvironment
    monkeypatch.setattr(itps, "Environment", OracleEnvironment)
    txt = open(os.path.join(GOLDEN, "afh_real_input.toml")).read()
    txt = re.sub(r"r_max = 3", "r_max = 5", txt)
    path = tmp_path / "in.toml"
    path.write_text(txt)
    itps.run(str(path), print_level=0, outdir=str(tmp_path / "out"))
    rows = []
    for line in open(tmp_path / "out" / "correlation.dat"):
        line = line.split("#")[0].strip()
        if line:
            rows.append([float(x) for x in line.split()])
    rows = np.array(rows)
    assert rows[:, 3:5].max() == 5
    short = rows[(rows[:, 3] <= 3) & (rows[:, 4] <= 3)]
    exp = np.array(json.load(open(os.path.join(GOLDEN, "afh_real_expected.json")))["correlation"])
    assert short.shape == exp.shape
    np.testing.assert_allclose(short, exp, rtol=1e-9, atol=1e-11)
