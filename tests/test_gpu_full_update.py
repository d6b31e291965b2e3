"""Full update on the GPU (tg_fu_bond and the front end's full-update steps).

* tg_fu_bond against the oracle's full_update_bond (pinned to the reference's
  full_update.dat and AntiferroHeisenberg_real / _complex goldens) in a CTM
  environment, for every bond direction and for real and complex tensors: the
  bond-contracted pair Tn1_new . Tn2_new (free of the gauge on the updated
  bond) and the least-squares iteration count;
* the reference's AntiferroHeisenberg_real, _complex and RSVD inputs through
  ``python -m tenes_b200`` (simple update, one full-update step with the fast
  full update's moves, CTMRG, observables) against their golden files, checked
  the way the reference checks them (test/fulltest.py.in: rtol 1e-3, atol 1e-4)."""

import json
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import tenes_oracle as O
from tenes_b200.std_ops import evolution_twosite, heisenberg_bond
from tests._helpers import gpu_env, load_env

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")
BOND = {0: (0, 2), 1: (1, 3), 2: (2, 0), 3: (3, 1)}


@pytest.mark.parametrize("is_complex", [False, True])
@pytest.mark.parametrize("leg", [0, 1, 2, 3])
def test_fu_bond_matches_oracle(leg, is_complex):
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
    r = O._FU_ROT[leg]
    _, _, it_ref, conv_ref = O.full_update_bond_horizontal(*args, Tn[source].transpose(r), Tn[tgt].transpose(r),
                                                           op, p)
    ra, rb = O.full_update_bond(*args, Tn[source], Tn[tgt], op, leg, p)
    ge = gpu_env(lat, Tn, 4, is_complex)
    load_env(ge, env)
    it, conv = ge.full_update_bond(source, leg, op)
    a, b = ge.get_site_tensor(source), ge.get_site_tensor(tgt)
    ge.close()
    la, lb = BOND[leg]
    assert (it, conv) == (it_ref, conv_ref)
    np.testing.assert_allclose(np.tensordot(a, b, ([la], [lb])), np.tensordot(ra, rb, ([la], [lb])),
                               rtol=1e-8, atol=1e-12)


def _rows(path):
    out = []
    for line in open(path):
        line = line.split("#")[0].strip()
        if line:
            out.append([float(w) for w in line.split()])
    return out


@pytest.mark.parametrize("stem", ["afh_real", "afh_complex", "rsvd"])
def test_afh_full_update_golden(tmp_path, stem):
    r = subprocess.run([sys.executable, "-m", "tenes_b200", os.path.join(GOLDEN, f"{stem}_input.toml"),
                        "--outdir", str(tmp_path), "--quiet"], cwd=REPO, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    exp = json.load(open(os.path.join(GOLDEN, f"{stem}_expected.json")))
    tol = exp["tolerance"]
    dens = {}
    for line in open(tmp_path / "density.dat"):
        if "=" in line:
            name, vals = line.split("=")
            dens[name.strip()] = [float(x) for x in vals.split()]
    # the complex golden's density.dat predates the reference's renaming of
    # the bond term to bond_hamiltonian
    dens = {("hamiltonian" if k == "bond_hamiltonian" and "hamiltonian" in exp["density"] else k): v
            for k, v in dens.items()}
    assert set(dens) == set(exp["density"])
    for k, v in exp["density"].items():
        np.testing.assert_allclose(dens[k], v, rtol=tol["rtol"], atol=tol["atol"], err_msg=k)
    for name, key in (("onesite_obs.dat", "onesite"), ("twosite_obs.dat", "twosite"),
                      ("multisite_obs_4.dat", "multisite"), ("correlation.dat", "correlation")):
        if key not in exp:  # the complex golden has no multisite file
            continue
        res, ref = _rows(tmp_path / name), exp[key]
        assert len(res) == len(ref), name
        np.testing.assert_allclose(np.array(res), np.array(ref), rtol=tol["rtol"], atol=tol["atol"], err_msg=name)


def test_full_update_time_evolution_matches_ground_state_steps(tmp_path):
    """Full-update time evolution on the GPU ends where the ground-state
    driver with the same full-update steps ends (the CPU test of
    tests/test_te_full_update.py, on the library)."""
    import tenes_b200.itps as itps
    from tests.test_te_full_update import NSTEP, TAU, _input, _rows
    te = itps.run(_input(tmp_path, "te.toml", "time"), print_level=0, outdir=str(tmp_path / "te"))
    gs = itps.run(_input(tmp_path, "gs.toml", "ground state"), print_level=0, outdir=str(tmp_path / "gs"))
    one_te, one_gs = _rows(tmp_path / "te" / "TE_onesite_obs.dat"), _rows(tmp_path / "gs" / "onesite_obs.dat")
    last = one_te[np.isclose(one_te[:, 0], NSTEP * TAU)][:, 1:]
    np.testing.assert_allclose(last, one_gs, rtol=0, atol=1e-9)
    for i in range(4):
        np.testing.assert_allclose(te.env.get_site_tensor(i), gs.env.get_site_tensor(i), rtol=0, atol=1e-9)
