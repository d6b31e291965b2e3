"""Ground state with a full-update step through the front end
(optimize.cpp:24-37, full_update.cpp:30-186) over the oracle-backed stand-in
of the environment, against the reference's AntiferroHeisenberg_real,
AntiferroHeisenberg_complex and RSVD goldens (100 simple-update steps, one
full-update step with the fast full update's single moves, CTMRG chi = 5 with
full-SVD or rSVD projectors, observables, correlations)."""

import json
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _rows(path):
    out = []
    for line in open(path):
        line = line.split("#")[0].strip()
        if line:
            out.append([float(w) for w in line.split()])
    return out


def _density(path):
    d = {}
    for line in open(path):
        if "=" in line:
            name, vals = line.split("=")
            d[name.strip()] = [float(x) for x in vals.split()]
    return d


@pytest.mark.parametrize("stem", ["afh_real", "afh_complex", "rsvd"])
def test_afh_full_update_driver_on_oracle(tmp_path, monkeypatch, stem):
    import tenes_b200.itps as itps
    from tests._oracle_env import OracleEnvironment
    monkeypatch.setattr(itps, "Environment", OracleEnvironment)
    it = itps.run(os.path.join(GOLDEN, f"{stem}_input.toml"), print_level=0, outdir=str(tmp_path))
    exp = json.load(open(os.path.join(GOLDEN, f"{stem}_expected.json")))
    dens = _density(tmp_path / "density.dat")
    # the complex golden's density.dat predates the reference's renaming of
    # the bond term to bond_hamiltonian
    dens = {("hamiltonian" if k == "bond_hamiltonian" and "hamiltonian" in exp["density"] else k): v
            for k, v in dens.items()}
    assert set(dens) == set(exp["density"])
    for k, v in exp["density"].items():
        np.testing.assert_allclose(dens[k], v, rtol=1e-10, atol=1e-12, err_msg=k)
    for name, key in (("onesite_obs.dat", "onesite"), ("twosite_obs.dat", "twosite"),
                      ("multisite_obs_4.dat", "multisite"), ("correlation.dat", "correlation")):
        if key not in exp:  # the complex golden has no multisite file
            continue
        res, ref = _rows(tmp_path / name), exp[key]
        assert len(res) == len(ref), name
        np.testing.assert_allclose(np.array(res), np.array(ref), rtol=1e-9, atol=1e-11, err_msg=name)
    assert it.t_fu > 0.0
    assert "time full update" in open(tmp_path / "time.dat").read()


def test_dimension_changing_gates_are_an_input_error(tmp_path, monkeypatch):
    """J1J2_AFH's gates change a site's physical dimension (2 -> 8 -> 2); the
    library keeps physical dimensions fixed and says so instead of misreading
    the operators."""
    import pytest

    import tenes_b200.itps as itps
    from tenes_b200.input import InputError
    from tests._oracle_env import OracleEnvironment
    monkeypatch.setattr(itps, "Environment", OracleEnvironment)
    with pytest.raises(InputError, match="change a site's physical dimension"):
        itps.run(os.path.join(GOLDEN, "j1j2_afh_input.toml"), print_level=0, outdir=str(tmp_path))
