"""Regenerate the golden fixtures under tests/golden/ from the reference tree.

Run once, in a container where the TeNeS source tree is mounted:

    python tests/golden/make_fixtures.py /root/reference

It copies the numbers of the reference's own test fixtures (not its sources)
into compact JSON / TOML files so that the tests never read the reference
tree at run time:

* simple_update_kat.json  <- test/data/simple_update.dat
  (known answer of core::Simple_update_bond, test/simple_update.cpp:28-160)
* full_update_kat.json    <- test/data/full_update.dat
  (known answer of core::Full_update_bond, test/full_update.cpp:28-140)
* te_tfi_input.toml       <- test/data/TE_TFI.toml (expert input file)
* te_tfi_expected.json    <- test/data/output_TE_TFI/TE_{density,onesite_obs,
  twosite_obs,multisite_obs_4,correlation_length,correlation}.dat
* afh_real_input.toml / afh_real_expected.json <- test/data/AntiferroHeisenberg_real.toml and
  output_AntiferroHeisenberg_real/{density,onesite_obs,twosite_obs,multisite_obs_4,correlation,
  correlation_length}.dat (simple update + one full-update step + CTMRG)
* {j1j2_afh,honeycomb,honeycomb_skew,afh_complex,rsvd}_{input.toml,expected.json} <- J1J2_AFH,
  Honeycomb, Honeycomb_skew, AntiferroHeisenberg_complex and RSVD (complex, rSVD up/down
  projectors) in the same form
* mt19937_seed11.json     <- draws of std::mt19937 + uniform_real_distribution
  produced by oracle/mt19937_draws.cpp compiled with the system g++
* restart_{0,1}_input.toml <- test/data/restart_{0,1}.toml (the reference's restart test,
  test/restart.py.in: save tensors, then load them)
* ft_{tfi_square,kitaev}_{input.toml,expected.json} <- FT_TFI_square and FT_Kitaev
  (finite temperature: density simple update, single-layer CTMRG, FT_{density,onesite_obs,
  twosite_obs,correlation_length,correlation}.dat)
* parameters_dat.json     <- output_*/parameters.dat of the ground-state and
  time-evolution goldens (PEPS_Parameters::save + SquareLattice::save + the
  start time), the run-dependent start_datetime value removed

The path of the TeNeS source tree is a required argument.
"""

import json
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def _rows(path):
    out = []
    with open(path) as f:
        for line in f:
            line = line.strip()
            if not line or line.startswith("#"):
                continue
            out.append([float(x) for x in line.split()])
    return out


def main(ref):
    data = os.path.join(ref, "test", "data")
    vals = [float(x) for x in open(os.path.join(data, "simple_update.dat")).read().split()]
    n = 2 * 2 * 2 * 2 * 2
    kat = {"T1": vals[:n], "T2": vals[n:2 * n], "lambda": vals[2 * n:2 * n + 2],
           "D": 2, "ldof": 2, "connect": 2, "tol": 1e-8,
           "source": "test/data/simple_update.dat; inputs test/simple_update.cpp:34-71"}
    with open(os.path.join(HERE, "simple_update_kat.json"), "w") as f:
        json.dump(kat, f, indent=1)

    vals = [float(x) for x in open(os.path.join(data, "full_update.dat")).read().split()]
    fu = {"T1": vals[:n], "T2": vals[n:2 * n], "D": 2, "ldof": 2, "chi": 4, "connect": 2, "tol": 1e-8,
          "source": "test/data/full_update.dat; inputs test/full_update.cpp:36-88"}
    with open(os.path.join(HERE, "full_update_kat.json"), "w") as f:
        json.dump(fu, f, indent=1)

    shutil.copyfile(os.path.join(data, "TE_TFI.toml"), os.path.join(HERE, "te_tfi_input.toml"))
    out = os.path.join(data, "output_TE_TFI")
    exp = {}
    for key, fname in (("density", "TE_density.dat"), ("onesite", "TE_onesite_obs.dat"),
                       ("twosite", "TE_twosite_obs.dat"), ("multisite", "TE_multisite_obs_4.dat"),
                       ("correlation_length", "TE_correlation_length.dat"),
                       ("correlation", "TE_correlation.dat")):
        exp[key] = _rows(os.path.join(out, fname))
    exp["tolerance"] = {"rtol": 1e-3, "atol": 1e-4, "source": "test/fulltest.py.in:141-142"}
    with open(os.path.join(HERE, "te_tfi_expected.json"), "w") as f:
        json.dump(exp, f)

    # ground state with one full-update step (test/data/AntiferroHeisenberg_real.toml)
    shutil.copyfile(os.path.join(data, "AntiferroHeisenberg_real.toml"), os.path.join(HERE, "afh_real_input.toml"))
    out = os.path.join(data, "output_AntiferroHeisenberg_real")
    exp = {}
    dens = {}
    for line in open(os.path.join(out, "density.dat")):
        if "=" in line:
            name, vals = line.split("=")
            dens[name.strip()] = [float(x) for x in vals.split()]
    exp["density"] = dens
    for key, fname in (("onesite", "onesite_obs.dat"), ("twosite", "twosite_obs.dat"),
                       ("multisite", "multisite_obs_4.dat"), ("correlation", "correlation.dat"),
                       ("correlation_length", "correlation_length.dat")):
        exp[key] = _rows(os.path.join(out, fname))
    exp["tolerance"] = {"rtol": 1e-3, "atol": 1e-4, "source": "test/fulltest.py.in:141-142"}
    with open(os.path.join(HERE, "afh_real_expected.json"), "w") as f:
        json.dump(exp, f)

    # further ground states with full-update steps
    for name, stem in (("J1J2_AFH", "j1j2_afh"), ("Honeycomb", "honeycomb"), ("Honeycomb_skew", "honeycomb_skew"),
                       ("AntiferroHeisenberg_complex", "afh_complex"), ("RSVD", "rsvd")):
        shutil.copyfile(os.path.join(data, name + ".toml"), os.path.join(HERE, stem + "_input.toml"))
        out = os.path.join(data, "output_" + name)
        exp = {}
        dens = {}
        for line in open(os.path.join(out, "density.dat")):
            if "=" in line:
                key, vals = line.split("=")
                dens[key.strip()] = [float(x) for x in vals.split()]
        exp["density"] = dens
        for key, fname in (("onesite", "onesite_obs.dat"), ("twosite", "twosite_obs.dat"),
                           ("multisite", "multisite_obs_4.dat"), ("correlation", "correlation.dat"),
                           ("correlation_length", "correlation_length.dat")):
            path = os.path.join(out, fname)
            if os.path.exists(path):
                exp[key] = _rows(path)
        exp["tolerance"] = {"rtol": 1e-3, "atol": 1e-4, "source": "test/fulltest.py.in:141-142"}
        with open(os.path.join(HERE, stem + "_expected.json"), "w") as f:
            json.dump(exp, f)

    for k in (0, 1):
        shutil.copyfile(os.path.join(data, f"restart_{k}.toml"), os.path.join(HERE, f"restart_{k}_input.toml"))

    # finite temperature (iTPO): density simple update + single-layer CTMRG
    for name, stem in (("FT_TFI_square", "ft_tfi_square"), ("FT_Kitaev", "ft_kitaev")):
        shutil.copyfile(os.path.join(data, name + ".toml"), os.path.join(HERE, stem + "_input.toml"))
        out = os.path.join(data, "output_" + name)
        exp = {}
        for key, fname in (("density", "FT_density.dat"), ("onesite", "FT_onesite_obs.dat"),
                           ("twosite", "FT_twosite_obs.dat"), ("correlation_length", "FT_correlation_length.dat"),
                           ("correlation", "FT_correlation.dat")):
            exp[key] = _rows(os.path.join(out, fname))
        exp["tolerance"] = {"rtol": 1e-3, "atol": 1e-4, "source": "test/fulltest.py.in:141-142"}
        with open(os.path.join(HERE, stem + "_expected.json"), "w") as f:
            json.dump(exp, f)

    pdat = {}
    for name, stem in (("TE_TFI", "te_tfi"), ("AntiferroHeisenberg_real", "afh_real"),
                       ("AntiferroHeisenberg_complex", "afh_complex"), ("RSVD", "rsvd"),
                       ("Honeycomb", "honeycomb"), ("Honeycomb_skew", "honeycomb_skew"),
                       ("J1J2_AFH", "j1j2_afh")):
        text = open(os.path.join(data, "output_" + name, "parameters.dat")).read()
        pdat[stem] = "".join(line for line in text.splitlines(keepends=True)
                             if not line.startswith("start_datetime"))
    with open(os.path.join(HERE, "parameters_dat.json"), "w") as f:
        json.dump({"files": pdat, "source": "test/data/output_*/parameters.dat, start_datetime line removed"}, f,
                  indent=1)

    with tempfile.TemporaryDirectory() as td:
        exe = os.path.join(td, "mt")
        subprocess.check_call(["g++", "-O2", "-o", exe, os.path.join(REPO, "oracle", "mt19937_draws.cpp")])
        txt = subprocess.check_output([exe, "11", "64"]).decode()
    draws = [float(x) for x in txt.split()]
    with open(os.path.join(HERE, "mt19937_seed11.json"), "w") as f:
        json.dump({"seed": 11, "uniform_pm1": draws,
                   "generator": "oracle/mt19937_draws.cpp (std::mt19937, "
                                "std::uniform_real_distribution<double>(-1, 1))"}, f)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_fixtures.py <path of the TeNeS source tree>")
    main(sys.argv[1])
