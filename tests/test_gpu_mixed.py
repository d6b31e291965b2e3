"""Mixed-precision CTMRG (3xTF32 tensor-core contractions, FP64 projector
algebra) against the FP64 path.  Tolerances are those of 3xTF32 products
(~1e-7 relative per product), not FP64 rounding."""
import numpy as np
import pytest

from oracle import tenes_oracle as O
from tenes_b200.std_ops import heisenberg_bond
from tests._helpers import (gpu_env, load_env, make_lattice, oracle_params, physical_tensors)

pytestmark = pytest.mark.gpu


def test_mixed_single_move_close_to_fp64():
    lat = make_lattice(2, 2, 3)
    Tn = physical_tensors(lat, 3)
    chi = 12
    p = oracle_params(chi)
    oe = O.init_env(Tn, p, lat)
    O.sweep(oe, Tn, p, lat)
    ge = gpu_env(lat, Tn, chi, False, mixed=True)
    load_env(ge, oe)
    O.left_move(oe, Tn, 0, p, lat)
    ge.move(0, 0)
    for w, name in enumerate(("C1", "C2", "C3", "C4", "eTt", "eTr", "eTb", "eTl")):
        for i in range(lat.N_UNIT):
            np.testing.assert_allclose(np.abs(ge.get_env(w, i)), np.abs(getattr(oe, name)[i]), rtol=0,
                                       atol=2e-5, err_msg=f"{name}[{i}]")


def _energy(env, lat):
    H = heisenberg_bond(1.0).real
    I = np.einsum("ac,bd->abcd", np.eye(2), np.eye(2))
    E = 0.0
    for i in range(lat.N_UNIT):
        for dx, dy in ((1, 0), (0, 1)):
            E += (env.contract_bond_op12(i, dx, dy, H) / env.contract_bond_op12(i, dx, dy, I)).real
    return E / lat.N_UNIT


@pytest.mark.parametrize("rsvd", [False, True])
def test_mixed_energy_close_to_fp64(rsvd):
    lat = make_lattice(2, 2, 3)
    Tn = physical_tensors(lat, 3, steps=60)
    chi, iters = 18, 12
    kw = dict(max_ctm_iteration=iters)
    if rsvd:
        kw.update(use_rsvd=True, rsvd_oversample_abs=10, rsvd_power_iters=2)
    e64 = gpu_env(lat, Tn, chi, False, **kw)
    e64.calc_ctm_environment(True)
    emx = gpu_env(lat, Tn, chi, False, mixed=True, **kw)
    emx.calc_ctm_environment(True)
    E64, Emx = _energy(e64, lat), _energy(emx, lat)
    assert abs(E64 - Emx) < 1e-6, (E64, Emx)
