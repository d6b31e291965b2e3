"""rSVD corner projectors on weakly converged site tensors: the c3 workload's
shapes (AFH 2x2, D = 6, chi = 72) after only 20 simple-update steps, at both
precisions.  The environment of such tensors gives rank-deficient, badly
conditioned range-finder panels; every CholeskyQR of the power iteration
must still find positive pivots (the library raises otherwise) and the sweeps
must give a finite, physical energy."""
import numpy as np
import pytest

import bench

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_rsvd_sweeps_on_weakly_converged_tensors(precision):
    env = bench.make_env("c3", bench.SEED, 0, "rsvd", 20, precision)
    try:
        for _ in range(5):
            env.sweep()
        env.sync()
        e = bench.bond_energy(env)
        assert np.isfinite(e) and -1.0 < e < 0.0, e
    finally:
        env.close()
