"""Local gauge fixing on the GPU (tg_su_fix_gauge) against the oracle's
iTPS::fix_local_gauge restatement (src/iTPS/simple_update.cpp:49-101,
core/local_gauge.cpp:44-224): sweep count, score and bond weights, which the
SVD and eigensolver sign choices leave alone, and the state itself up to those
gauges (the one-site reduced density matrices of the weighted tensors)."""

import numpy as np
import pytest

from oracle import tenes_oracle as O
from tests._helpers import gpu_env
from tests.test_local_gauge import su_state

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("is_complex", [False, True])
@pytest.mark.parametrize("maxiter,eps", [(1, 1e-2), (100, 1e-8)])
def test_fix_local_gauge_matches_oracle(is_complex, maxiter, eps):
    lat, Tn, lam, p = su_state(is_complex, seed=3)
    ge = gpu_env(lat, Tn, 4, is_complex)
    for i in range(lat.N_UNIT):
        for leg in range(4):
            ge.set_lambda(i, leg, lam[i][leg])
    sweeps, score = ge.fix_local_gauge(maxiter, eps)
    o_sweeps, o_score = O.fix_local_gauge(Tn, lam, lat, p, maxiter=maxiter, eps=eps)
    assert sweeps == o_sweeps
    assert abs(score - o_score) <= 1e-8 * max(1.0, o_score)
    for i in range(lat.N_UNIT):
        for leg in range(4):
            np.testing.assert_allclose(ge.get_lambda(i, leg), lam[i][leg], rtol=1e-9, atol=1e-12)
        # sum over the virtual legs of T conj(T): invariant under the bond gauges
        a, b = ge.get_site_tensor(i), Tn[i]
        np.testing.assert_allclose(np.tensordot(a, a.conj(), ([0, 1, 2, 3], [0, 1, 2, 3])),
                                   np.tensordot(b, b.conj(), ([0, 1, 2, 3], [0, 1, 2, 3])), rtol=1e-8, atol=1e-11)
    ge.close()
