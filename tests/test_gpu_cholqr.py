"""The one-launch cluster CholeskyQR of the rSVD range finder against numpy:
orthonormality of the result, its span against the input's, and equality
with the Q of a Householder QR (positive diagonal) for full-rank panels.
Rank-deficient panels (zero rows, dependent columns) still give an
orthonormal basis containing the input's span, which is what the shifted
passes and the perturbation after the first pass are for."""
import ctypes as C

import numpy as np
import pytest

from tenes_b200 import _lib
from tenes_b200._lib import check, dptr

pytestmark = pytest.mark.gpu


def cholqr(Y, passes):
    y = np.asfortranarray(Y).copy(order="F")
    n, k = Y.shape
    flag = C.c_int(0)
    buf = np.ascontiguousarray(y.T)  # column-major n x k = row-major k x n
    check(_lib.load().tg_cholqr_host(n, k, dptr(buf), passes, C.byref(flag)))
    return buf.T.copy(), flag.value


def panel(n, k, cond, seed):
    rng = np.random.default_rng(seed)
    U, _ = np.linalg.qr(rng.standard_normal((n, k)))
    V, _ = np.linalg.qr(rng.standard_normal((k, k)))
    s = np.logspace(0, -np.log10(cond), k) if k > 1 else np.ones(1)
    return (U * s) @ V.T


@pytest.mark.parametrize("n,k", [(2592, 82), (2592, 96), (5000, 90), (300, 17), (64, 64), (37, 5), (5, 3),
                                 (9, 1)])
@pytest.mark.parametrize("passes", [2, 4])
def test_orthonormal_and_same_span(n, k, passes):
    Y = panel(n, k, 1e6, n + k)
    Q, flag = cholqr(Y, passes)
    assert flag == 0
    orth = np.abs(Q.T @ Q - np.eye(k)).max()
    # two shifted passes leave a basis with condition number ~1e4 at most; four are orthonormal to rounding
    assert orth <= (1e-2 if passes == 2 else 1e-13 * max(1, k / 32)), orth
    Qo, _ = np.linalg.qr(Q)
    resid = np.linalg.norm(Y - Qo @ (Qo.T @ Y)) / np.linalg.norm(Y)
    assert resid <= 1e-12, resid


@pytest.mark.parametrize("n,k", [(2592, 82), (1000, 40)])
def test_equals_householder_q(n, k):
    Y = panel(n, k, 1e3, 7 * n + k)
    Q, flag = cholqr(Y, 4)
    assert flag == 0
    Qh, R = np.linalg.qr(Y)
    Qh = Qh * np.sign(np.diag(R))
    # the 1e-14 perturbation and rounding amplified by the condition number 1e3
    assert np.abs(Q - Qh).max() <= 1e-10


def test_rank_deficient_panel():
    n, k = 2592, 82
    rng = np.random.default_rng(3)
    Y = panel(n, 60, 1e4, 11) @ rng.standard_normal((60, k))  # rank 60
    Y[::3] = 0.0  # exactly-zero rows, as zero-padded environment legs give
    Q, flag = cholqr(Y, 4)
    assert flag == 0
    assert np.abs(Q.T @ Q - np.eye(k)).max() <= 1e-12
    resid = np.linalg.norm(Y - Q @ (Q.T @ Y)) / np.linalg.norm(Y)
    assert resid <= 1e-12, resid
