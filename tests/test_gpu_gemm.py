"""The contraction kernels against numpy FP64: the FP64 DMMA product to
rounding, and the 3xTF32 tcgen05 product (FP32 accumulation over K chunks of
at most 1024, summed in FP64) to the accuracy of an FP32 product:
|C - C_ref| <= 2e-6 * (|A| |B|) elementwise."""
import ctypes as C

import numpy as np
import pytest

from tenes_b200 import _lib
from tenes_b200._lib import check, dptr

pytestmark = pytest.mark.gpu


def _run(A, B, layout_a, layout_b, layout_c, prec, seed_c=None):
    """C = A B through tg_gemm_host with the requested row/column-major layouts."""
    M, K = A.shape
    N = B.shape[1]
    a = np.ascontiguousarray(A if layout_a == "r" else A.T)
    sAm, sAk = (K, 1) if layout_a == "r" else (1, M)
    b = np.ascontiguousarray(B if layout_b == "r" else B.T)
    sBk, sBn = (N, 1) if layout_b == "r" else (1, K)
    c = np.zeros((M, N) if layout_c == "r" else (N, M))
    sCm, sCn = (N, 1) if layout_c == "r" else (1, M)
    check(_lib.load().tg_gemm_host(M, N, K, dptr(a), sAm, sAk, dptr(b), sBk, sBn, dptr(c), sCm, sCn, prec))
    return c if layout_c == "r" else c.T


SHAPES = [(128, 128, 16), (200, 37, 100), (36, 1000, 72), (1000, 36, 72), (2592, 82, 2592), (130, 257, 1030),
          (1, 1, 1), (17, 300, 5),
          # one side <= 96 and the other >= 2048: the streaming kernel for long operands
          (36, 5000, 72), (5000, 72, 36), (72, 4100, 35), (4099, 17, 96), (96, 4096, 1), (5, 6000, 3),
          (2592, 82, 82), (72, 2592, 72), (2048, 96, 96),
          # FP64: one narrow column tile (64 < N <= 96, a multiple of 8 columns), with and without
          # split-K; N <= 64 stays on 64-wide tiles
          (300, 90, 500), (700, 95, 16), (1500, 72, 200), (4000, 72, 64), (130, 250, 2000),
          (500, 36, 700), (3000, 20, 300), (257, 5, 1000), (129, 41, 2100), (64, 88, 3000), (2592, 82, 2600)]


@pytest.mark.parametrize("M,N,K", SHAPES)
@pytest.mark.parametrize("prec", [0, 1])
def test_gemm_matches_numpy(M, N, K, prec):
    rng = np.random.default_rng(M * 7 + N * 3 + K)
    A = rng.standard_normal((M, K))
    B = rng.standard_normal((K, N))
    ref = A @ B
    bound = np.abs(A) @ np.abs(B)
    for la, lb, lc in [("r", "r", "r"), ("c", "c", "c"), ("r", "c", "r"), ("c", "r", "c")]:
        got = _run(A, B, la, lb, lc, prec)
        err = np.abs(got - ref)
        if prec == 0:
            assert np.all(err <= 1e-13 * bound + 1e-300), (la, lb, lc, err.max())
        else:
            assert np.all(err <= 2e-6 * bound), (la, lb, lc, (err / bound).max())


def test_tf32x3_is_more_accurate_than_one_tf32_product():
    """The hi/lo split recovers ~FP32 accuracy: far below TF32's 2^-11."""
    rng = np.random.default_rng(5)
    A = rng.standard_normal((256, 512))
    B = rng.standard_normal((512, 96))
    got = _run(A, B, "r", "r", "r", 1)
    rel = np.abs(got - A @ B) / (np.abs(A) @ np.abs(B))
    assert rel.max() < 1e-6


def _group(probs, is_complex):
    """probs: list of (A, B, flags) -> C_i through tg_gemm_group_host."""
    mnk, flags, a_parts, b_parts = [], [], [], []
    for A, B, f in probs:
        M, K = A.shape
        N = B.shape[1]
        mnk += [M, N, K]
        flags.append(f)
        a_parts.append((A.T if f & 1 else A).ravel())
        b_parts.append((B.T if f & 2 else B).ravel())
    dt = np.complex128 if is_complex else np.float64
    a = np.ascontiguousarray(np.concatenate(a_parts).astype(dt))
    b = np.ascontiguousarray(np.concatenate(b_parts).astype(dt))
    n_c = sum(A.shape[0] * B.shape[1] for A, B, _ in probs)
    c = np.zeros(n_c, dtype=dt)
    m = np.array(mnk, dtype=np.int64)
    fl = np.array(flags, dtype=np.int32)
    as_d = lambda x: x.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
    check(_lib.load().tg_gemm_group_host(len(probs), m.ctypes.data_as(C.POINTER(C.c_int64)),
                                         fl.ctypes.data_as(C.POINTER(C.c_int)), int(is_complex), as_d(a), as_d(b),
                                         as_d(c)))
    out, off = [], 0
    for A, B, _ in probs:
        sz = A.shape[0] * B.shape[1]
        out.append(c[off:off + sz].reshape(A.shape[0], B.shape[1]))
        off += sz
    return out


@pytest.mark.parametrize("is_complex", [False, True])
def test_gemm_group_matches_numpy(is_complex):
    """The grouped persistent product over problems of uneven shapes (tiles of
    one problem and ragged edges in every dimension), every operand layout and,
    for complex operands, conjugation, against numpy; complex products are 3M:
    the error is bounded by the moduli of the real and imaginary parts."""
    rng = np.random.default_rng(11 + int(is_complex))
    shapes = [(72, 2592, 72), (300, 36, 500), (1, 1, 1), (65, 129, 17), (200, 90, 1000), (37, 5, 3),
              (1024, 64, 64), (7, 300, 250)]
    probs = []
    for n, (M, N, K) in enumerate(shapes):
        A = rng.standard_normal((M, K))
        B = rng.standard_normal((K, N))
        if is_complex:
            A = A + 1j * rng.standard_normal((M, K))
            B = B + 1j * rng.standard_normal((K, N))
        probs.append((A, B, n % (16 if is_complex else 4)))
    got = _group(probs, is_complex)
    for (A, B, f), g in zip(probs, got):
        Ao = A.conj() if f & 4 else A
        Bo = B.conj() if f & 8 else B
        ref = Ao @ Bo
        bound = (np.abs(A.real) + np.abs(A.imag)) @ (np.abs(B.real) + np.abs(B.imag))
        err = np.abs(g - ref)
        assert np.all(err <= 2e-13 * bound + 1e-300), (A.shape, B.shape, f, (err / bound).max())
    tuned = C.c_int64()
    wins = (C.c_int64 * 2)()
    check(_lib.load().tg_gemm_group_stats(C.byref(tuned), wins, 2))
    assert tuned.value >= 1 and wins[0] + wins[1] == tuned.value


def test_gemm_group_more_problems_than_one_launch_holds():
    """More problems than one launch's table (24): the rest go to further launches."""
    rng = np.random.default_rng(3)
    probs = [(rng.standard_normal((20 + i, 30)), rng.standard_normal((30, 10 + 3 * i)), i % 4) for i in range(30)]
    for (A, B, _), g in zip(probs, _group(probs, False)):
        np.testing.assert_allclose(g, A @ B, rtol=0, atol=1e-12 * np.abs(A).max() * np.abs(B).max() * 30)
