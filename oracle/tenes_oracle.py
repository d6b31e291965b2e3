"""CPU oracle for the iTPS CTMRG path -- TEST INFRASTRUCTURE ONLY.

This module is a plain numpy (float64 / complex128) restatement of the
reference TeNeS algorithm for the CTMRG environment, the simple-update bond
step and the observables that read the environment.  Only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` may import it, and only as the checker or as the timed
CPU baseline.  The product path (``tenes_b200``) never imports it.

Every function names the reference file:line it follows (paths relative to
the TeNeS source tree).  The tensordot sequences are mirrored one for one
with ``numpy.tensordot`` / ``transpose``, whose leg conventions (free legs of
the first operand, then of the second; ``transpose(t, axes)[i] = t[axes[i]]``)
are the ones mptensor's ``tensordot`` / ``transpose`` use.

Parity pins (checked in ``tests/test_oracle_golden.py``):
  * ``test/data/simple_update.dat`` (known-answer test of the bond step).
  * ``test/data/full_update.dat`` (known-answer test of the full-update bond
    step) and ``test/data/output_AntiferroHeisenberg_real/*`` (simple update,
    one full-update step, CTMRG, observables).
  * ``test/data/output_TE_TFI/*`` (simple update + CTMRG + one-site, two-site
    and multisite observables, complex tensors, chi = 10).
The randomized SVD of mptensor (``rsvd``) is not part of the reference tree;
the rSVD here is the standard Halko et al. range finder with a counter-based
test matrix and its parity against the reference is unpinned.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np

# ---------------------------------------------------------------------------
# Random numbers: std::mt19937 + std::uniform_real_distribution<double>(-1, 1)
# as implemented by libstdc++ (generate_canonical<double, 53> draws two 32-bit
# words, low word first).  Used by iTPS::initialize_tensors
# (src/iTPS/tensors.cpp:83-128).
# ---------------------------------------------------------------------------


class MT19937:
    """Mersenne twister MT19937 (Matsumoto & Nishimura 1998), 32-bit output."""

    def __init__(self, seed: int):
        self.mt = [0] * 624
        self.mt[0] = seed & 0xFFFFFFFF
        for i in range(1, 624):
            prev = self.mt[i - 1]
            self.mt[i] = (1812433253 * (prev ^ (prev >> 30)) + i) & 0xFFFFFFFF
        self.idx = 624

    def _twist(self):
        mt = self.mt
        for i in range(624):
            y = (mt[i] & 0x80000000) | (mt[(i + 1) % 624] & 0x7FFFFFFF)
            v = mt[(i + 397) % 624] ^ (y >> 1)
            if y & 1:
                v ^= 0x9908B0DF
            mt[i] = v
        self.idx = 0

    def __call__(self) -> int:
        if self.idx >= 624:
            self._twist()
        y = self.mt[self.idx]
        self.idx += 1
        y ^= y >> 11
        y ^= (y << 7) & 0x9D2C5680
        y ^= (y << 15) & 0xEFC60000
        y ^= y >> 18
        return y & 0xFFFFFFFF


def uniform_pm1(gen: MT19937) -> float:
    """libstdc++ uniform_real_distribution<double>(-1, 1)(gen)."""
    lo = gen()
    hi = gen()
    r = (float(lo) + float(hi) * 4294967296.0) / 18446744073709551616.0
    if r >= 1.0:
        r = math.nextafter(1.0, 0.0)
    return r * 2.0 + (-1.0)


# ---------------------------------------------------------------------------
# Lattice (src/SquareLattice.hpp:54-163, src/SquareLattice.cpp:48-137)
# ---------------------------------------------------------------------------


def _cmod(a: int, b: int) -> int:
    """C++ remainder (sign follows the dividend)."""
    return int(math.fmod(a, b))


class Lattice:
    """Square unit cell with optional skew boundary (SquareLattice.cpp:48-114)."""

    def __init__(self, LX: int, LY: int, skew: int = 0):
        if LX <= 0 or LY <= 0:
            raise ValueError("Lattice.X and Lattice.Y should be positive")
        self.LX, self.LY = LX, LY
        self.N_UNIT = LX * LY
        self.skew = _cmod(skew, LX)
        self.LX_noskew = LX
        if skew == 0:
            self.LY_noskew = LY
        else:
            s = skew % LX
            self.LY_noskew = LY * ((LX * s // math.gcd(LX, s)) // s)
        self.physical_dims = [-1] * self.N_UNIT
        self.virtual_dims = [[-1] * 4 for _ in range(self.N_UNIT)]
        self.initial_dirs: List[List[float]] = [[0.0] for _ in range(self.N_UNIT)]
        self.noises = [0.0] * self.N_UNIT
        self._calc_neighbors()

    def _calc_neighbors(self):
        LX, LY = self.LX, self.LY
        tl = [[ix + iy * LX for iy in range(LY)] for ix in range(LX)]
        self._tl = tl
        nn = [[0] * 4 for _ in range(self.N_UNIT)]
        for iy in range(LY):
            for ix in range(LX):
                i = ix + iy * LX
                nn[i][0] = tl[(ix - 1 + LX) % LX][iy]
                nn[i][1] = tl[ix][(iy + 1) % LY]
                nn[i][2] = tl[(ix + 1) % LX][iy]
                nn[i][3] = tl[ix][(iy - 1 + LY) % LY]
        if self.skew != 0:
            for ix in range(LX):
                nn[ix][3] = tl[_cmod(ix + LX + self.skew, LX)][LY - 1]
                nn[self.N_UNIT + ix - LX][1] = tl[_cmod(ix + LX - self.skew, LX)][0]
        self._nn = nn
        par = [0] * self.N_UNIT
        for ix in range(LX):
            par[ix] = -1 if ix % 2 != 0 else 1
        for iy in range(1, LY):
            for ix in range(LX):
                s = self.index(ix, iy)
                par[s] = -par[self.bottom(s)]
        self._parity = par

    def index(self, x: int, y: int) -> int:
        """SquareLattice::index (SquareLattice.hpp:85-100)."""
        y_offset = 0
        if y >= self.LY:
            y_offset = y // self.LY
        elif y < 0:
            y_offset = int((y + 1) / self.LY) - 1
        y -= self.LY * y_offset
        x -= self.skew * y_offset
        x = _cmod(x, self.LX)
        if x < 0:
            x += self.LX
        return self._tl[x][y]

    def neighbor(self, i: int, d: int) -> int:
        return self._nn[i][d]

    def left(self, i):
        return self._nn[i][0]

    def top(self, i):
        return self._nn[i][1]

    def right(self, i):
        return self._nn[i][2]

    def bottom(self, i):
        return self._nn[i][3]

    def parity(self, i):
        return self._parity[i]

    def other(self, i: int, dx: int, dy: int) -> int:
        """SquareLattice::other (SquareLattice.cpp:116-137)."""
        while dx != 0:
            if dx > 0:
                i = self.right(i)
                dx -= 1
            else:
                i = self.left(i)
                dx += 1
        while dy != 0:
            if dy > 0:
                i = self.top(i)
                dy -= 1
            else:
                i = self.bottom(i)
                dy += 1
        return i


# ---------------------------------------------------------------------------
# Parameters (src/iTPS/PEPS_Parameters.cpp:30-77)
# ---------------------------------------------------------------------------


@dataclass
class Params:
    CHI: int = 2
    Inverse_projector_cut: float = 1e-12
    CTM_Convergence_Epsilon: float = 1e-6
    Max_CTM_Iteration: int = 100
    CTM_Projector_corner: bool = True
    Use_RSVD: bool = False
    RSVD_Oversampling_factor: float = 2.0
    Inverse_lambda_cut: float = 1e-12
    seed: int = 11
    # rSVD power iterations and absolute oversampling (new knobs; the
    # reference's rsvd lives in mptensor).  When rsvd_oversample_abs is not
    # None, k = cut + rsvd_oversample_abs, otherwise k = factor * cut.
    rsvd_power_iters: int = 2
    rsvd_oversample_abs: Optional[int] = None
    rsvd_seed: int = 0
    # full update (PEPS_Parameters.cpp:57-62)
    Inverse_Env_cut: float = 1e-12
    Full_Inverse_precision: float = 1e-12
    Full_Convergence_Epsilon: float = 1e-6
    Full_max_iteration: int = 100
    Full_Gauge_Fix: bool = True


def initialize_tensors(lat: Lattice, seed: int, is_real: bool) -> List[np.ndarray]:
    """iTPS::initialize_tensors (src/iTPS/tensors.cpp:38-137).

    Tn[0,0,0,0,p] = initial_state[p]; every other entry is
    noise * U(-1,1), drawn in column-major (first leg fastest) order from
    mt19937(seed) (real part) and mt19937(seed*11+137) (imaginary part).
    """
    gen = MT19937(seed)
    gen_im = MT19937(seed * 11 + 137)
    dtype = np.float64 if is_real else np.complex128
    Tn = []
    for i in range(lat.N_UNIT):
        pdim = lat.physical_dims[i]
        vd = lat.virtual_dims[i]
        ndim = vd[0] * vd[1] * vd[2] * vd[3] * pdim
        ran_re = np.empty(ndim)
        ran_im = np.empty(ndim)
        for j in range(ndim):
            ran_re[j] = uniform_pm1(gen)
            ran_im[j] = uniform_pm1(gen_im)
        d = list(lat.initial_dirs[i])
        dir_im = [0.0] * pdim
        if all(x == 0.0 for x in d):
            d = [0.0] * pdim
            for j in range(pdim):
                d[j] = uniform_pm1(gen)
                dir_im[j] = uniform_pm1(gen_im)
        # column-major linear index nr = i0 + i1*D0 + ... (tensors.cpp:121-123)
        vals = lat.noises[i] * (ran_re + 1j * ran_im)
        T = vals.reshape((pdim, vd[3], vd[2], vd[1], vd[0])).transpose(4, 3, 2, 1, 0).copy()
        for p in range(pdim):
            T[0, 0, 0, 0, p] = complex(d[p] if p < len(d) else 0.0, dir_im[p])
        Tn.append(T.real.copy() if is_real else T.astype(np.complex128))
    return Tn


# ---------------------------------------------------------------------------
# CTMRG core (src/iTPS/core/ctm.cpp)
# ---------------------------------------------------------------------------

td = np.tensordot
cj = np.conj


def _corner_block_LT(C1, eT1, eT8, Tn1):
    """LT = Tn1*(((C1*eT1)*eT8)*conj(Tn1)), legs (t12,t41,e12,e78,tc12,tc41).

    src/iTPS/core/ctm.cpp:207-212."""
    return td(Tn1, td(td(td(C1, eT1, ([1], [0])), eT8, ([0], [1])), cj(Tn1), ([2, 5], [1, 0])),
              ([0, 1, 4], [3, 1, 6]))


def _corner_block_LB(C4, eT7, eT6, Tn4):
    """LB = Tn4*(((C4*eT7)*eT6)*conj(Tn4)), legs (t41,t34,e78,e56,tc41,tc34).

    src/iTPS/core/ctm.cpp:222-227."""
    return td(Tn4, td(td(td(C4, eT7, ([1], [0])), eT6, ([0], [1])), cj(Tn4), ([2, 5], [0, 3])),
              ([0, 3, 4], [1, 3, 6]))


def _truncation(s: np.ndarray, cut: int, inv_cut: float) -> Tuple[int, np.ndarray]:
    """Keep singular values with s_i/s_0 > cutoff; return cut and 1/sqrt(s).

    src/iTPS/core/ctm.cpp:245-256 and 275-288."""
    denom = s[0]
    s_c = []
    for i in range(cut):
        if s[i] / denom > inv_cut:
            s_c.append(1.0 / math.sqrt(s[i]))
        else:
            cut = i
            break
    return cut, np.array(s_c, dtype=np.float64)


def counter_normal(shape: Sequence[int], seed: int, stream: int) -> np.ndarray:
    """Counter-based standard normals (splitmix64 + Box-Muller).

    Element n of the flattened (row-major) array uses the two 64-bit hashes of
    counters 2n and 2n+1 under key (seed, stream).  The CUDA rSVD draws the
    same numbers, so GPU and oracle rSVD see the same test matrix.
    """
    n = int(np.prod(shape))
    idx = np.arange(2 * n, dtype=np.uint64)
    key = np.uint64((seed * 0x9E3779B97F4A7C15 + stream * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF)
    with np.errstate(over="ignore"):
        z = idx * np.uint64(0x9E3779B97F4A7C15) + key
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    u = ((z >> np.uint64(11)).astype(np.float64) + 0.5) * (1.0 / 9007199254740992.0)
    u1 = u[0::2]
    u2 = u[1::2]
    r = np.sqrt(-2.0 * np.log(u1))
    return (r * np.cos(2.0 * np.pi * u2)).reshape(shape)


def rsvd_matrix(apply_M: Callable[[np.ndarray], np.ndarray],
                apply_MH: Callable[[np.ndarray], np.ndarray],
                ncol: int, k: int, q: int, seed: int, stream: int, dtype):
    """Randomized SVD (Halko, Martinsson & Tropp 2011, Alg. 4.4 + 5.1).

    apply_M(X) = M @ X, apply_MH(Y) = M^H @ Y.  Returns U, s, VH of the rank-k
    approximation.  Stand-in for mptensor::rsvd (ctm.cpp:243-244)."""
    Om = counter_normal((ncol, k), seed, stream)
    if np.iscomplexobj(np.zeros(1, dtype=dtype)):
        Om = Om + 1j * counter_normal((ncol, k), seed, stream + 1)
    Y = apply_M(Om)
    Q, _ = np.linalg.qr(Y)
    for _ in range(q):
        Z = apply_MH(Q)
        Q2, _ = np.linalg.qr(Z)
        Y = apply_M(Q2)
        Q, _ = np.linalg.qr(Y)
    B = apply_MH(Q).conj().T  # B = Q^H M  (k x ncol)
    Ub, s, VH = np.linalg.svd(B, full_matrices=False)
    return Q @ Ub, s, VH


def calc_projector_left_block(C1, C4, eT1, eT6, eT7, eT8, Tn1, Tn4, p: Params):
    """Calc_projector_left_block (src/iTPS/core/ctm.cpp:174-318)."""
    e12 = eT1.shape[1]
    e56 = eT6.shape[0]
    e78 = eT8.shape[0]
    t12 = Tn1.shape[2]
    t41 = Tn1.shape[3]
    t34 = Tn4.shape[2]
    if t41 != 1:
        LT = _corner_block_LT(C1, eT1, eT8, Tn1)
        LB = _corner_block_LB(C4, eT7, eT6, Tn4)
        if (t12 != 1 and t34 != 1) and p.Use_RSVD:
            cut = min(p.CHI, e78 * t41 * t41, e12 * t12 * t12, e56 * t34 * t34)
            k = (cut + p.rsvd_oversample_abs) if p.rsvd_oversample_abs is not None \
                else int(p.RSVD_Oversampling_factor * cut)
            nrow = t12 * e12 * t12
            ncol = t34 * e56 * t34
            k = min(k, nrow, ncol)
            # M[(r,c,rc),(r',h,rc')] = LT . LB (ctm.cpp:84-87, 119-122)

            def apply_M(X):
                Xt = X.reshape(t34, e56, t34, -1)
                return td(LT, td(LB, Xt, ([1, 3, 5], [0, 1, 2])), ([1, 3, 5], [0, 1, 2])) \
                    .reshape(nrow, -1)

            def apply_MH(Y):
                Yt = Y.reshape(t12, e12, t12, -1)
                Z = td(cj(LT), Yt, ([0, 2, 4], [0, 1, 2]))  # (s,d,sc,k)
                return td(cj(LB), Z, ([0, 2, 4], [0, 1, 2])).reshape(ncol, -1)

            U, s, VT = rsvd_matrix(apply_M, apply_MH, ncol, k, p.rsvd_power_iters,
                                   p.rsvd_seed, 0, LT.dtype)
            U = U.reshape(t12, e12, t12, -1)
            VT = VT.reshape(-1, t34, e56, t34)
        else:
            M = td(LT, LB, ([1, 3, 5], [0, 2, 4]))
            sh = M.shape
            U, s, VT = np.linalg.svd(M.reshape(sh[0] * sh[1] * sh[2], -1), full_matrices=False)
            U = U.reshape(sh[0], sh[1], sh[2], -1)
            VT = VT.reshape(-1, sh[3], sh[4], sh[5])
            cut = min(len(s), p.CHI)
        cut, s_c = _truncation(s, cut, p.Inverse_projector_cut)
        U_c = U[:, :, :, :cut] * s_c[None, None, None, :]
        VT_c = VT[:cut] * s_c[:, None, None, None]
        PU = td(LB, cj(VT_c), ([1, 3, 5], [1, 2, 3])).transpose(1, 0, 2, 3)
        PL = td(LT, cj(U_c), ([0, 2, 4], [0, 1, 2])).transpose(1, 0, 2, 3)
        return PU, PL
    eye = np.eye(e78, dtype=C1.dtype)
    return eye.reshape(e78, t41, t41, e78).copy(), eye.reshape(e78, t41, t41, e78).copy()


def calc_projector_updown_blocks(C1, C2, C3, C4, eT1, eT2, eT3, eT4, eT5, eT6, eT7, eT8,
                                 Tn1, Tn2, Tn3, Tn4, p: Params):
    """Calc_projector_updown_blocks (src/iTPS/core/ctm.cpp:320-491)."""
    e34 = eT3.shape[1]
    e78 = eT7.shape[1]
    t23 = Tn2.shape[3]
    t41 = Tn4.shape[1]
    if t41 != 1:
        LT = _corner_block_LT(C1, eT1, eT8, Tn1)
        RT = td(Tn2, td(td(td(C2, eT3, ([1], [0])), eT2, ([0], [1])), cj(Tn2), ([2, 5], [2, 1])),
                ([1, 2, 4], [3, 1, 6]))
        RB = td(Tn3, td(td(td(C3, eT5, ([1], [0])), eT4, ([0], [1])), cj(Tn3), ([2, 5], [3, 2])),
                ([2, 3, 4], [3, 1, 6]))
        LB = _corner_block_LB(C4, eT7, eT6, Tn4)
        if t23 != 1 and p.Use_RSVD:
            cut = min(p.CHI, e34 * t23 * t23)
            k = (cut + p.rsvd_oversample_abs) if p.rsvd_oversample_abs is not None \
                else int(p.RSVD_Oversampling_factor * cut)
            n = t23 * e34 * t23
            k = min(k, n)
            R1 = td(RT, LT, ([0, 3, 4], [0, 2, 4]))
            R2 = td(RB, LB, ([0, 2, 4], [1, 3, 5]))
            Mfull = td(R1, R2, ([3, 4, 5], [3, 4, 5])).reshape(n, n)
            U, s, VT = rsvd_matrix(lambda X: Mfull @ X, lambda Y: Mfull.conj().T @ Y, n, k,
                                   p.rsvd_power_iters, p.rsvd_seed, 0, LT.dtype)
            U = U.reshape(t23, e34, t23, -1)
            VT = VT.reshape(-1, t23, e34, t23)
            cut, s_c = _truncation(s, cut, p.Inverse_projector_cut)
            U_c = U[..., :cut] * s_c[None, None, None, :]
            VT_c = VT[:cut] * s_c[:, None, None, None]
            PU = td(LB, td(RB, cj(VT_c), ([1, 3, 5], [1, 2, 3])), ([1, 3, 5], [0, 1, 2])) \
                .transpose(1, 0, 2, 3)
            PL = td(LT, td(RT, cj(U_c), ([1, 2, 5], [0, 1, 2])), ([0, 2, 4], [0, 1, 2])) \
                .transpose(1, 0, 2, 3)
            return PU, PL
        R1 = td(RT, LT, ([0, 3, 4], [0, 2, 4]))
        R2 = td(RB, LB, ([0, 2, 4], [1, 3, 5]))
        M = td(R1, R2, ([3, 4, 5], [3, 4, 5]))
        sh = M.shape
        U, s, VT = np.linalg.svd(M.reshape(sh[0] * sh[1] * sh[2], -1), full_matrices=False)
        U = U.reshape(sh[0], sh[1], sh[2], -1)
        VT = VT.reshape(-1, sh[3], sh[4], sh[5])
        cut = min(len(s), p.CHI)
        cut, s_c = _truncation(s, cut, p.Inverse_projector_cut)
        U_c = U[..., :cut] * s_c[None, None, None, :]
        VT_c = VT[:cut] * s_c[:, None, None, None]
        PU = td(R2, cj(VT_c), ([0, 1, 2], [1, 2, 3])).transpose(1, 0, 2, 3)
        PL = td(R1, cj(U_c), ([0, 1, 2], [0, 1, 2])).transpose(1, 0, 2, 3)
        return PU, PL
    eye = np.eye(e78, dtype=C1.dtype)
    return eye.reshape(e78, t41, t41, e78).copy(), eye.reshape(e78, t41, t41, e78).copy()


def max_abs(t: np.ndarray) -> float:
    return float(np.max(np.abs(t)))


def calc_next_ctm(C1, C4, eT1, eT6, PU, PL):
    """Calc_Next_CTM (src/iTPS/core/ctm.cpp:493-518)."""
    C1o = td(PU, td(C1, eT1, ([1], [0])), ([0, 1, 2], [0, 2, 3]))
    C4o = td(td(eT6, C4, ([1], [0])), PL, ([3, 1, 2], [0, 1, 2]))
    return C1o / max_abs(C1o), C4o / max_abs(C4o)


def calc_next_et(eT8, Tn1, PU, PL):
    """Calc_Next_eT (src/iTPS/core/ctm.cpp:520-552)."""
    e = td(td(Tn1, td(cj(Tn1), td(eT8, PL, ([1], [0])), ([0, 1], [2, 4])), ([0, 1, 4], [4, 5, 2])),
           PU, ([1, 3, 4], [1, 2, 0])).transpose(3, 2, 0, 1)
    return e / max_abs(e)


@dataclass
class Env:
    """Corner and edge tensors of every site (iTPS.hpp:307-318)."""
    C1: List[np.ndarray]
    C2: List[np.ndarray]
    C3: List[np.ndarray]
    C4: List[np.ndarray]
    eTt: List[np.ndarray]
    eTr: List[np.ndarray]
    eTb: List[np.ndarray]
    eTl: List[np.ndarray]

    def copy(self) -> "Env":
        return Env(*[[t.copy() for t in getattr(self, n)] for n in
                     ("C1", "C2", "C3", "C4", "eTt", "eTr", "eTb", "eTl")])


def _rot(T, axes):
    return T.transpose(axes)


def _proj(env: Env, Tn, idx, p: Params, corner_args, updown_args, rot):
    if p.CTM_Projector_corner:
        return calc_projector_left_block(*corner_args, p)
    return calc_projector_updown_blocks(*updown_args, p)


def left_move(env: Env, Tn, ix: int, p: Params, lat: Lattice):
    """Left_move (src/iTPS/core/ctm.cpp:562-616)."""
    C1, C2, C3, C4 = env.C1, env.C2, env.C3, env.C4
    eTt, eTr, eTb, eTl = env.eTt, env.eTr, env.eTb, env.eTl
    LY = lat.LY_noskew
    PUs, PLs = [None] * LY, [None] * LY
    for iy in range(LY):
        i = lat.index(ix, iy)
        j = lat.right(i)
        k = lat.bottom(j)
        l = lat.left(k)
        if p.CTM_Projector_corner:
            PUs[iy], PLs[iy] = calc_projector_left_block(C1[i], C4[l], eTt[i], eTb[l], eTl[l],
                                                         eTl[i], Tn[i], Tn[l], p)
        else:
            PUs[iy], PLs[iy] = calc_projector_updown_blocks(
                C1[i], C2[j], C3[k], C4[l], eTt[i], eTt[j], eTr[j], eTr[k], eTb[k], eTb[l],
                eTl[l], eTl[i], Tn[i], Tn[j], Tn[k], Tn[l], p)
    C1b, C4b, eTlb = list(C1), list(C4), list(eTl)
    for iy in range(LY):
        i = lat.index(ix, iy)
        j = lat.right(i)
        k = lat.bottom(j)
        l = lat.left(k)
        up = (iy + 1) % LY
        dn = (iy - 1 + LY) % LY
        C1[j], C4[k] = calc_next_ctm(C1b[i], C4b[l], eTt[i], eTb[l], PUs[up], PLs[dn])
        eTl[j] = calc_next_et(eTlb[i], Tn[i], PUs[iy], PLs[up])
        eTl[k] = calc_next_et(eTlb[l], Tn[l], PUs[dn], PLs[iy])


def right_move(env: Env, Tn, ix: int, p: Params, lat: Lattice):
    """Right_move (src/iTPS/core/ctm.cpp:618-681); Tn rotated by (2,3,0,1,4)."""
    C1, C2, C3, C4 = env.C1, env.C2, env.C3, env.C4
    eTt, eTr, eTb, eTl = env.eTt, env.eTr, env.eTb, env.eTl
    R = (2, 3, 0, 1, 4)
    LY = lat.LY_noskew
    PUs, PLs = [None] * LY, [None] * LY
    for iy in range(LY):
        k = lat.index(ix, iy)
        l = lat.left(k)
        i = lat.top(l)
        j = lat.right(i)
        if p.CTM_Projector_corner:
            PUs[iy], PLs[iy] = calc_projector_left_block(C3[k], C2[j], eTb[k], eTt[j], eTr[j],
                                                         eTr[k], _rot(Tn[k], R), _rot(Tn[j], R), p)
        else:
            PUs[iy], PLs[iy] = calc_projector_updown_blocks(
                C3[k], C4[l], C1[i], C2[j], eTb[k], eTb[l], eTl[l], eTl[i], eTt[i], eTt[j],
                eTr[j], eTr[k], _rot(Tn[k], R), _rot(Tn[l], R), _rot(Tn[i], R), _rot(Tn[j], R), p)
    C2b, C3b, eTrb = list(C2), list(C3), list(eTr)
    for iy in range(LY):
        k = lat.index(ix, iy)
        l = lat.left(k)
        i = lat.top(l)
        j = lat.right(i)
        up = (iy + 1) % LY
        dn = (iy - 1 + LY) % LY
        C3[l], C2[i] = calc_next_ctm(C3b[k], C2b[j], eTb[k], eTt[j], PUs[dn], PLs[up])
        eTr[l] = calc_next_et(eTrb[k], _rot(Tn[k], R), PUs[iy], PLs[dn])
        eTr[i] = calc_next_et(eTrb[j], _rot(Tn[j], R), PUs[up], PLs[iy])


def top_move(env: Env, Tn, iy: int, p: Params, lat: Lattice):
    """Top_move (src/iTPS/core/ctm.cpp:683-746); Tn rotated by (1,2,3,0,4)."""
    C1, C2, C3, C4 = env.C1, env.C2, env.C3, env.C4
    eTt, eTr, eTb, eTl = env.eTt, env.eTr, env.eTb, env.eTl
    R = (1, 2, 3, 0, 4)
    LX = lat.LX_noskew
    PUs, PLs = [None] * LX, [None] * LX
    for ix in range(LX):
        j = lat.index(ix, iy)
        k = lat.bottom(j)
        l = lat.left(k)
        i = lat.top(l)
        if p.CTM_Projector_corner:
            PUs[ix], PLs[ix] = calc_projector_left_block(C2[j], C1[i], eTr[j], eTl[i], eTt[i],
                                                         eTt[j], _rot(Tn[j], R), _rot(Tn[i], R), p)
        else:
            PUs[ix], PLs[ix] = calc_projector_updown_blocks(
                C2[j], C3[k], C4[l], C1[i], eTr[j], eTr[k], eTb[k], eTb[l], eTl[l], eTl[i],
                eTt[i], eTt[j], _rot(Tn[j], R), _rot(Tn[k], R), _rot(Tn[l], R), _rot(Tn[i], R), p)
    C1b, C2b, eTtb = list(C1), list(C2), list(eTt)
    for ix in range(LX):
        j = lat.index(ix, iy)
        k = lat.bottom(j)
        l = lat.left(k)
        i = lat.top(l)
        rt = (ix + 1) % LX
        lf = (ix - 1 + LX) % LX
        C2[k], C1[l] = calc_next_ctm(C2b[j], C1b[i], eTr[j], eTl[i], PUs[rt], PLs[lf])
        eTt[k] = calc_next_et(eTtb[j], _rot(Tn[j], R), PUs[ix], PLs[rt])
        eTt[l] = calc_next_et(eTtb[i], _rot(Tn[i], R), PUs[lf], PLs[ix])


def bottom_move(env: Env, Tn, iy: int, p: Params, lat: Lattice):
    """Bottom_move (src/iTPS/core/ctm.cpp:748-813); Tn rotated by (3,0,1,2,4)."""
    C1, C2, C3, C4 = env.C1, env.C2, env.C3, env.C4
    eTt, eTr, eTb, eTl = env.eTt, env.eTr, env.eTb, env.eTl
    R = (3, 0, 1, 2, 4)
    LX = lat.LX_noskew
    PUs, PLs = [None] * LX, [None] * LX
    for ix in range(LX):
        l = lat.index(ix, iy)
        i = lat.top(l)
        j = lat.right(i)
        k = lat.bottom(j)
        if p.CTM_Projector_corner:
            PUs[ix], PLs[ix] = calc_projector_left_block(C4[l], C3[k], eTl[l], eTr[k], eTb[k],
                                                         eTb[l], _rot(Tn[l], R), _rot(Tn[k], R), p)
        else:
            PUs[ix], PLs[ix] = calc_projector_updown_blocks(
                C4[l], C1[i], C2[j], C3[k], eTl[l], eTl[i], eTt[i], eTt[j], eTr[j], eTr[k],
                eTb[k], eTb[l], _rot(Tn[l], R), _rot(Tn[i], R), _rot(Tn[j], R), _rot(Tn[k], R), p)
    C3b, C4b, eTbb = list(C3), list(C4), list(eTb)
    for ix in range(LX):
        l = lat.index(ix, iy)
        i = lat.top(l)
        j = lat.right(i)
        k = lat.bottom(j)
        rt = (ix + 1) % LX
        lf = (ix - 1 + LX) % LX
        C4[i], C3[j] = calc_next_ctm(C4b[l], C3b[k], eTl[l], eTr[k], PUs[lf], PLs[rt])
        eTb[i] = calc_next_et(eTbb[l], _rot(Tn[l], R), PUs[ix], PLs[lf])
        eTb[j] = calc_next_et(eTbb[k], _rot(Tn[k], R), PUs[rt], PLs[ix])


def _fit_chi(t: np.ndarray, chi: int) -> np.ndarray:
    """extend (zero pad) / slice the first two legs to chi (ctm.cpp:998-1012)."""
    d1, d2 = t.shape[0], t.shape[1]
    out = np.zeros((chi, chi) + t.shape[2:], dtype=t.dtype)
    m1, m2 = min(d1, chi), min(d2, chi)
    out[:m1, :m2] = t[:m1, :m2]
    return out


def init_env(Tn, p: Params, lat: Lattice) -> Env:
    """Environment initialisation (src/iTPS/core/ctm.cpp:984-1193).

    The merged double-layer index (ket, bra) is linearised row-major; this only
    matters when D^2 > chi (then the slice keeps a different subset)."""
    chi = p.CHI
    N = lat.N_UNIT
    C1, C2, C3, C4, eTt, eTr, eTb, eTl = ([None] * N for _ in range(8))
    for i in range(N):
        T = Tn[lat.top(lat.left(i))]
        X = td(T, cj(T), ([0, 1, 4], [0, 1, 4])).transpose(1, 3, 0, 2)
        C1[i] = _fit_chi(X.reshape(X.shape[0] * X.shape[1], -1), chi)
        T = Tn[lat.top(lat.right(i))]
        X = td(T, cj(T), ([1, 2, 4], [1, 2, 4])).transpose(0, 2, 1, 3)
        C2[i] = _fit_chi(X.reshape(X.shape[0] * X.shape[1], -1), chi)
        T = Tn[lat.bottom(lat.right(i))]
        X = td(T, cj(T), ([2, 3, 4], [2, 3, 4])).transpose(1, 3, 0, 2)
        C3[i] = _fit_chi(X.reshape(X.shape[0] * X.shape[1], -1), chi)
        T = Tn[lat.bottom(lat.left(i))]
        X = td(T, cj(T), ([0, 3, 4], [0, 3, 4])).transpose(1, 3, 0, 2)
        C4[i] = _fit_chi(X.reshape(X.shape[0] * X.shape[1], -1), chi)
        T = Tn[lat.top(i)]
        X = td(T, cj(T), ([1, 4], [1, 4])).transpose(0, 3, 1, 4, 2, 5)
        s = X.shape
        eTt[i] = _fit_chi(X.reshape(s[0] * s[1], s[2] * s[3], s[4], s[5]), chi)
        T = Tn[lat.right(i)]
        X = td(T, cj(T), ([2, 4], [2, 4])).transpose(1, 4, 2, 5, 0, 3)
        s = X.shape
        eTr[i] = _fit_chi(X.reshape(s[0] * s[1], s[2] * s[3], s[4], s[5]), chi)
        T = Tn[lat.bottom(i)]
        X = td(T, cj(T), ([3, 4], [3, 4])).transpose(2, 5, 0, 3, 1, 4)
        s = X.shape
        eTb[i] = _fit_chi(X.reshape(s[0] * s[1], s[2] * s[3], s[4], s[5]), chi)
        T = Tn[lat.left(i)]
        X = td(T, cj(T), ([0, 4], [0, 4])).transpose(2, 5, 0, 3, 1, 4)
        s = X.shape
        eTl[i] = _fit_chi(X.reshape(s[0] * s[1], s[2] * s[3], s[4], s[5]), chi)
    return Env(C1, C2, C3, C4, eTt, eTr, eTb, eTl)


def corner_spectrum(C: np.ndarray) -> np.ndarray:
    """L2-normalised singular values of a corner (ctm.cpp:830-847)."""
    s = np.linalg.svd(C, compute_uv=False)
    return s / math.sqrt(float(np.sum(s * s)))


def check_convergence(env: Env, old: Env, p: Params, lat: Lattice) -> Tuple[bool, float]:
    """Check_Convergence_CTM (src/iTPS/core/ctm.cpp:815-969), including the
    early break on the first corner whose spectrum moved by more than eps."""
    sig_max = 0.0
    for i in range(lat.N_UNIT):
        for name in ("C1", "C2", "C3", "C4"):
            ln = corner_spectrum(getattr(env, name)[i])
            lo = corner_spectrum(getattr(old, name)[i])
            n = min(len(ln), len(lo))
            sig = math.sqrt(float(np.sum((ln[:n] - lo[:n]) ** 2)) + float(np.sum(ln[n:] ** 2)))
            if sig > p.CTM_Convergence_Epsilon:
                return False, sig
            if sig > sig_max:
                sig_max = sig
    return True, sig_max


def sweep(env: Env, Tn, p: Params, lat: Lattice):
    """One CTMRG iteration: left, right, top, bottom moves (ctm.cpp:1205-1228)."""
    LX, LY = lat.LX_noskew, lat.LY_noskew
    for ix in range(LX):
        left_move(env, Tn, ix, p, lat)
    for ix in range(0, -LX, -1):
        right_move(env, Tn, (ix + 1 + LX) % LX, p, lat)
    for iy in range(0, -LY, -1):
        top_move(env, Tn, (iy + 1 + LY) % LY, p, lat)
    for iy in range(LY):
        bottom_move(env, Tn, iy, p, lat)


def calc_ctm_environment(Tn, p: Params, lat: Lattice, env: Optional[Env] = None,
                         on_sweep: Optional[Callable[[int, Env], None]] = None):
    """Calc_CTM_Environment (src/iTPS/core/ctm.cpp:971-1253).

    Returns (env, iterations, converged, sig_max)."""
    if env is None:
        env = init_env(Tn, p, lat)
    old = env.copy()
    count = 0
    conv = False
    sig_max = 0.0
    while (not conv) and count < p.Max_CTM_Iteration:
        sweep(env, Tn, p, lat)
        conv, sig_max = check_convergence(env, old, p, lat)
        count += 1
        old = env.copy()
        if on_sweep is not None:
            on_sweep(count, env)
    return env, count, conv, sig_max


# ---------------------------------------------------------------------------
# Full update (src/iTPS/core/full_update.cpp:31-455).  mptensor's matrix
# factorisations of a tensor over (row legs | column legs) are restated as
# numpy's on the reshaped matrix: qr -> Q (rows..., k), R (k, cols...);
# svd -> U (rows..., k), s, VT (k, cols...); eigh -> ascending w,
# Z (rows..., k); all thin, k = min(rows, cols).
# ---------------------------------------------------------------------------


def _split(A, rows, cols):
    A = np.transpose(A, list(rows) + list(cols))
    rs = A.shape[:len(rows)]
    cs = A.shape[len(rows):]
    return A.reshape(int(np.prod(rs)), int(np.prod(cs))), rs, cs


def _qr_legs(A, rows, cols):
    M, rs, cs = _split(A, rows, cols)
    Q, R = np.linalg.qr(M)
    return Q.reshape(rs + (-1,)), R.reshape((-1,) + cs)


def _svd_legs(A, rows, cols):
    M, rs, cs = _split(A, rows, cols)
    U, s, VT = np.linalg.svd(M, full_matrices=False)
    return U.reshape(rs + (-1,)), s, VT.reshape((-1,) + cs)


def _eigh_legs(A, rows, cols):
    M, rs, cs = _split(A, rows, cols)
    w, Z = np.linalg.eigh(M)
    return w, Z.reshape(rs + (-1,))


def _mulvec(A, v, leg):
    sh = [1] * A.ndim
    sh[leg] = -1
    return A * np.asarray(v).reshape(sh)


def _trace(A, B, a, b):
    return td(A, B, (list(a), list(b)))


def create_environment_two_sites(C1, C2, C3, C4, eT1, eT2, eT3, eT4, eT5, eT6, Q1, Q2):
    """Create_Environment_two_sites (core/full_update.cpp:50-83): the bond
    environment of two double-layer halves, legs (t1, t2, tc1, tc2)."""
    right = td(td(C2, eT2, ([0], [1])),
               td(td(td(td(C3, eT4, ([1], [0])), eT3, ([0], [1])), cj(Q2), ([2, 5], [3, 2])), Q2,
                  ([1, 3], [3, 2])),
               ([0, 2, 3], [1, 5, 3]))
    left = td(td(C1, eT1, ([1], [0])),
              td(td(td(td(C4, eT6, ([1], [0])), eT5, ([0], [1])), cj(Q1), ([2, 5], [0, 2])), Q1,
                 ([1, 3], [0, 2])),
              ([0, 2, 3], [0, 4, 2]))
    return td(right, left, ([0, 1], [0, 1])).transpose(3, 1, 2, 0)


def _pinv_t(A, cut):
    """conj(u s^-1) conj(vt) of A = u s vt, values below cut * s_0 dropped
    (the pseudo-inverse, transposed, of core/full_update.cpp:158-184)."""
    u, s, vt = np.linalg.svd(A, full_matrices=False)
    sinv = np.array([1.0 / x if x / s[0] > cut else 0.0 for x in s])
    return td(cj(u * sinv[None, :]), cj(vt), ([1], [0]))


def _fu_delta(E, Theta, R1, R2):
    """-2 <R1 R2|E|Theta> + <R1 R2|E|R1 R2> (core/full_update.cpp:238-254)."""
    ET = td(E, Theta, ([0, 1], [0, 1]))
    a = _trace(td(ET, cj(R2), ([1, 3], [0, 2])), cj(R1), (0, 1, 2), (0, 2, 1))
    b = _trace(R1, td(R2, td(E, td(cj(R1), cj(R2), ([1], [1])), ([2, 3], [0, 2])), ([0, 2], [1, 3])),
               (0, 1, 2), (1, 0, 2))
    return -2.0 * a + b


def _fu_solve(N_mat, W_vec, prec):
    """R = pinv(N) W (core/full_update.cpp:276-296, 311-329)."""
    U, s, VT = _svd_legs(N_mat, (1, 3), (0, 2))
    sinv = np.array([1.0 / x if x / s[0] > prec else 0.0 for x in s])
    N_inv = td(cj(_mulvec(U, sinv, 2)), cj(VT), ([2], [0]))
    return td(N_inv, W_vec, ([0, 1], [0, 2]))


def full_update_bond_horizontal(C1, C2, C3, C4, eT1, eT2, eT3, eT4, eT5, eT6, Tn1, Tn2, op12, p: Params):
    """Full_update_bond_horizontal (core/full_update.cpp:85-389): returns
    (Tn1_new, Tn2_new, iterations, converged)."""
    D_connect = Tn1.shape[2]
    Q1, R1 = _qr_legs(Tn1, (0, 1, 3), (2, 4))
    Q2, R2 = _qr_legs(Tn2, (1, 2, 3), (0, 4))
    envR1, envR2 = R1.shape[0], R2.shape[0]
    Theta = td(td(R1, R2, ([1], [1])), op12, ([1, 3], [0, 1]))
    E = create_environment_two_sites(C1, C2, C3, C4, eT1, eT2, eT3, eT4, eT5, eT6, Q1, Q2.transpose(3, 0, 1, 2))
    E = 0.5 * (E + cj(E.transpose(2, 3, 0, 1)))
    w, Z = _eigh_legs(E, (0, 1), (2, 3))
    w_max = abs(w[envR1 * envR2 - 1])
    w = np.array([math.sqrt(x) if x / w_max > p.Inverse_Env_cut else 0.0 for x in w])
    Z = _mulvec(Z, w, 2)
    if p.Full_Gauge_Fix:
        _, LR1 = _qr_legs(Z, (2, 1), (0,))
        _, LR2 = _qr_legs(Z, (2, 0), (1,))
        Theta = td(LR1, td(LR2, Theta, ([1], [1])), ([1], [1]))
        LR1_inv = _pinv_t(LR1, p.Inverse_Env_cut)
        LR2_inv = _pinv_t(LR2, p.Inverse_Env_cut)
        Z = td(td(Z, LR1_inv, ([0], [1])), LR2_inv, ([0], [1]))
        E = td(Z, cj(Z), ([0], [0]))
    else:
        E = td(Z, cj(Z), ([2], [2]))
    # initial guess from the SVD of Theta, truncated to D_connect
    U, s, VT = _svd_legs(Theta, (0, 2), (1, 3))
    lam = np.zeros(D_connect)
    lam[:min(D_connect, len(s))] = s[:D_connect]
    U = U[:, :, :D_connect]
    VT = VT[:D_connect]
    lam = np.sqrt(lam / math.sqrt(float(np.sum(lam * lam))))
    U = _mulvec(U, lam[:U.shape[2]], 2)
    VT = _mulvec(VT, lam[:VT.shape[0]], 0)
    R1 = U.transpose(0, 2, 1)
    R2 = VT.transpose(1, 0, 2)
    C_phi = _trace(td(E, Theta, ([0, 1], [0, 1])), cj(Theta), (0, 1, 2, 3), (0, 1, 2, 3))
    old = _fu_delta(E, Theta, R1, R2)
    count, conv = 0, False
    while not conv and count < p.Full_max_iteration:
        W = td(td(E, Theta, ([0, 1], [0, 1])), cj(R2), ([1, 3], [0, 2]))
        N = td(td(E, R2, ([1], [0])), cj(R2), ([2, 4], [0, 2]))
        R1 = _fu_solve(N, W, p.Full_Inverse_precision)
        W = td(td(E, Theta, ([0, 1], [0, 1])), cj(R1), ([0, 2], [0, 2]))
        N = td(td(E, R1, ([0], [0])), cj(R1), ([1, 4], [0, 2]))
        R2 = _fu_solve(N, W, p.Full_Inverse_precision)
        delta = _fu_delta(E, Theta, R1, R2)
        if abs(old - delta) / abs(C_phi) < p.Full_Convergence_Epsilon:
            conv = True
        old = delta
        count += 1
    if p.Full_Gauge_Fix:
        R1 = td(LR1_inv, R1, ([0], [0]))
        R2 = td(LR2_inv, R2, ([0], [0]))
    # balancing and normalisation
    q1, r1 = _qr_legs(R1, (0, 2), (1,))
    q2, r2 = _qr_legs(R2, (0, 2), (1,))
    U, s, VT = np.linalg.svd(td(r1, r2, ([1], [1])), full_matrices=False)
    n = math.sqrt(float(np.sum(s[:D_connect] ** 2)))
    s = s.copy()
    s[:D_connect] = np.sqrt(s[:D_connect] / n)
    U = U * s[None, :]
    VT = VT * s[:, None]
    R1 = td(q1, U, ([2], [0]))
    R2 = td(q2, VT, ([2], [1]))
    Tn1_new = td(Q1, R1, ([3], [0])).transpose(0, 1, 4, 2, 3)
    Tn2_new = td(Q2, R2, ([3], [0])).transpose(4, 0, 1, 2, 3)
    return Tn1_new, Tn2_new, count, conv


_FU_ROT = {0: (2, 3, 0, 1, 4), 1: (3, 0, 1, 2, 4), 2: (0, 1, 2, 3, 4), 3: (1, 2, 3, 0, 4)}
_FU_BACK = {0: (2, 3, 0, 1, 4), 1: (1, 2, 3, 0, 4), 2: (0, 1, 2, 3, 4), 3: (3, 0, 1, 2, 4)}


def full_update_bond(C1, C2, C3, C4, eT1, eT2, eT3, eT4, eT5, eT6, Tn1, Tn2, op12, connect1: int, p: Params):
    """Full_update_bond (core/full_update.cpp:391-455): the bond on leg
    connect1 of Tn1 rotated onto the horizontal case and back."""
    r = _FU_ROT[connect1]
    a, b, _, _ = full_update_bond_horizontal(C1, C2, C3, C4, eT1, eT2, eT3, eT4, eT5, eT6,
                                             Tn1.transpose(r), Tn2.transpose(r), op12, p)
    k = _FU_BACK[connect1]
    return a.transpose(k), b.transpose(k)


def full_update_op(env: "Env", Tn, source: int, leg: int, op, p: Params, lat: "Lattice",
                   fast: bool = True) -> None:
    """iTPS::full_update(up) (src/iTPS/full_update.cpp:30-149): the bond
    (source, leg) updated with the environment tensors that face it, then the
    fast full update's single moves through the two columns (rows) of the bond
    (or a full CTMRG when ``fast`` is False).  Tn and env are updated in place.
    A one-site operator (leg < 0) is applied as tensordot(Tn, op, 4, 0)."""
    if leg < 0:
        Tn[source] = td(Tn[source], op, ([4], [0]))
        return
    tgt = lat.neighbor(source, leg)
    args = full_update_env_args(env, source, leg, lat)
    Tn[source], Tn[tgt] = full_update_bond(*args, Tn[source], Tn[tgt], op, leg, p)
    _full_update_moves(env, Tn, source, tgt, leg, p, lat, fast)


def full_update_env_args(env: "Env", source: int, leg: int, lat: "Lattice"):
    """The ten environment tensors facing the bond (source, leg), in the
    argument order of Full_update_bond (src/iTPS/full_update.cpp:42-116)."""
    tgt = lat.neighbor(source, leg)
    e = env
    if leg == 0:
        args = (e.C4[source], e.C2[tgt], e.C1[tgt], e.C3[source], e.eTb[source], e.eTb[tgt], e.eTl[tgt],
                e.eTt[tgt], e.eTt[source], e.eTr[source])
    elif leg == 1:
        args = (e.C4[source], e.C1[tgt], e.C2[tgt], e.C3[source], e.eTl[source], e.eTl[tgt], e.eTt[tgt],
                e.eTr[tgt], e.eTr[source], e.eTb[source])
    elif leg == 2:
        args = (e.C1[source], e.C2[tgt], e.C3[tgt], e.C4[source], e.eTt[source], e.eTt[tgt], e.eTr[tgt],
                e.eTb[tgt], e.eTb[source], e.eTl[source])
    else:
        args = (e.C2[source], e.C3[tgt], e.C4[tgt], e.C1[source], e.eTr[source], e.eTr[tgt], e.eTb[tgt],
                e.eTl[tgt], e.eTl[source], e.eTt[source])
    return args


def _full_update_moves(env, Tn, source, tgt, leg, p, lat, fast):
    """The fast full update's single moves (src/iTPS/full_update.cpp:122-148)."""
    if not fast:
        new, _, _, _ = calc_ctm_environment(Tn, p, lat)
        for name in ("C1", "C2", "C3", "C4", "eTt", "eTr", "eTb", "eTl"):
            setattr(env, name, getattr(new, name))
        return
    LX = lat.LX
    if leg == 0:
        right_move(env, Tn, source % LX, p, lat)
        left_move(env, Tn, tgt % LX, p, lat)
    elif leg == 1:
        bottom_move(env, Tn, source // LX, p, lat)
        top_move(env, Tn, tgt // LX, p, lat)
    elif leg == 2:
        left_move(env, Tn, source % LX, p, lat)
        right_move(env, Tn, tgt % LX, p, lat)
    else:
        top_move(env, Tn, source // LX, p, lat)
        bottom_move(env, Tn, tgt // LX, p, lat)


# ---------------------------------------------------------------------------
# Simple update (src/iTPS/core/simple_update.cpp:50-198,
#                src/iTPS/simple_update.cpp:25-46)
# ---------------------------------------------------------------------------

_PERM_TO_LAST = {0: (1, 2, 3, 0, 4), 1: (0, 2, 3, 1, 4), 2: (0, 1, 3, 2, 4), 3: (0, 1, 2, 3, 4)}
_OUTER = {0: (1, 2, 3), 1: (0, 2, 3), 2: (0, 1, 3), 3: (0, 1, 2)}
_BACK1 = {0: (4, 0, 1, 2, 3), 1: (0, 4, 1, 2, 3), 2: (0, 1, 4, 2, 3), 3: (0, 1, 2, 4, 3)}
_BACK2 = {0: (3, 0, 1, 2, 4), 1: (0, 3, 1, 2, 4), 2: (0, 1, 3, 2, 4), 3: (0, 1, 2, 3, 4)}


def _scale_legs(T, lam, legs, axes_of):
    T = T.copy()
    for leg, ax in zip(legs, axes_of):
        sh = [1] * T.ndim
        sh[ax] = -1
        T = T * np.asarray(lam[leg], dtype=np.float64).reshape(sh)
    return T


def _qr_tensor(A: np.ndarray):
    """qr(A, Axes(0,1,2), Axes(3,4)) -> Q (a,b,c,k), R (k,d,p)."""
    s = A.shape
    Q, R = np.linalg.qr(A.reshape(s[0] * s[1] * s[2], s[3] * s[4]))
    return Q.reshape(s[0], s[1], s[2], -1), R.reshape(-1, s[3], s[4])


def simple_update_bond(Tn1, Tn2, lambda1, lambda2, op12, connect1: int, p: Params):
    """Simple_update_bond (src/iTPS/core/simple_update.cpp:50-198)."""
    connect2 = (connect1 + 2) % 4
    lam1_inv = [np.where(np.asarray(l) > p.Inverse_lambda_cut, 1.0 / np.maximum(np.asarray(l), 1e-300), 0.0)
                for l in lambda1]
    lam2_inv = [np.where(np.asarray(l) > p.Inverse_lambda_cut, 1.0 / np.maximum(np.asarray(l), 1e-300), 0.0)
                for l in lambda2]
    dc = Tn1.shape[connect1]
    o1 = _OUTER[connect1]
    T1 = _scale_legs(Tn1, lambda1, o1, o1).transpose(_PERM_TO_LAST[connect1])
    o2 = _OUTER[connect2]
    T2 = _scale_legs(Tn2, lambda2, o2, o2).transpose(_PERM_TO_LAST[connect2])
    Q1, R1 = _qr_tensor(T1)
    Q2, R2 = _qr_tensor(T2)
    Theta = td(td(R1, R2, ([1], [1])), op12, ([1, 3], [0, 1]))
    s0 = Theta.shape  # (c1, c2, m1o, m2o)
    U, s, VT = np.linalg.svd(Theta.transpose(0, 2, 1, 3).reshape(s0[0] * s0[2], s0[1] * s0[3]),
                             full_matrices=False)
    U = U.reshape(s0[0], s0[2], -1)
    VT = VT.reshape(-1, s0[1], s0[3])
    lam_c = s[:dc].copy()
    norm = math.sqrt(float(np.sum(lam_c * lam_c)))
    lam_c = np.sqrt(lam_c / norm)
    Uc = U[:, :, :dc] * lam_c[None, None, :]
    VTc = VT[:dc] * lam_c[:, None, None]
    Q1 = _scale_legs(Q1, lam1_inv, o1, (0, 1, 2))
    Tn1_new = td(Q1, Uc, ([3], [0])).transpose(_BACK1[connect1])
    Q2 = _scale_legs(Q2, lam2_inv, o2, (0, 1, 2))
    Tn2_new = td(Q2, VTc, ([3], [1])).transpose(_BACK2[connect2])
    return Tn1_new, Tn2_new, lam_c


# local gauge fixing of the simple update: after the transpose of
# local_gauge.cpp, leg `connect` of the contracted tensor goes back to its
# place from the last position (the physical leg is 4th before it)
_GAUGE_BACK = {0: (4, 0, 1, 2, 3), 1: (0, 4, 1, 2, 3), 2: (0, 1, 4, 2, 3), 3: (0, 1, 2, 4, 3)}


def _inv_cut(v, cut):
    v = np.asarray(v, dtype=float)
    return np.where(v > cut, 1.0 / np.maximum(v, 1e-300), 0.0)


def boundary_tensor(Tn, lam, connect: int, p: Params):
    """boundary_tensor (src/iTPS/core/local_gauge.cpp:190-224): the site
    tensor with the weights on its other three legs and the inverse weight on
    `connect`, contracted with its conjugate over every leg but `connect`:
    M[a, b] = sum conj(T)[.., a, ..] T[.., b, ..]."""
    T = Tn
    for leg in range(4):
        v = _inv_cut(lam[leg], p.Inverse_lambda_cut) if leg == connect else np.asarray(lam[leg], dtype=float)
        T = _mulvec(T, v, leg)
    rest = [l for l in range(5) if l != connect]
    return td(cj(T), T, (rest, rest))


def local_gauge_bond(Tn1, Tn2, lambda1, lambda2, connect1: int, p: Params):
    """core::fix_local_gauge (src/iTPS/core/local_gauge.cpp:44-158): bring the
    bond (Tn1 leg connect1, Tn2 leg connect1 + 2) to the gauge in which both
    boundary tensors are the identity.  Returns Tn1_new, Tn2_new, lambda_c.

    The eigenvalues of the boundary tensors are square-rooted and inverted
    without a cutoff, and the inverse weight of Tn2 is gated on
    lambda1[connect2] (local_gauge.cpp:136-142), both as the reference does."""
    connect2 = (connect1 + 2) % 4
    M1 = boundary_tensor(Tn1, lambda1, connect1, p)
    M2 = boundary_tensor(Tn2, lambda2, connect2, p)
    D1, U1 = np.linalg.eigh(M1)
    D2, U2 = np.linalg.eigh(M2)
    D1, D2 = np.sqrt(D1), np.sqrt(D2)
    U1s = U1 * np.asarray(lambda1[connect1], dtype=float)[:, None] * D1[None, :]
    U2s = U2 * np.asarray(lambda2[connect2], dtype=float)[:, None] * D2[None, :]
    W1, lam_c, W2 = np.linalg.svd(td(cj(U1s), cj(U2s), ([0], [0])), full_matrices=False)
    lam_c = np.sqrt(lam_c / math.sqrt(float(np.sum(lam_c * lam_c))))
    W1 = W1 / D1[:, None]
    W2 = W2 / D2[None, :]
    l1 = np.asarray(lambda1[connect1], dtype=float)
    inv1 = _inv_cut(l1, p.Inverse_lambda_cut)
    T1 = td(_mulvec(Tn1, inv1, connect1), U1 @ W1, ([connect1], [0])).transpose(_GAUGE_BACK[connect1])
    T1 = _mulvec(T1, lam_c, connect1)
    gate = np.asarray(lambda1[connect2], dtype=float) > p.Inverse_lambda_cut
    l2 = np.asarray(lambda2[connect2], dtype=float)
    inv2 = np.where(gate, 1.0 / np.where(gate, l2, 1.0), 0.0)
    T2 = td(_mulvec(Tn2, inv2, connect2), td(U2, W2, ([1], [1])), ([connect2], [0])).transpose(_GAUGE_BACK[connect2])
    T2 = _mulvec(T2, lam_c, connect2)
    return T1, T2, lam_c


def gauge_score(Tn, lam, lat: "Lattice", p: Params) -> float:
    """max |eigenvalue - 1| of every boundary tensor (the convergence check of
    iTPS::fix_local_gauge, src/iTPS/simple_update.cpp:80-97)."""
    score = 0.0
    for site in range(lat.N_UNIT):
        for leg in range(4):
            if lat.virtual_dims[site][leg] <= 1:
                continue
            w = np.linalg.eigvalsh(boundary_tensor(Tn[site], lam[site], leg, p))
            score = max(score, float(np.max(np.abs(w - 1.0))))
    return score


def fix_local_gauge(Tn, lam, lat: "Lattice", p: Params, maxiter: int = 100, eps: float = 1e-2):
    """iTPS::fix_local_gauge (src/iTPS/simple_update.cpp:49-101): sweeps over
    the bonds (sites of parity +1 then -1; source legs 2 then 1) until every
    boundary tensor is within eps of the identity, at most maxiter sweeps.
    Tn and lam are updated in place; returns (sweeps, score)."""
    score = float("nan")
    for it in range(maxiter):
        for parity in (1, -1):
            for sleg in (2, 1):
                tleg = (sleg + 2) % 4
                for s in range(lat.N_UNIT):
                    if lat.parity(s) != parity or lat.virtual_dims[s][sleg] <= 1:
                        continue
                    t = lat.neighbor(s, sleg)
                    T1, T2, lc = local_gauge_bond(Tn[s], Tn[t], lam[s], lam[t], sleg, p)
                    lam[s][sleg] = lc
                    lam[t][tleg] = lc
                    Tn[s] = T1
                    Tn[t] = T2
        score = gauge_score(Tn, lam, lat, p)
        if score < eps:
            return it + 1, score
    return maxiter, score


# ---------------------------------------------------------------------------
# Observables (src/iTPS/core/contract_itps_ctm/ctm.cpp)
# ---------------------------------------------------------------------------


def contract_one_site(C1, C2, C3, C4, eT1, eT2, eT3, eT4, Tn1, op1):
    """Contract_one_site_iTPS_CTM (contract_itps_ctm/ctm.cpp:89-113)."""
    X = td(td(td(C2, td(C3, eT2, ([0], [1])), ([1], [1])), td(C1, eT1, ([1], [0])), ([0], [1])),
           td(td(td(C4, eT4, ([1], [0])), eT3, ([0], [1])), cj(Tn1), ([2, 5], [0, 3])),
           ([0, 2, 3, 5], [2, 5, 0, 4]))
    W = td(X, Tn1, ([0, 1, 2, 3], [2, 1, 0, 3]))
    return complex(np.sum(W * op1.T))


def contract_two_sites_horizontal_op12(C1, C2, C3, C4, eT1, eT2, eT3, eT4, eT5, eT6, Tn1, Tn2, op12):
    """Contract_two_sites_horizontal_op12_iTPS_CTM (contract_itps_ctm/ctm.cpp:213-264)."""
    A = td(eT1, td(Tn1, td(cj(Tn1), td(eT5, td(C1, td(C4, eT6, ([1], [0])), ([0], [1])), ([1], [1])),
                               ([0, 3], [5, 2])), ([0, 3], [6, 4])), ([0, 2, 3], [7, 0, 3]))
    B = td(eT2, td(Tn2, td(cj(Tn2), td(eT4, td(C2, td(C3, eT3, ([0], [1])), ([1], [1])), ([0], [1])),
                               ([2, 3], [5, 2])), ([2, 3], [6, 4])), ([1, 2, 3], [7, 1, 4]))
    X = td(A, B, ([0, 1, 3, 5], [0, 1, 3, 5]))
    return complex(np.sum(op12 * X.transpose(0, 2, 1, 3)))


def contract_two_sites_vertical_op12(C1, C2, C3, C4, eT1, eT2, eT3, eT4, eT5, eT6, Tn1, Tn2, op12):
    """Contract_two_sites_vertical_op12_iTPS_CTM (contract_itps_ctm/ctm.cpp:266-319)."""
    A = td(eT2, td(Tn1, td(cj(Tn1), td(eT6, td(C1, td(C2, eT1, ([0], [1])), ([1], [1])), ([1], [0])),
                               ([0, 1], [2, 5])), ([0, 1], [4, 6])), ([0, 2, 3], [7, 0, 3]))
    B = td(eT3, td(Tn2, td(cj(Tn2), td(eT5, td(C3, td(C4, eT4, ([0], [1])), ([1], [1])), ([0], [1])),
                               ([0, 3], [2, 5])), ([0, 3], [4, 6])), ([1, 2, 3], [7, 1, 4]))
    X = td(A, B, ([0, 1, 3, 5], [0, 1, 3, 5]))
    return complex(np.sum(op12 * X.transpose(0, 2, 1, 3)))


def contract_window(C: Sequence[np.ndarray], eTt, eTr, eTb, eTl, Tn, op) -> complex:
    """Generic nrow x ncol window <op> (Contract_RxC_iTPS_CTM,
    contract_itps_ctm/ctm.cpp:45-87 and ctm_RxC.cpp), contracted row by row.

    Row 0 is the top row, column 0 the left column.  op[r][c] is applied as
    sum_{p,q} Tn[...,p] op[p,q] conj(Tn[...,q]), the convention of
    Contract_one_site_iTPS_CTM (ctm.cpp:111)."""
    nrow, ncol = len(Tn), len(Tn[0])
    # top boundary: legs (a, k0, kb0, ..., k_{n-1}, kb_{n-1}, b)
    B = C[0]
    for c in range(ncol):
        B = td(B, eTt[c], ([B.ndim - 1], [0]))          # (..., b', k, kb)
        B = np.moveaxis(B, B.ndim - 3, B.ndim - 1)       # (..., k, kb, b')
    B = td(B, C[1], ([B.ndim - 1], [0]))                 # (a, k.., r)
    for r in range(nrow):
        # absorb left edge: eTl (bottom, top, rk, rb); contract top with a
        B = td(eTl[r], B, ([1], [0]))                     # (a', y, yb, k0, kb0, ..., r)
        for c in range(ncol):
            T = Tn[r][c]
            Tc = cj(T)
            o = op[r][c]
            # B legs: (a', [z..done..], y, yb, k_c, kb_c, ..., r)
            pos = 1 + 2 * c
            # contract y, k_c with T legs (0,1)
            B = np.moveaxis(B, [pos, pos + 1, pos + 2, pos + 3], [B.ndim - 4, B.ndim - 3, B.ndim - 2,
                                                                    B.ndim - 1])
            # now (..., y, yb, k, kb)
            B = td(B, T, ([B.ndim - 4, B.ndim - 2], [0, 1]))  # (..., yb, kb, y', z, p)
            B = td(B, o, ([B.ndim - 1], [0]))                   # (..., yb, kb, y', z, q)
            B = td(B, Tc, ([B.ndim - 5, B.ndim - 4, B.ndim - 1], [0, 1, 4]))  # (..., y', z, yb', zb)
            # reorder to (..., z, zb, y', yb') then move back into position
            n = B.ndim
            B = B.transpose(list(range(n - 4)) + [n - 3, n - 1, n - 4, n - 2])
            B = np.moveaxis(B, [n - 4, n - 3, n - 2, n - 1], [pos, pos + 1, pos + 2, pos + 3])
        # contract right legs y, yb (at pos 1+2*ncol, 2+2*ncol) and r (last) with eTr
        n = B.ndim
        B = td(B, eTr[r], ([n - 1, n - 3, n - 2], [0, 2, 3]))  # (a', z..., r')
    # bottom: C4 (e, f), eTb[c] (right, left, uk, ub), C3 (g, h)
    X = td(C[3], B, ([1], [0]))                                 # (e, z0, zb0, ..., r')
    for c in range(ncol):
        X = td(eTb[c], X, ([1, 2, 3], [0, 1, 2]))                # (e_next, ..., r')
    val = td(X, C[2], ([0, X.ndim - 1], [1, 0]))
    return complex(val)


# ---------------------------------------------------------------------------
# Long-range correlations along a strip (contract_itps_ctm/correlation.cpp:
# StartCorrelation_iTPS_CTM, Transfer_iTPS_CTM, FinishCorrelation_iTPS_CTM;
# driver correlation_function.cpp:42-220).  The strip state A has legs
# (e1r, e3r, n1r, n2r).
# ---------------------------------------------------------------------------


def start_correlation(C1, C4, eT1, eT3, eT4, Tn1, op):
    """StartCorrelation_iTPS_CTM (contract_itps_ctm/correlation.cpp:30-57)."""
    X = td(eT3, td(C1, td(C4, eT4, ([1], [0])), ([0], [1])), ([1], [1]))
    X = td(td(cj(Tn1), op, ([4], [1])), X, ([0, 3], [5, 2]))
    X = td(Tn1, X, ([0, 3, 4], [6, 4, 2]))
    return td(eT1, X, ([0, 2, 3], [5, 0, 2])).transpose(0, 3, 1, 2)


def transfer_correlation(A, eT1, eT3, Tn1):
    """Transfer_iTPS_CTM (contract_itps_ctm/correlation.cpp:59-77)."""
    X = td(cj(Tn1), td(A, eT3, ([1], [1])), ([0, 3], [2, 5]))
    X = td(Tn1, X, ([0, 3, 4], [4, 6, 2]))
    return td(eT1, X, ([0, 2, 3], [4, 0, 2])).transpose(0, 3, 1, 2)


def finish_correlation(A, C2, C3, eT1, eT2, eT3, Tn1, op):
    """FinishCorrelation_iTPS_CTM (contract_itps_ctm/correlation.cpp:79-104)."""
    X = td(eT3, td(C2, td(C3, eT2, ([0], [1])), ([1], [1])), ([0], [1]))
    X = td(cj(Tn1), X, ([2, 3], [5, 2]))
    X = td(td(A, eT1, ([0], [0])), X, ([0, 2, 3, 5], [3, 0, 5, 1]))
    X = td(Tn1, X, ([0, 1, 2, 3], [0, 1, 4, 3]))
    return complex(np.sum(op * X))


_VROT = (3, 0, 1, 2, 4)


def correlation_strip(env: "Env", Tn, lat: "Lattice", left: int, vertical: bool, r_max: int, left_op,
                      right_ops):
    """<O_left O_right> / <1> at distances 1..r_max to the right (vertical:
    up) of `left`, as correlation_function.cpp:70-212 computes them.
    right_ops(site) lists the right operators for a site; returns
    [[value for each right op] for r in 1..r_max]."""
    e = env
    eye = lambda s: np.eye(lat.physical_dims[s], dtype=Tn[s].dtype)  # noqa: E731
    if not vertical:
        args = (e.C1[left], e.C4[left], e.eTt[left], e.eTb[left], e.eTl[left], Tn[left])
    else:
        args = (e.C4[left], e.C3[left], e.eTl[left], e.eTr[left], e.eTb[left], Tn[left].transpose(_VROT))
    A = start_correlation(*args, left_op)
    An = start_correlation(*args, eye(left))
    out = []
    site = left
    for _ in range(r_max):
        site = lat.top(site) if vertical else lat.right(site)
        if not vertical:
            fin = (e.C2[site], e.C3[site], e.eTt[site], e.eTr[site], e.eTb[site], Tn[site])
            tra = (e.eTt[site], e.eTb[site], Tn[site])
        else:
            tn = Tn[site].transpose(_VROT)
            fin = (e.C1[site], e.C2[site], e.eTl[site], e.eTt[site], e.eTr[site], tn)
            tra = (e.eTl[site], e.eTr[site], tn)
        norm = finish_correlation(An, *fin, eye(site))
        out.append([finish_correlation(A, *fin, op) / norm for op in right_ops(site)])
        A = transfer_correlation(A, *tra)
        An = transfer_correlation(An, *tra)
    return out


# ---------------------------------------------------------------------------
# Measurement driver (src/iTPS/onesite_obs.cpp:35-123, twosite_obs.cpp:31-260,
# multisite_obs.cpp:31-232, density.cpp:30-76)
# ---------------------------------------------------------------------------


@dataclass
class OneSiteOp:
    name: str
    group: int
    site: int
    op: np.ndarray
    coeff: complex = 1.0


@dataclass
class TwoSiteOp:
    name: str
    group: int
    source: int
    dx: int
    dy: int
    op: Optional[np.ndarray] = None
    ops_indices: Tuple[int, ...] = ()
    coeff: complex = 1.0


@dataclass
class MultiSiteOp:
    name: str
    group: int
    source: int
    dxs: Tuple[int, ...]
    dys: Tuple[int, ...]
    ops_indices: Tuple[int, ...]
    coeff: complex = 1.0


def _window(env: Env, Tn, lat: Lattice, source: int, source_col: int, source_row: int,
            nrow: int, ncol: int):
    idx = [[lat.other(source, c - source_col, source_row - r) for c in range(ncol)]
           for r in range(nrow)]
    C = [env.C1[idx[0][0]], env.C2[idx[0][ncol - 1]], env.C3[idx[nrow - 1][ncol - 1]],
         env.C4[idx[nrow - 1][0]]]
    eTt = [env.eTt[idx[0][c]] for c in range(ncol)]
    eTb = [env.eTb[idx[nrow - 1][c]] for c in range(ncol)]
    eTl = [env.eTl[idx[r][0]] for r in range(nrow)]
    eTr = [env.eTr[idx[r][ncol - 1]] for r in range(nrow)]
    T = [[Tn[idx[r][c]] for c in range(ncol)] for r in range(nrow)]
    return idx, C, eTt, eTr, eTb, eTl, T


def measure_onesite(env: Env, Tn, lat: Lattice, ops: Sequence[OneSiteOp], ngroups: int):
    """measure_onesite (src/iTPS/onesite_obs.cpp:35-123).  Returns
    (values[group][site], norms[site])."""
    N = lat.N_UNIT
    norm = []
    for i in range(N):
        d = Tn[i].shape[4]
        norm.append(contract_one_site(env.C1[i], env.C2[i], env.C3[i], env.C4[i], env.eTt[i],
                                      env.eTr[i], env.eTb[i], env.eTl[i], Tn[i], np.eye(d)))
    vals = [[complex("nan")] * N for _ in range(ngroups)]
    for o in ops:
        i = o.site
        v = contract_one_site(env.C1[i], env.C2[i], env.C3[i], env.C4[i], env.eTt[i], env.eTr[i],
                              env.eTb[i], env.eTl[i], Tn[i], o.op)
        vals[o.group][i] = o.coeff * v / norm[i]
    return vals, norm


def _site_op(onesite: Sequence[OneSiteOp], site: int, group: int) -> np.ndarray:
    for o in onesite:
        if o.site == site and o.group == group:
            return o.op
    raise KeyError((site, group))


def measure_twosite(env: Env, Tn, lat: Lattice, ops: Sequence[TwoSiteOp],
                    onesite: Sequence[OneSiteOp], ngroups: int):
    """measure_twosite (src/iTPS/twosite_obs.cpp:31-260).  Returns a list of
    dicts {(source, dx, dy): value} per group."""
    ret: List[Dict] = [dict() for _ in range(ngroups)]
    norms: Dict = {}
    for o in ops:
        dx, dy = o.dx, o.dy
        ncol, nrow = abs(dx) + 1, abs(dy) + 1
        if ncol > 4 or nrow > 4:
            continue
        source_col, target_col = (0, ncol - 1) if dx >= 0 else (ncol - 1, 0)
        source_row, target_row = (nrow - 1, 0) if dy >= 0 else (0, nrow - 1)
        idx, C, eTt, eTr, eTb, eTl, T = _window(env, Tn, lat, o.source, source_col, source_row,
                                                nrow, ncol)
        ident = [[np.eye(T[r][c].shape[4]) for c in range(ncol)] for r in range(nrow)]
        key = (idx[nrow - 1][0], nrow - 1, ncol - 1)
        if key not in norms:
            norms[key] = contract_window(C, eTt, eTr, eTb, eTl, T, ident)
        norm = norms[key]
        value = 0.0
        if not o.ops_indices:
            if nrow * ncol == 2:
                if nrow == 2:
                    top, bottom = idx[0][0], idx[1][0]
                    oo = o.op if top == o.source else o.op.transpose(1, 0, 3, 2)
                    value = contract_two_sites_vertical_op12(
                        env.C1[top], env.C2[top], env.C3[bottom], env.C4[bottom], env.eTt[top],
                        env.eTr[top], env.eTr[bottom], env.eTb[bottom], env.eTl[bottom],
                        env.eTl[top], T[0][0], T[1][0], oo)
                else:
                    left, right = idx[0][0], idx[0][1]
                    oo = o.op if left == o.source else o.op.transpose(1, 0, 3, 2)
                    value = contract_two_sites_horizontal_op12(
                        env.C1[left], env.C2[right], env.C3[right], env.C4[left], env.eTt[left],
                        env.eTt[right], env.eTr[right], env.eTb[right], env.eTb[left],
                        env.eTl[left], T[0][0], T[0][1], oo)
            else:
                sh = o.op.shape
                U, s, VT = np.linalg.svd(o.op.transpose(0, 2, 1, 3).reshape(sh[0] * sh[2], -1),
                                         full_matrices=False)
                U = U.reshape(sh[0], sh[2], -1)
                VT = VT.reshape(-1, sh[1], sh[3])
                for si in range(len(s)):
                    opw = [row[:] for row in ident]
                    opw[source_row][source_col] = U[:, :, si]
                    opw[target_row][target_col] = VT[si]
                    value += contract_window(C, eTt, eTr, eTb, eTl, T, opw) * s[si]
        else:
            opw = [row[:] for row in ident]
            opw[source_row][source_col] = _site_op(onesite, o.source, o.ops_indices[0])
            tgt = lat.other(o.source, dx, dy)
            opw[target_row][target_col] = _site_op(onesite, tgt, o.ops_indices[1])
            value = contract_window(C, eTt, eTr, eTb, eTl, T, opw)
        ret[o.group][(o.source, o.dx, o.dy)] = o.coeff * value / norm
    return ret, norms


def measure_multisite(env: Env, Tn, lat: Lattice, ops: Sequence[MultiSiteOp],
                      onesite: Sequence[OneSiteOp], ngroups: int):
    """measure_multisite (src/iTPS/multisite_obs.cpp:31-232)."""
    ret: List[Dict] = [dict() for _ in range(ngroups)]
    norms: Dict = {}
    for o in ops:
        mindx, maxdx = min(0, *o.dxs), max(0, *o.dxs)
        mindy, maxdy = min(0, *o.dys), max(0, *o.dys)
        ncol, nrow = maxdx - mindx + 1, maxdy - mindy + 1
        if ncol > 4 or nrow > 4:
            continue
        source_col, source_row = -mindx, maxdy
        idx, C, eTt, eTr, eTb, eTl, T = _window(env, Tn, lat, o.source, source_col, source_row,
                                                nrow, ncol)
        ident = [[np.eye(T[r][c].shape[4]) for c in range(ncol)] for r in range(nrow)]
        key = (idx[nrow - 1][0], nrow - 1, ncol - 1)
        if key not in norms:
            norms[key] = contract_window(C, eTt, eTr, eTb, eTl, T, ident)
        opw = [row[:] for row in ident]
        opw[source_row][source_col] = _site_op(onesite, o.source, o.ops_indices[0])
        for n, (dx, dy) in enumerate(zip(o.dxs, o.dys)):
            tgt = lat.other(o.source, dx, dy)
            opw[source_row - dy][source_col + dx] = _site_op(onesite, tgt, o.ops_indices[n + 1])
        value = contract_window(C, eTt, eTr, eTb, eTl, T, opw)
        ret[o.group][(o.source, o.dxs, o.dys)] = o.coeff * value / norms[key]
    return ret


# ---------------------------------------------------------------------------
# Transfer matrix and correlation length (src/iTPS/transfer_matrix.cpp:84-308,
# src/arnoldi.cpp:34-181, src/tensor.cpp:23-112, correlation_length.cpp:24-125)
# ---------------------------------------------------------------------------


def tm_matvec_horizontal(env: Env, lat: Lattice, y: int, vec: np.ndarray) -> np.ndarray:
    """TransferMatrix_ctm::matvec_horizontal (transfer_matrix.cpp:187-242)."""
    s0 = lat.index(0, y)
    s1 = lat.top(s0)
    chi0 = env.eTt[s0].shape[0]
    chi1 = env.eTb[s1].shape[1]
    v = vec.reshape(chi0, chi1)
    for x in range(lat.LX):
        site = lat.index(x, y)
        top = env.eTt[site]
        bottom = env.eTb[lat.top(site)]
        v = td(top, td(bottom, v, ([1], [1])), ([0, 2, 3], [3, 1, 2]))
    return v.reshape(-1)


def tm_matvec_vertical(env: Env, lat: Lattice, x: int, vec: np.ndarray) -> np.ndarray:
    """TransferMatrix_ctm::matvec_vertical (transfer_matrix.cpp:244-308)."""
    s0 = lat.index(x, 0)
    s1 = lat.left(s0)
    chi0 = env.eTl[s0].shape[0]
    chi1 = env.eTr[s1].shape[1]
    v = vec.reshape(chi0, chi1)
    x_orig = x
    while True:
        for y in range(lat.LY):
            site = lat.index(x, y)
            left = env.eTl[site]
            right = env.eTr[lat.left(site)]
            v = td(left, td(right, v, ([1], [1])), ([0, 2, 3], [3, 1, 2]))
        x = (x + lat.skew + lat.LX) % lat.LX
        if x == x_orig:
            break
    return v.reshape(-1)


def tm_initial_vector(env: Env, lat: Lattice, direction: int, fixed: int) -> np.ndarray:
    """TransferMatrix_ctm::initial_vector (transfer_matrix.cpp:161-185)."""
    if direction == 0:
        site = lat.index(0, fixed)
        return td(env.C1[site], env.C4[lat.top(site)], ([0], [1])).reshape(-1)
    site = lat.index(fixed, 0)
    return td(env.C4[site], env.C3[lat.left(site)], ([0], [1])).reshape(-1)


def _sorted_eigvals(h: np.ndarray, nev: int) -> np.ndarray:
    """eigen() (src/tensor.cpp:91-112): eigenvalues sorted by |.| descending."""
    w = np.linalg.eigvals(h)
    order = np.argsort(-np.abs(w) ** 2, kind="stable")
    return w[order[:nev]]


def arnoldi_eigvals(matvec, v0: np.ndarray, nev: int, maxvec: int, mindim: int, maxiter: int,
                    rtol: float) -> np.ndarray:
    """Arnoldi::initialize/run/eigenvalues (src/arnoldi.cpp:45-96) with the
    implicitly shifted restart of arnoldi.cpp:117-167."""
    N = v0.shape[0]
    dtype = np.result_type(v0.dtype, np.float64)
    Q = [np.zeros(N, dtype=dtype) for _ in range(maxvec + 1)]
    H = np.zeros((maxvec + 1, maxvec), dtype=dtype)

    def orth(k):
        for j in range(k):
            x = np.vdot(Q[j], Q[k])
            H[j, k - 1] = x
            Q[k] = Q[k] - Q[j] * x
        nrm = math.sqrt(float(np.real(np.vdot(Q[k], Q[k]))))
        Q[k] = Q[k] * (1.0 / nrm)
        if k > 0:
            H[k, k - 1] = nrm

    def residue(k):
        h = H[:k, :k]
        w, V = np.linalg.eig(h)
        order = np.argsort(-np.abs(w) ** 2, kind="stable")[:nev]
        hk = H[k, k - 1]
        return [abs(hk * V[-1, o]) / abs(w[o]) for o in order]

    Q[0] = v0.astype(dtype)
    orth(0)
    mindim = max(mindim, nev)
    for k in range(1, nev + 1):
        Q[k] = matvec(Q[k - 1])
        orth(k)
    res_nev = 1.0
    for it in range(1, maxiter + 1):
        for k in range(nev + 1, maxvec + 1):
            Q[k] = matvec(Q[k - 1])
            orth(k)
            res_nev = residue(k)[nev - 1]
            if res_nev <= rtol:
                break
        if res_nev <= rtol or it == maxiter:
            break
        # implicit restart (arnoldi.cpp:117-167)
        k = maxvec
        h = H[:maxvec, :maxvec].copy()
        w = np.linalg.eigvals(h)
        order = np.argsort(-np.abs(w) ** 2, kind="stable")
        w = w[order]
        for i in range(k - mindim):
            sigma = w[i] if np.iscomplexobj(h) else w[i].real
            q, _ = np.linalg.qr(h - sigma * np.eye(k))
            h = q.conj().T @ h @ q
            Qm = np.stack(Q[:k], axis=1) @ q
            for j in range(k):
                Q[j] = Qm[:, j].copy()
        h[np.abs(h) ** 2 < 1e-28] = 0.0
        H[:maxvec, :maxvec] = h
    return _sorted_eigvals(H[:maxvec, :maxvec], nev)


@dataclass
class TMParams:
    """TransferMatrix_Parameters defaults (transfer_matrix.hpp:29-47)."""
    num_eigvals: int = 4
    maxdim_dense_eigensolver: int = 200
    arnoldi_maxdim: int = 50
    arnoldi_restartdim: int = 20
    arnoldi_maxiter: int = 1
    arnoldi_rtol: float = 1e-10


def tm_eigenvalues(env: Env, lat: Lattice, direction: int, fixed: int, tp: TMParams,
                   matvec: Optional[Callable] = None) -> np.ndarray:
    """TransferMatrix::eigenvalues (transfer_matrix.cpp:84-142).  matvec
    (env, lat, fixed, v) replaces the double-layer matvec of the direction
    (the iTPO environment's rank-3 edges have their own)."""
    if direction == 0:
        s0 = lat.index(0, fixed)
        N = env.eTt[s0].shape[0] * env.eTb[lat.top(s0)].shape[1]
        f = matvec or tm_matvec_horizontal
    else:
        s0 = lat.index(fixed, 0)
        N = env.eTl[s0].shape[0] * env.eTr[lat.left(s0)].shape[1]
        f = matvec or tm_matvec_vertical
    mv = lambda v: f(env, lat, fixed, v)  # noqa: E731
    nev = min(tp.num_eigvals, N)
    if N == 1:
        return np.array([1.0 + 0j])
    if N <= tp.maxdim_dense_eigensolver:
        dt = env.eTt[0].dtype
        M = np.stack([mv(e) for e in np.eye(N, dtype=dt)], axis=1)
        return _sorted_eigvals(M, nev)
    maxvec, maxiter = tp.arnoldi_maxdim, tp.arnoldi_maxiter
    if N < maxvec:
        maxvec, maxiter = N, 1
    v0 = tm_initial_vector(env, lat, direction, fixed)
    return arnoldi_eigvals(mv, v0, nev, maxvec, tp.arnoldi_restartdim, maxiter, tp.arnoldi_rtol)


def correlation_length(eigvals: np.ndarray, L: int) -> Tuple[float, List[float]]:
    """xi = -L / ln|t1/t0| and e_i = -ln|t_i/t_0| / L (correlation_length.cpp:99-118)."""
    if len(eigvals) == 1:
        return 0.0, []
    e0 = abs(eigvals[0])
    e1 = abs(eigvals[1]) / e0
    xi = -L / math.log(e1)
    return xi, [-math.log(abs(e) / e0) / L for e in eigvals[1:]]
