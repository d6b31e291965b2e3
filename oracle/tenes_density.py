"""CPU oracle for the iTPO (finite-temperature) path -- TEST INFRASTRUCTURE ONLY.

A plain numpy restatement of TeNeS's density-operator branch:

* the single-layer CTMRG of src/iTPS/core/ctm_single.cpp (environment of the
  traced tensors Tn_single = sum_p Tn[..., p, p], corner and up/down
  projectors, Next_CTM / Next_eT, the four moves, initialisation and the
  convergence loop of Calc_CTM_Environment_density);
* the density contractions of src/iTPS/core/contract_density_ctm/ (one site,
  nearest-neighbour op12, R x C windows of one-site operators, the
  correlation strip) and the rank-3 transfer matrix of
  src/iTPS/transfer_matrix.cpp:187-308;
* the density simple update (src/iTPS/simple_update.cpp:141-178) and the
  finite-temperature driver (src/iTPS/finite_temperature.cpp:22-86 with
  measure.cpp:110-144).

Only ``tests/`` and the CPU legs of ``bench.py`` may import it.  Leg orders
follow mptensor's tensordot / transpose, as numpy's do.  Edge tensors are
rank 3 (chi, chi, D) and unpadded: their first two legs grow from the bond
dimensions of the initial environment to chi as the reference's do.

Parity pins (tests/test_oracle_density.py): test/data/output_FT_TFI_square and
test/data/output_FT_Kitaev (the reference's own finite-temperature runs).
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

from oracle import tenes_oracle as O

td = np.tensordot
cj = np.conj


def single_tensor(T: np.ndarray) -> np.ndarray:
    """Make_single_tensor_density (ctm_single.cpp:43-50): trace over the two
    physical legs (4, 5)."""
    return np.einsum("abcdpp->abcd", T)


# ---------------------------------------------------------------------------
# Environment initialisation (ctm_single.cpp:752-960): every corner / edge is
# the traced tensor of the neighbouring site summed over its outer legs (a
# contraction with all-ones vectors), not padded to chi.
# ---------------------------------------------------------------------------


@dataclass
class Env:
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


def init_env(Ts: Sequence[np.ndarray], lat: O.Lattice) -> Env:
    N = lat.N_UNIT
    C1, C2, C3, C4, eTt, eTr, eTb, eTl = ([None] * N for _ in range(8))
    for i in range(N):
        A = Ts[lat.top(lat.left(i))]
        C1[i] = A.sum(axis=(0, 1)).transpose(1, 0)          # (b, r)
        A = Ts[lat.top(lat.right(i))]
        C2[i] = A.sum(axis=(1, 2))                           # (l, b)
        A = Ts[lat.bottom(lat.right(i))]
        C3[i] = A.sum(axis=(2, 3)).transpose(1, 0)          # (t, l)
        A = Ts[lat.bottom(lat.left(i))]
        C4[i] = A.sum(axis=(0, 3)).transpose(1, 0)          # (r, t)
        eTt[i] = Ts[lat.top(i)].sum(axis=1)                  # (l, r, b)
        eTr[i] = Ts[lat.right(i)].sum(axis=2).transpose(1, 2, 0)   # (t, b, l)
        eTb[i] = Ts[lat.bottom(i)].sum(axis=3).transpose(2, 0, 1)  # (r, l, t)
        eTl[i] = Ts[lat.left(i)].sum(axis=0).transpose(2, 0, 1)    # (b, t, r)
    return Env(C1, C2, C3, C4, eTt, eTr, eTb, eTl)


# ---------------------------------------------------------------------------
# Projectors (ctm_single.cpp:125-436)
# ---------------------------------------------------------------------------


def _LT(C1, eT1, eT8, T1):
    """(((C1*eT1)*eT8)*Tn1_s), legs (e78, t41, e12, t12) (ctm_single.cpp:149-153)."""
    return td(td(td(C1, eT1, ([1], [0])), eT8, ([0], [1])), T1, ([1, 3], [1, 0])).transpose(1, 3, 0, 2)


def _LB(C4, eT7, eT6, T4):
    """(((C4*eT7)*eT6)*Tn4_s), legs (e78, t41, e56, t34) (ctm_single.cpp:162-166)."""
    return td(td(td(C4, eT7, ([1], [0])), eT6, ([0], [1])), T4, ([1, 3], [0, 3])).transpose(0, 2, 1, 3)


def _RT(C2, eT3, eT2, T2):
    """(((C2*eT3)*eT2)*Tn2_s), legs (e12, t12, e34, t23) (ctm_single.cpp:306-310)."""
    return td(td(td(C2, eT3, ([1], [0])), eT2, ([0], [1])), T2, ([1, 3], [2, 1])).transpose(1, 2, 0, 3)


def _RB(C3, eT5, eT4, T3):
    """(((C3*eT5)*eT4)*Tn3_s), legs (e56, t34, e34, t23) (ctm_single.cpp:319-323)."""
    return td(td(td(C3, eT5, ([1], [0])), eT4, ([0], [1])), T3, ([1, 3], [3, 2])).transpose(0, 2, 1, 3)


def _sketch(p: O.Params, cut: int) -> int:
    if p.rsvd_oversample_abs is not None:
        return cut + p.rsvd_oversample_abs
    return int(p.RSVD_Oversampling_factor * cut)


def _weights(s: np.ndarray, cut: int, bound: int, thr: float) -> Tuple[int, np.ndarray]:
    """The truncation loops of ctm_single.cpp (206-216, 229-239, 368-378,
    400-410): s_c = 1/sqrt(s_i) while s_i/s_0 > thr, for i < bound; a value
    at or below thr ends the loop and sets cut to its index.  Entries in
    [bound, cut) stay 0 (s_c is zero-initialised to length cut)."""
    denom = s[0]
    w = np.zeros(cut)
    for i in range(bound):
        if i >= len(s):
            break
        if s[i] / denom > thr:
            if i < cut:
                w[i] = 1.0 / math.sqrt(s[i])
        else:
            cut = i
            break
    out = np.zeros(cut)
    n = min(cut, len(w))
    out[:n] = w[:n]
    return cut, out


def proj_left_block(C1, C4, eT1, eT6, eT7, eT8, T1, T4, p: O.Params):
    """Calc_projector_left_block_single (ctm_single.cpp:125-265)."""
    e12, e56, e78 = eT1.shape[1], eT6.shape[0], eT8.shape[0]
    t12, t41, t34 = T1.shape[2], T1.shape[3], T4.shape[2]
    if t41 == 1:
        eye = np.eye(e78, dtype=C1.dtype)
        return eye.reshape(e78, 1, e78).copy(), eye.reshape(e78, 1, e78).copy()
    LT = _LT(C1, eT1, eT8, T1).reshape(e78 * t41, e12 * t12)
    LB = _LB(C4, eT7, eT6, T4).reshape(e78 * t41, e56 * t34)
    cut = min(p.CHI, e78 * t41, e12 * t12, e56 * t34)
    if t12 != 1 and t34 != 1 and p.Use_RSVD:
        k = min(_sketch(p, cut), e12 * t12, e56 * t34)
        U, s, VT = O.rsvd_matrix(lambda X: LT.T @ (LB @ X), lambda Y: cj(LB).T @ (cj(LT) @ Y),
                                 e56 * t34, k, p.rsvd_power_iters, p.rsvd_seed, 0, LT.dtype)
    else:
        U, s, VT = np.linalg.svd(LT.T @ LB, full_matrices=False)
    cut, w = _weights(s, cut, cut, p.Inverse_projector_cut)
    U_c = U[:, :cut] * w[None, :]
    VT_c = VT[:cut] * w[:, None]
    PU = (LB @ cj(VT_c).T).reshape(e78, t41, cut)
    PL = (LT @ cj(U_c)).reshape(e78, t41, cut)
    return PU, PL


def proj_updown(C1, C2, C3, C4, eT1, eT2, eT3, eT4, eT5, eT6, eT7, eT8, T1, T2, T3, T4, p: O.Params,
                edge_bound: bool = True):
    """Calc_projector_updown_blocks_single (ctm_single.cpp:267-436).

    The full-SVD branch's truncation loop runs over i < e78 (the edge
    dimension) rather than i < cut (ctm_single.cpp:403); edge_bound=True
    keeps that, False runs it over i < cut as the rSVD branch does."""
    e12, e34, e56, e78 = eT1.shape[1], eT3.shape[1], eT5.shape[1], eT7.shape[1]
    t12, t23, t34, t41 = T1.shape[2], T2.shape[3], T3.shape[0], T4.shape[1]
    if t41 == 1:
        eye = np.eye(e78, dtype=C1.dtype)
        return eye.reshape(e78, 1, e78).copy(), eye.reshape(e78, 1, e78).copy()
    LT = _LT(C1, eT1, eT8, T1).reshape(e78 * t41, e12 * t12)
    RT = _RT(C2, eT3, eT2, T2).reshape(e12 * t12, e34 * t23)
    RB = _RB(C3, eT5, eT4, T3).reshape(e56 * t34, e34 * t23)
    LB = _LB(C4, eT7, eT6, T4).reshape(e78 * t41, e56 * t34)
    cut = min(p.CHI, e34 * t23)
    if t23 != 1 and p.Use_RSVD:
        n = e34 * t23
        k = min(_sketch(p, cut), n)
        # Mult_col_ud_single: RT^T (LT^T (LB (RB X)))  (ctm_single.cpp:80-101)
        U, s, VT = O.rsvd_matrix(lambda X: RT.T @ (LT.T @ (LB @ (RB @ X))),
                                 lambda Y: cj(RB).T @ (cj(LB).T @ (cj(LT) @ (cj(RT) @ Y))),
                                 n, k, p.rsvd_power_iters, p.rsvd_seed, 0, LT.dtype)
        cut, w = _weights(s, cut, cut, p.Inverse_projector_cut)
        U_c = U[:, :cut] * w[None, :]
        VT_c = VT[:cut] * w[:, None]
        PU = (LB @ (RB @ cj(VT_c).T)).reshape(e78, t41, cut)
        PL = (LT @ (RT @ cj(U_c))).reshape(e78, t41, cut)
        return PU, PL
    R1 = RT.T @ LT.T          # tensordot(RT, LT, (0), (1)): (e34 t23, e78 t41)
    R2 = RB.T @ LB.T          # tensordot(RB, LB, (0), (1))
    U, s, VT = np.linalg.svd(R1 @ R2.T, full_matrices=False)
    cut, w = _weights(s, cut, e78 if edge_bound else cut, p.Inverse_projector_cut)
    U_c = U[:, :cut] * w[None, :]
    VT_c = VT[:cut] * w[:, None]
    PU = (R2.T @ cj(VT_c).T).reshape(e78, t41, cut)
    PL = (R1.T @ cj(U_c)).reshape(e78, t41, cut)
    return PU, PL


def next_ctm(C1, C4, eT1, eT6, PU, PL):
    """Calc_Next_CTM_single (ctm_single.cpp:438-451)."""
    C1o = td(PU, td(C1, eT1, ([1], [0])), ([0, 1], [0, 2]))
    C4o = td(td(eT6, C4, ([1], [0])), PL, ([2, 1], [0, 1]))
    return C1o / O.max_abs(C1o), C4o / O.max_abs(C4o)


def next_et(eT8, T1, PU, PL):
    """Calc_Next_eT_single (ctm_single.cpp:453-473)."""
    e = td(td(T1, td(eT8, PL, ([1], [0])), ([0, 1], [1, 2])), PU, ([1, 2], [1, 0])).transpose(2, 1, 0)
    return e / O.max_abs(e)


# ---------------------------------------------------------------------------
# Moves (ctm_single.cpp:483-735): the pairing of projectors and the update
# order of Left/Right/Top/Bottom_move_single are those of the double-layer
# moves; the site tensors are rotated by (2,3,0,1), (1,2,3,0), (3,0,1,2).
# ---------------------------------------------------------------------------

_RR, _RT_, _RBm = (2, 3, 0, 1), (1, 2, 3, 0), (3, 0, 1, 2)


def _projectors(corner_args, updown_args, p, edge_bound):
    if p.CTM_Projector_corner:
        return proj_left_block(*corner_args, p)
    return proj_updown(*updown_args, p, edge_bound=edge_bound)


def left_move(e: Env, Ts, ix: int, p: O.Params, lat: O.Lattice, edge_bound=True):
    LY = lat.LY_noskew
    PUs, PLs = [None] * LY, [None] * LY
    for iy in range(LY):
        i = lat.index(ix, iy)
        j = lat.right(i)
        k = lat.bottom(j)
        l = lat.left(k)
        PUs[iy], PLs[iy] = _projectors(
            (e.C1[i], e.C4[l], e.eTt[i], e.eTb[l], e.eTl[l], e.eTl[i], Ts[i], Ts[l]),
            (e.C1[i], e.C2[j], e.C3[k], e.C4[l], e.eTt[i], e.eTt[j], e.eTr[j], e.eTr[k], e.eTb[k], e.eTb[l],
             e.eTl[l], e.eTl[i], Ts[i], Ts[j], Ts[k], Ts[l]), p, edge_bound)
    C1b, C4b, eTlb = list(e.C1), list(e.C4), list(e.eTl)
    for iy in range(LY):
        i = lat.index(ix, iy)
        j = lat.right(i)
        k = lat.bottom(j)
        l = lat.left(k)
        up, dn = (iy + 1) % LY, (iy - 1 + LY) % LY
        e.C1[j], e.C4[k] = next_ctm(C1b[i], C4b[l], e.eTt[i], e.eTb[l], PUs[up], PLs[dn])
        e.eTl[j] = next_et(eTlb[i], Ts[i], PUs[iy], PLs[up])
        e.eTl[k] = next_et(eTlb[l], Ts[l], PUs[dn], PLs[iy])


def right_move(e: Env, Ts, ix: int, p: O.Params, lat: O.Lattice, edge_bound=True):
    LY = lat.LY_noskew
    R = lambda s: Ts[s].transpose(_RR)  # noqa: E731
    PUs, PLs = [None] * LY, [None] * LY
    for iy in range(LY):
        k = lat.index(ix, iy)
        l = lat.left(k)
        i = lat.top(l)
        j = lat.right(i)
        PUs[iy], PLs[iy] = _projectors(
            (e.C3[k], e.C2[j], e.eTb[k], e.eTt[j], e.eTr[j], e.eTr[k], R(k), R(j)),
            (e.C3[k], e.C4[l], e.C1[i], e.C2[j], e.eTb[k], e.eTb[l], e.eTl[l], e.eTl[i], e.eTt[i], e.eTt[j],
             e.eTr[j], e.eTr[k], R(k), R(l), R(i), R(j)), p, edge_bound)
    C2b, C3b, eTrb = list(e.C2), list(e.C3), list(e.eTr)
    for iy in range(LY):
        k = lat.index(ix, iy)
        l = lat.left(k)
        i = lat.top(l)
        j = lat.right(i)
        up, dn = (iy + 1) % LY, (iy - 1 + LY) % LY
        e.C3[l], e.C2[i] = next_ctm(C3b[k], C2b[j], e.eTb[k], e.eTt[j], PUs[dn], PLs[up])
        e.eTr[l] = next_et(eTrb[k], R(k), PUs[iy], PLs[dn])
        e.eTr[i] = next_et(eTrb[j], R(j), PUs[up], PLs[iy])


def top_move(e: Env, Ts, iy: int, p: O.Params, lat: O.Lattice, edge_bound=True):
    LX = lat.LX_noskew
    R = lambda s: Ts[s].transpose(_RT_)  # noqa: E731
    PUs, PLs = [None] * LX, [None] * LX
    for ix in range(LX):
        j = lat.index(ix, iy)
        k = lat.bottom(j)
        l = lat.left(k)
        i = lat.top(l)
        PUs[ix], PLs[ix] = _projectors(
            (e.C2[j], e.C1[i], e.eTr[j], e.eTl[i], e.eTt[i], e.eTt[j], R(j), R(i)),
            (e.C2[j], e.C3[k], e.C4[l], e.C1[i], e.eTr[j], e.eTr[k], e.eTb[k], e.eTb[l], e.eTl[l], e.eTl[i],
             e.eTt[i], e.eTt[j], R(j), R(k), R(l), R(i)), p, edge_bound)
    C1b, C2b, eTtb = list(e.C1), list(e.C2), list(e.eTt)
    for ix in range(LX):
        j = lat.index(ix, iy)
        k = lat.bottom(j)
        l = lat.left(k)
        i = lat.top(l)
        rt, lf = (ix + 1) % LX, (ix - 1 + LX) % LX
        e.C2[k], e.C1[l] = next_ctm(C2b[j], C1b[i], e.eTr[j], e.eTl[i], PUs[rt], PLs[lf])
        e.eTt[k] = next_et(eTtb[j], R(j), PUs[ix], PLs[rt])
        e.eTt[l] = next_et(eTtb[i], R(i), PUs[lf], PLs[ix])


def bottom_move(e: Env, Ts, iy: int, p: O.Params, lat: O.Lattice, edge_bound=True):
    LX = lat.LX_noskew
    R = lambda s: Ts[s].transpose(_RBm)  # noqa: E731
    PUs, PLs = [None] * LX, [None] * LX
    for ix in range(LX):
        l = lat.index(ix, iy)
        i = lat.top(l)
        j = lat.right(i)
        k = lat.bottom(j)
        PUs[ix], PLs[ix] = _projectors(
            (e.C4[l], e.C3[k], e.eTl[l], e.eTr[k], e.eTb[k], e.eTb[l], R(l), R(k)),
            (e.C4[l], e.C1[i], e.C2[j], e.C3[k], e.eTl[l], e.eTl[i], e.eTt[i], e.eTt[j], e.eTr[j], e.eTr[k],
             e.eTb[k], e.eTb[l], R(l), R(i), R(j), R(k)), p, edge_bound)
    C3b, C4b, eTbb = list(e.C3), list(e.C4), list(e.eTb)
    for ix in range(LX):
        l = lat.index(ix, iy)
        i = lat.top(l)
        j = lat.right(i)
        k = lat.bottom(j)
        rt, lf = (ix + 1) % LX, (ix - 1 + LX) % LX
        e.C4[i], e.C3[j] = next_ctm(C4b[l], C3b[k], e.eTl[l], e.eTr[k], PUs[lf], PLs[rt])
        e.eTb[i] = next_et(eTbb[l], R(l), PUs[ix], PLs[lf])
        e.eTb[j] = next_et(eTbb[k], R(k), PUs[rt], PLs[ix])


def sweep(e: Env, Ts, p: O.Params, lat: O.Lattice, edge_bound=True):
    """One iteration of Calc_CTM_Environment_density (ctm_single.cpp:998-1026)."""
    LX, LY = lat.LX_noskew, lat.LY_noskew
    for ix in range(LX):
        left_move(e, Ts, ix, p, lat, edge_bound)
    for ix in range(0, -LX, -1):
        right_move(e, Ts, (ix + 1 + LX) % LX, p, lat, edge_bound)
    for iy in range(0, -LY, -1):
        top_move(e, Ts, (iy + 1 + LY) % LY, p, lat, edge_bound)
    for iy in range(LY):
        bottom_move(e, Ts, iy, p, lat, edge_bound)


def check_convergence(e: Env, old: Env, p: O.Params, lat: O.Lattice) -> Tuple[bool, float]:
    """Check_Convergence_CTM (ctm.cpp:815-969) on the single-layer corners.
    While the corners still grow, the old spectrum is shorter than the new
    one; the missing entries count as zeros."""
    return O.check_convergence(e, old, p, lat)


def calc_ctm_environment(Tn, p: O.Params, lat: O.Lattice, env: Optional[Env] = None, edge_bound=True):
    """Calc_CTM_Environment_density (ctm_single.cpp:737-1050).  Tn are the
    rank-6 density tensors.  Returns (env, iterations, converged, sig_max)."""
    Ts = [single_tensor(t) for t in Tn]
    if env is None:
        env = init_env(Ts, lat)
    old = env.copy()
    count, conv, sig = 0, False, 0.0
    while (not conv) and count < p.Max_CTM_Iteration:
        sweep(env, Ts, p, lat, edge_bound)
        conv, sig = check_convergence(env, old, p, lat)
        count += 1
        old = env.copy()
    return env, count, conv, sig


# ---------------------------------------------------------------------------
# Density contractions (contract_density_ctm/ctm.cpp, correlation.cpp)
# ---------------------------------------------------------------------------


def op_tensor(T: np.ndarray, op: np.ndarray) -> np.ndarray:
    """sum_{p,q} op[p,q] Tn[..., p, q]: the contraction trace(op1, Tn1 ...,
    Axes(0,1), Axes(0,1)) and tensordot(Tn1, op, Axes(4,5), Axes(0,1)) of
    contract_density_ctm/ctm.cpp:103, correlation.cpp:46."""
    return td(T, op, ([4, 5], [0, 1]))


def contract_one_site(C1, C2, C3, C4, eT1, eT2, eT3, eT4, T, op) -> complex:
    """Contract_one_site_density_CTM (contract_density_ctm/ctm.cpp:89-116):
    (op1*(Tn1*((eT1*(C1*eT4))*((C2*eT2)*(C3*(C4*eT3))))))."""
    X = td(td(eT1, td(C1, eT4, ([0], [1])), ([0], [0])),
           td(td(C2, eT2, ([1], [0])), td(C3, td(C4, eT3, ([0], [1])), ([1], [1])), ([1], [0])),
           ([0, 2], [0, 2]))
    return complex(np.sum(td(T, X, ([0, 1, 2, 3], [1, 0, 2, 3])) * op))


def contract_window(C, eTt, eTr, eTb, eTl, A) -> complex:
    """Contract_RxC_density_CTM (contract_density_ctm/ctm_RxC.cpp) for
    single-layer site tensors A[r][c] (rank 4, the operators already
    contracted in by op_tensor), row 0 on top, contracted row by row."""
    nrow, ncol = len(A), len(A[0])
    B = C[0]                                   # (a, b)
    for c in range(ncol):
        B = td(B, eTt[c], ([B.ndim - 1], [0]))  # (..., b', k)
        B = np.moveaxis(B, B.ndim - 2, B.ndim - 1)
    B = td(B, C[1], ([B.ndim - 1], [0]))       # (a, k0..k_{n-1}, r)
    for r in range(nrow):
        B = td(eTl[r], B, ([1], [0]))           # (a', y, k0, ..., r)
        for c in range(ncol):
            pos = 1 + c
            # legs y (pos) and k_c (pos + 1) against A's left and top
            B = np.moveaxis(B, [pos, pos + 1], [B.ndim - 2, B.ndim - 1])
            B = td(B, A[r][c], ([B.ndim - 2, B.ndim - 1], [0, 1]))  # (..., y', z)
            B = np.moveaxis(B, [B.ndim - 1, B.ndim - 2], [pos, pos + 1])  # z at pos, y' next
        n = B.ndim
        B = td(B, eTr[r], ([n - 1, n - 2], [0, 2]))  # (a', z..., r')
    X = td(C[3], B, ([1], [0]))
    for c in range(ncol):
        X = td(eTb[c], X, ([1, 2], [0, 1]))
    return complex(td(X, C[2], ([0, X.ndim - 1], [1, 0])))


def start_correlation(C1, C4, eT1, eT3, eT4, T, op):
    """StartCorrelation_density_CTM (correlation.cpp:33-52); legs
    (eT1_r, eT3_r, Tn1_r)."""
    X = td(op_tensor(T, op), td(eT3, td(C4, eT4, ([1], [0])), ([1], [0])), ([0, 3], [3, 1]))
    return td(td(C1, eT1, ([1], [0])), X, ([0, 2], [3, 0])).transpose(0, 2, 1)


def transfer_correlation(A, eT1, eT3, T):
    """Transfer_density_CTM (correlation.cpp:54-71)."""
    X = td(single_tensor(T), td(A, eT3, ([1], [1])), ([0, 3], [1, 3]))
    return td(eT1, X, ([0, 2], [2, 0])).transpose(0, 2, 1)


def finish_correlation(A, C2, C3, eT1, eT2, eT3, T, op) -> complex:
    """FinishCorrelation_density_CTM (correlation.cpp:73-98):
    (op*(Tn1*((A*eT1)*(eT3*(C2*(C3*eT2))))))."""
    Y = td(eT3, td(C2, td(C3, eT2, ([0], [1])), ([1], [1])), ([0], [1]))
    # X: (A's Tn1_r, eT1's D leg, eT3's D leg, eT2's D leg) against the
    # operator's site tensor (l, t, b, r)
    X = td(td(A, eT1, ([0], [0])), Y, ([0, 2], [0, 2]))
    return complex(td(X, op_tensor(T, op), ([0, 1, 2, 3], [0, 1, 3, 2])))


_VROT = (3, 0, 1, 2, 4, 5)


def correlation_strip(e: Env, Tn, lat: O.Lattice, left: int, vertical: bool, r_max: int, left_op, right_ops):
    """measure_correlation_ctm for an iTPO (correlation_function.cpp:42-220):
    <O_left O_right> / <1> at distances 1..r_max to the right (vertical:
    up)."""
    eye = lambda s: np.eye(Tn[s].shape[4], dtype=Tn[s].dtype)  # noqa: E731
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


def tm_matvec_horizontal(e: Env, lat: O.Lattice, y: int, vec: np.ndarray) -> np.ndarray:
    """matvec_horizontal, rank-3 (iTPO) branch (transfer_matrix.cpp:200-216)."""
    s0 = lat.index(0, y)
    s1 = lat.top(s0)
    c0, c1 = e.eTt[s0].shape[0], e.eTb[s1].shape[1]
    v = vec.reshape(c0, c1)
    for x in range(lat.LX):
        site = lat.index(x, y)
        v = td(e.eTt[site], td(e.eTb[lat.top(site)], v, ([1], [1])), ([0, 2], [2, 1]))
    return v.reshape(-1)


def tm_matvec_vertical(e: Env, lat: O.Lattice, x: int, vec: np.ndarray) -> np.ndarray:
    """matvec_vertical, rank-3 (iTPO) branch (transfer_matrix.cpp:258-280)."""
    s0 = lat.index(x, 0)
    s1 = lat.left(s0)
    c0, c1 = e.eTl[s0].shape[0], e.eTr[s1].shape[1]
    v = vec.reshape(c0, c1)
    x0 = x
    while True:
        for y in range(lat.LY):
            site = lat.index(x, y)
            v = td(e.eTl[site], td(e.eTr[lat.left(site)], v, ([1], [1])), ([0, 2], [2, 1]))
        x = (x + lat.skew + lat.LX) % lat.LX
        if x == x0:
            break
    return v.reshape(-1)


def tm_eigenvalues(e: Env, lat: O.Lattice, direction: int, fixed: int, tp: O.TMParams) -> np.ndarray:
    """TransferMatrix::eigenvalues on the iTPO environment: the initial vector
    and the dense / Arnoldi choice of the double-layer version
    (transfer_matrix.cpp:84-185), with the rank-3 matvecs."""
    return O.tm_eigenvalues(e, lat, direction, fixed, tp,
                            matvec=(tm_matvec_horizontal if direction == 0 else tm_matvec_vertical))


# ---------------------------------------------------------------------------
# Density simple update and the finite-temperature driver
# ---------------------------------------------------------------------------


def kron4(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """mptensor::kron of two rank-4 tensors: out[i*B + j] = a[i] b[j] on
    every leg."""
    s = [x * y for x, y in zip(a.shape, b.shape)]
    return np.einsum("abcd,efgh->aebfcgdh", a, b).reshape(s)


def su_density(Tn, lam, lat: O.Lattice, up, p: O.Params):
    """iTPS::simple_update_density (simple_update.cpp:141-178): a one-site
    operator acts as op on leg 4 and conj(op) on leg 5; a bond operator runs
    Simple_update_bond on the tensors with their physical legs merged
    (d -> d*d) and the operator kron(op, conj(op))."""
    s = up.source_site
    if up.is_onesite():
        T = td(Tn[s], up.op, ([4], [0]))
        Tn[s] = td(T, cj(up.op), ([4], [1]))
        return
    leg = up.source_leg
    tg = lat.neighbor(s, leg)
    A, B = Tn[s], Tn[tg]
    a = A.reshape(A.shape[:4] + (A.shape[4] * A.shape[5],))
    b = B.reshape(B.shape[:4] + (B.shape[4] * B.shape[5],))
    n1, n2, lc = O.simple_update_bond(a, b, lam[s], lam[tg], kron4(up.op, cj(up.op)), leg, p)
    lam[s][leg] = lc
    lam[tg][(leg + 2) % 4] = lc
    d1, d2 = up.op.shape[2], up.op.shape[3]
    Tn[s] = n1.reshape(n1.shape[:4] + (d1, d1))
    Tn[tg] = n2.reshape(n2.shape[:4] + (d2, d2))


def initial_density(lat: O.Lattice, is_real: bool) -> List[np.ndarray]:
    """iTPS::initialize_tensors_density (tensors.cpp:140-208): the identity
    operator on every site, Tn[0,0,0,0,p,p] = 1."""
    out = []
    dt = np.float64 if is_real else np.complex128
    for i in range(lat.N_UNIT):
        d = lat.physical_dims[i]
        v = lat.virtual_dims[i]
        T = np.zeros((v[0], v[1], v[2], v[3], d, d), dtype=dt)
        for k in range(d):
            T[0, 0, 0, 0, k, k] = 1.0
        out.append(T)
    return out


def _window(e: Env, lat: O.Lattice, source, source_col, source_row, nrow, ncol):
    idx = [[lat.other(source, c - source_col, source_row - r) for c in range(ncol)] for r in range(nrow)]
    C = [e.C1[idx[0][0]], e.C2[idx[0][ncol - 1]], e.C3[idx[nrow - 1][ncol - 1]], e.C4[idx[nrow - 1][0]]]
    eTt = [e.eTt[idx[0][c]] for c in range(ncol)]
    eTb = [e.eTb[idx[nrow - 1][c]] for c in range(ncol)]
    eTl = [e.eTl[idx[r][0]] for r in range(nrow)]
    eTr = [e.eTr[idx[r][ncol - 1]] for r in range(nrow)]
    return idx, C, eTt, eTr, eTb, eTl


def measure_onesite(e: Env, Tn, lat: O.Lattice, ops, ngroups: int):
    """measure_onesite, density branch (onesite_obs.cpp:72-86)."""
    N = lat.N_UNIT
    norm = []
    for i in range(N):
        d = Tn[i].shape[4]
        norm.append(contract_one_site(e.C1[i], e.C2[i], e.C3[i], e.C4[i], e.eTt[i], e.eTr[i], e.eTb[i],
                                      e.eTl[i], Tn[i], np.eye(d)))
    vals = [[complex("nan")] * N for _ in range(ngroups)]
    for o in ops:
        i = o.site
        v = contract_one_site(e.C1[i], e.C2[i], e.C3[i], e.C4[i], e.eTt[i], e.eTr[i], e.eTb[i], e.eTl[i],
                              Tn[i], o.op)
        vals[o.group][i] = o.coeff * v / norm[i]
    return vals, norm


def _site_op(onesite, site, group):
    for o in onesite:
        if o.site == site and o.group == group:
            return o.op
    raise KeyError((site, group))


def _window_value(C, eTt, eTr, eTb, eTl, Tn, idx, opw):
    nrow, ncol = len(idx), len(idx[0])
    A = [[op_tensor(Tn[idx[r][c]], opw[r][c]) for c in range(ncol)] for r in range(nrow)]
    return contract_window(C, eTt, eTr, eTb, eTl, A)


def measure_twosite(e: Env, Tn, lat: O.Lattice, ops, onesite, ngroups: int):
    """measure_twosite with is_TPO (twosite_obs.cpp:31-260): the norm and the
    ops_indices products through Contract_density_CTM; an op12 is split by
    its SVD over (0,2 | 1,3) into products (for a nearest-neighbour bond the
    reference contracts op12 directly; the two agree up to rounding)."""
    ret = [dict() for _ in range(ngroups)]
    norms = {}
    for o in ops:
        dx, dy = o.dx, o.dy
        ncol, nrow = abs(dx) + 1, abs(dy) + 1
        if ncol > 4 or nrow > 4:
            continue
        source_col, target_col = (0, ncol - 1) if dx >= 0 else (ncol - 1, 0)
        source_row, target_row = (nrow - 1, 0) if dy >= 0 else (0, nrow - 1)
        idx, C, eTt, eTr, eTb, eTl = _window(e, lat, o.source, source_col, source_row, nrow, ncol)
        ident = [[np.eye(Tn[idx[r][c]].shape[4]) for c in range(ncol)] for r in range(nrow)]
        key = (idx[nrow - 1][0], nrow - 1, ncol - 1)
        if key not in norms:
            norms[key] = _window_value(C, eTt, eTr, eTb, eTl, Tn, idx, ident)
        value = 0.0
        if not o.ops_indices:
            sh = o.op.shape
            U, s, VT = np.linalg.svd(o.op.transpose(0, 2, 1, 3).reshape(sh[0] * sh[2], -1), full_matrices=False)
            U = U.reshape(sh[0], sh[2], -1)
            VT = VT.reshape(-1, sh[1], sh[3])
            for si in range(len(s)):
                opw = [row[:] for row in ident]
                opw[source_row][source_col] = U[:, :, si]
                opw[target_row][target_col] = VT[si]
                value += _window_value(C, eTt, eTr, eTb, eTl, Tn, idx, opw) * s[si]
        else:
            opw = [row[:] for row in ident]
            opw[source_row][source_col] = _site_op(onesite, o.source, o.ops_indices[0])
            tgt = lat.other(o.source, dx, dy)
            opw[target_row][target_col] = _site_op(onesite, tgt, o.ops_indices[1])
            value = _window_value(C, eTt, eTr, eTb, eTl, Tn, idx, opw)
        ret[o.group][(o.source, o.dx, o.dy)] = o.coeff * value / norms[key]
    return ret, norms


def measure_multisite(e: Env, Tn, lat: O.Lattice, ops, onesite, ngroups: int):
    """measure_multisite with is_density (multisite_obs.cpp:31-232)."""
    ret = [dict() for _ in range(ngroups)]
    norms = {}
    for o in ops:
        mindx, maxdx = min(0, *o.dxs), max(0, *o.dxs)
        mindy, maxdy = min(0, *o.dys), max(0, *o.dys)
        ncol, nrow = maxdx - mindx + 1, maxdy - mindy + 1
        if ncol > 4 or nrow > 4:
            continue
        source_col, source_row = -mindx, maxdy
        idx, C, eTt, eTr, eTb, eTl = _window(e, lat, o.source, source_col, source_row, nrow, ncol)
        ident = [[np.eye(Tn[idx[r][c]].shape[4]) for c in range(ncol)] for r in range(nrow)]
        key = (idx[nrow - 1][0], nrow - 1, ncol - 1)
        if key not in norms:
            norms[key] = _window_value(C, eTt, eTr, eTb, eTl, Tn, idx, ident)
        opw = [row[:] for row in ident]
        opw[source_row][source_col] = _site_op(onesite, o.source, o.ops_indices[0])
        for n, (dx, dy) in enumerate(zip(o.dxs, o.dys)):
            opw[source_row - dy][source_col + dx] = _site_op(onesite, lat.other(o.source, dx, dy),
                                                             o.ops_indices[n + 1])
        ret[o.group][(o.source, o.dxs, o.dys)] = o.coeff * _window_value(C, eTt, eTr, eTb, eTl, Tn, idx,
                                                                           opw) / norms[key]
    return ret


def contract_op12(e: Env, Tn, lat: O.Lattice, source: int, dx: int, dy: int, op) -> complex:
    """<op12> of a nearest-neighbour bond with the source/target rule of
    twosite_obs.cpp:186-222, as the sum over the SVD split of op12 of
    one-site-operator windows (equal to Contract_two_sites_*_op12_density_CTM
    up to rounding)."""
    ncol, nrow = abs(dx) + 1, abs(dy) + 1
    source_col, target_col = (0, ncol - 1) if dx >= 0 else (ncol - 1, 0)
    source_row, target_row = (nrow - 1, 0) if dy >= 0 else (0, nrow - 1)
    idx, C, eTt, eTr, eTb, eTl = _window(e, lat, source, source_col, source_row, nrow, ncol)
    sh = op.shape
    U, s, VT = np.linalg.svd(op.transpose(0, 2, 1, 3).reshape(sh[0] * sh[2], -1), full_matrices=False)
    U = U.reshape(sh[0], sh[2], -1)
    VT = VT.reshape(-1, sh[1], sh[3])
    value = 0.0
    for si in range(len(s)):
        opw = [[np.eye(Tn[idx[r][c]].shape[4]) for c in range(ncol)] for r in range(nrow)]
        opw[source_row][source_col] = U[:, :, si]
        opw[target_row][target_col] = VT[si]
        value += _window_value(C, eTt, eTr, eTb, eTl, Tn, idx, opw) * s[si]
    return complex(value)


def window_value(e: Env, Tn, lat: O.Lattice, source: int, nrow: int, ncol: int, source_row: int,
                 source_col: int, ops) -> complex:
    """Contract_density_CTM over the nrow x ncol window whose source sits at
    (source_row, source_col); ops maps (row, col) to a one-site operator."""
    idx, C, eTt, eTr, eTb, eTl = _window(e, lat, source, source_col, source_row, nrow, ncol)
    opw = [[ops.get((r, c), np.eye(Tn[idx[r][c]].shape[4])) for c in range(ncol)] for r in range(nrow)]
    return _window_value(C, eTt, eTr, eTb, eTl, Tn, idx, opw)
