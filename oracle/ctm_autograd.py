"""FP64 host autograd reference of the CTMRG energy gradient -- TEST INFRASTRUCTURE ONLY.

A torch (float64, CPU) restatement of the oracle's CTMRG forward for real
site tensors with full-SVD projectors, corner or up/down:

  * environment initialisation  (src/iTPS/core/ctm.cpp:984-1193,
    ``tenes_oracle.init_env``),
  * the four moves              (ctm.cpp:562-813, ``tenes_oracle.left_move`` ...),
  * the corner projectors       (ctm.cpp:174-318 without the rSVD branch),
  * the up/down projectors      (ctm.cpp:320-491 without the rSVD branch),
  * Calc_Next_CTM / Calc_Next_eT (ctm.cpp:493-552),
  * the N x M window contraction (contract_itps_ctm/ctm.cpp:45-87,
    ``tenes_oracle.contract_window``),

differentiated by torch autograd, except for the truncated SVD of the
projectors, whose backward is the closed form written out in
``svd_backward`` (real case, Lorentzian-broadened 1/(s_j^2 - s_i^2) plus the
(1 - U U^T) / (1 - V V^T) terms of a thin SVD).  The reference has no
gradient code, so this restatement is the checker for the library's adjoint:
its forward is tied to the numpy oracle (equal energies), its backward to
central finite differences.  Only ``tests/`` import it.
"""

from __future__ import annotations

from typing import Dict, List, Sequence, Tuple

import torch

from . import tenes_oracle as O


def td(a, b, x, y):
    return torch.tensordot(a, b, dims=(list(x), list(y)))


def svd_backward(U, s, Vh, gU, gs, gVh, eps):
    """dL/dM of M = U diag(s) Vh (thin, real) from dL/dU, dL/ds, dL/dVh.

    F_ij = (s_j^2 - s_i^2) / ((s_j^2 - s_i^2)^2 + eps (s_i^2 + s_j^2)^2), F_ii = 0
    (broadened relative to the pair's own scale);
    core = diag(gs) + (F o (J - J^T)) S + S (F o (K - K^T)), J = U^T gU, K = V^T gV;
    gM = U core Vh + (1 - U U^T) gU S^-1 Vh + U S^-1 gVh (1 - V V^T)."""
    m, k = U.shape
    n = Vh.shape[1]
    gU = torch.zeros_like(U) if gU is None else gU
    gVh = torch.zeros_like(Vh) if gVh is None else gVh
    gs = torch.zeros_like(s) if gs is None else gs
    J = U.T @ gU
    K = Vh @ gVh.T
    d = s[None, :] ** 2 - s[:, None] ** 2
    q = s[None, :] ** 2 + s[:, None] ** 2
    den = d * d + eps * q * q
    F = torch.where(den > 0, d / torch.where(den > 0, den, torch.ones_like(den)), torch.zeros_like(den))
    F.fill_diagonal_(0.0)
    core = torch.diag(gs) + (F * (J - J.T)) * s[None, :] + s[:, None] * (F * (K - K.T))
    gM = U @ core @ Vh
    sinv = torch.where(s > 0, 1.0 / torch.where(s > 0, s, torch.ones_like(s)), torch.zeros_like(s))
    if m > k:
        gM = gM + ((gU - U @ J) * sinv[None, :]) @ Vh
    if n > k:
        gM = gM + U @ (sinv[:, None] * (gVh - (gVh @ Vh.T) @ Vh))
    return gM


class TruncSVD(torch.autograd.Function):
    """Thin SVD with the broadened backward of ``svd_backward``."""

    @staticmethod
    def forward(ctx, M, eps):
        U, s, Vh = torch.linalg.svd(M, full_matrices=False)
        ctx.save_for_backward(U, s, Vh)
        ctx.eps = eps
        return U, s, Vh

    @staticmethod
    def backward(ctx, gU, gs, gVh):
        U, s, Vh = ctx.saved_tensors
        return svd_backward(U, s, Vh, gU, gs, gVh, ctx.eps), None


def _block_LT(C1, eT1, eT8, T1):
    """ctm.cpp:207-212 (``tenes_oracle._corner_block_LT``)."""
    X = td(td(td(C1, eT1, [1], [0]), eT8, [0], [1]), T1, [2, 5], [1, 0])
    return td(T1, X, [0, 1, 4], [3, 1, 6])


def _block_LB(C4, eT7, eT6, T4):
    """ctm.cpp:222-227 (``tenes_oracle._corner_block_LB``)."""
    X = td(td(td(C4, eT7, [1], [0]), eT6, [0], [1]), T4, [2, 5], [0, 3])
    return td(T4, X, [0, 3, 4], [1, 3, 6])


def projector(C1, C4, eT1, eT6, eT7, eT8, T1, T4, chi, cutoff, eps):
    """Calc_projector_left_block, full-SVD branch (ctm.cpp:174-318)."""
    e78 = eT8.shape[0]
    t41 = T1.shape[3]
    if t41 == 1:
        eye = torch.eye(e78, dtype=C1.dtype)
        return eye.reshape(e78, 1, 1, e78), eye.reshape(e78, 1, 1, e78)
    LT = _block_LT(C1, eT1, eT8, T1)
    LB = _block_LB(C4, eT7, eT6, T4)
    M = td(LT, LB, [1, 3, 5], [0, 2, 4])
    sh = M.shape
    U, s, Vh = TruncSVD.apply(M.reshape(sh[0] * sh[1] * sh[2], -1), eps)
    cut, _ = O._truncation(s.detach().numpy(), min(len(s), chi), cutoff)
    sc = s[:cut] ** -0.5
    Uc = (U[:, :cut] * sc[None, :]).reshape(sh[0], sh[1], sh[2], cut)
    Vc = (Vh[:cut] * sc[:, None]).reshape(cut, sh[3], sh[4], sh[5])
    PU = td(LB, Vc, [1, 3, 5], [1, 2, 3]).permute(1, 0, 2, 3)
    PL = td(LT, Uc, [0, 2, 4], [0, 1, 2]).permute(1, 0, 2, 3)
    return PU, PL


def projector_ud(C1, C2, C3, C4, eT1, eT2, eT3, eT4, eT5, eT6, eT7, eT8, T1, T2, T3, T4, chi, cutoff, eps):
    """Calc_projector_updown_blocks, full-SVD branch (ctm.cpp:320-491;
    ``tenes_oracle.calc_projector_updown_blocks``)."""
    e78 = eT7.shape[1]
    t41 = T4.shape[1]
    if t41 == 1:
        eye = torch.eye(e78, dtype=C1.dtype)
        return eye.reshape(e78, 1, 1, e78), eye.reshape(e78, 1, 1, e78)
    LT = _block_LT(C1, eT1, eT8, T1)
    RT = td(T2, td(td(td(C2, eT3, [1], [0]), eT2, [0], [1]), T2, [2, 5], [2, 1]), [1, 2, 4], [3, 1, 6])
    RB = td(T3, td(td(td(C3, eT5, [1], [0]), eT4, [0], [1]), T3, [2, 5], [3, 2]), [2, 3, 4], [3, 1, 6])
    LB = _block_LB(C4, eT7, eT6, T4)
    R1 = td(RT, LT, [0, 3, 4], [0, 2, 4])
    R2 = td(RB, LB, [0, 2, 4], [1, 3, 5])
    M = td(R1, R2, [3, 4, 5], [3, 4, 5])
    sh = M.shape
    U, s, Vh = TruncSVD.apply(M.reshape(sh[0] * sh[1] * sh[2], -1), eps)
    cut, _ = O._truncation(s.detach().numpy(), min(len(s), chi), cutoff)
    sc = s[:cut] ** -0.5
    Uc = (U[:, :cut] * sc[None, :]).reshape(sh[0], sh[1], sh[2], cut)
    Vc = (Vh[:cut] * sc[:, None]).reshape(cut, sh[3], sh[4], sh[5])
    PU = td(R2, Vc, [0, 1, 2], [1, 2, 3]).permute(1, 0, 2, 3)
    PL = td(R1, Uc, [0, 1, 2], [0, 1, 2]).permute(1, 0, 2, 3)
    return PU, PL


def _normalized(t):
    return t / t.abs().max()


def next_ctm(C1, C4, eT1, eT6, PU, PL):
    """ctm.cpp:493-518."""
    C1o = td(PU, td(C1, eT1, [1], [0]), [0, 1, 2], [0, 2, 3])
    C4o = td(td(eT6, C4, [1], [0]), PL, [3, 1, 2], [0, 1, 2])
    return _normalized(C1o), _normalized(C4o)


def next_et(eT8, T1, PU, PL):
    """ctm.cpp:520-552."""
    X = td(T1, td(eT8, PL, [1], [0]), [0, 1], [2, 4])
    X = td(T1, X, [0, 1, 4], [4, 5, 2])
    return _normalized(td(X, PU, [1, 3, 4], [1, 2, 0]).permute(3, 2, 0, 1))


def _fit(X, chi):
    """extend / slice the first two legs to chi (ctm.cpp:998-1012)."""
    out = torch.zeros((chi, chi) + tuple(X.shape[2:]), dtype=X.dtype)
    m1, m2 = min(X.shape[0], chi), min(X.shape[1], chi)
    out[:m1, :m2] = X[:m1, :m2]
    return out


def init_env(Tn, chi, lat: O.Lattice):
    """ctm.cpp:984-1193 (``tenes_oracle.init_env``), real tensors."""
    N = lat.N_UNIT
    env = {k: [None] * N for k in ("C1", "C2", "C3", "C4", "eTt", "eTr", "eTb", "eTl")}
    for i in range(N):
        T = Tn[lat.top(lat.left(i))]
        X = td(T, T, [0, 1, 4], [0, 1, 4]).permute(1, 3, 0, 2)
        env["C1"][i] = _fit(X.reshape(X.shape[0] * X.shape[1], -1), chi)
        T = Tn[lat.top(lat.right(i))]
        X = td(T, T, [1, 2, 4], [1, 2, 4]).permute(0, 2, 1, 3)
        env["C2"][i] = _fit(X.reshape(X.shape[0] * X.shape[1], -1), chi)
        T = Tn[lat.bottom(lat.right(i))]
        X = td(T, T, [2, 3, 4], [2, 3, 4]).permute(1, 3, 0, 2)
        env["C3"][i] = _fit(X.reshape(X.shape[0] * X.shape[1], -1), chi)
        T = Tn[lat.bottom(lat.left(i))]
        X = td(T, T, [0, 3, 4], [0, 3, 4]).permute(1, 3, 0, 2)
        env["C4"][i] = _fit(X.reshape(X.shape[0] * X.shape[1], -1), chi)
        for name, nb, legs, perm in (("eTt", lat.top(i), [1, 4], (0, 3, 1, 4, 2, 5)),
                                     ("eTr", lat.right(i), [2, 4], (1, 4, 2, 5, 0, 3)),
                                     ("eTb", lat.bottom(i), [3, 4], (2, 5, 0, 3, 1, 4)),
                                     ("eTl", lat.left(i), [0, 4], (2, 5, 0, 3, 1, 4))):
            T = Tn[nb]
            X = td(T, T, legs, legs).permute(*perm)
            s = X.shape
            env[name][i] = _fit(X.reshape(s[0] * s[1], s[2] * s[3], s[4], s[5]), chi)
    return env


_RIGHT, _TOP, _BOTTOM = (2, 3, 0, 1, 4), (1, 2, 3, 0, 4), (3, 0, 1, 2, 4)


def sweep(env, Tn, chi, lat: O.Lattice, cutoff=1e-12, eps=1e-12, corner=True):
    """One CTMRG iteration (ctm.cpp:1205-1228) with the index rules of the
    oracle's left/right/top/bottom moves (ctm.cpp:562-813); corner=False
    takes the up/down projectors."""
    C1, C2, C3, C4 = env["C1"], env["C2"], env["C3"], env["C4"]
    eTt, eTr, eTb, eTl = env["eTt"], env["eTr"], env["eTb"], env["eTl"]
    LX, LY = lat.LX_noskew, lat.LY_noskew
    R = lambda t, p: t.permute(*p)  # noqa: E731

    def P(*a, ud):
        """the corner projector of `a`, or with corner=False the up/down one of `ud`"""
        if corner:
            return projector(*a, chi, cutoff, eps)
        return projector_ud(*ud, chi, cutoff, eps)

    for ix in range(LX):  # Left_move
        PU, PL = [None] * LY, [None] * LY
        for iy in range(LY):
            i = lat.index(ix, iy); j = lat.right(i); k = lat.bottom(j); l = lat.left(k)  # noqa: E702
            PU[iy], PL[iy] = P(C1[i], C4[l], eTt[i], eTb[l], eTl[l], eTl[i], Tn[i], Tn[l],
                               ud=(C1[i], C2[j], C3[k], C4[l], eTt[i], eTt[j], eTr[j], eTr[k], eTb[k], eTb[l],
                                   eTl[l], eTl[i], Tn[i], Tn[j], Tn[k], Tn[l]))
        C1b, C4b, eTlb = list(C1), list(C4), list(eTl)
        for iy in range(LY):
            i = lat.index(ix, iy); j = lat.right(i); k = lat.bottom(j); l = lat.left(k)  # noqa: E702
            up, dn = (iy + 1) % LY, (iy - 1 + LY) % LY
            C1[j], C4[k] = next_ctm(C1b[i], C4b[l], eTt[i], eTb[l], PU[up], PL[dn])
            eTl[j] = next_et(eTlb[i], Tn[i], PU[iy], PL[up])
            eTl[k] = next_et(eTlb[l], Tn[l], PU[dn], PL[iy])
    for ix0 in range(0, -LX, -1):  # Right_move
        ix = (ix0 + 1 + LX) % LX
        PU, PL = [None] * LY, [None] * LY
        for iy in range(LY):
            k = lat.index(ix, iy); l = lat.left(k); i = lat.top(l); j = lat.right(i)  # noqa: E702
            PU[iy], PL[iy] = P(C3[k], C2[j], eTb[k], eTt[j], eTr[j], eTr[k], R(Tn[k], _RIGHT), R(Tn[j], _RIGHT),
                               ud=(C3[k], C4[l], C1[i], C2[j], eTb[k], eTb[l], eTl[l], eTl[i], eTt[i], eTt[j],
                                   eTr[j], eTr[k], R(Tn[k], _RIGHT), R(Tn[l], _RIGHT), R(Tn[i], _RIGHT),
                                   R(Tn[j], _RIGHT)))
        C2b, C3b, eTrb = list(C2), list(C3), list(eTr)
        for iy in range(LY):
            k = lat.index(ix, iy); l = lat.left(k); i = lat.top(l); j = lat.right(i)  # noqa: E702
            up, dn = (iy + 1) % LY, (iy - 1 + LY) % LY
            C3[l], C2[i] = next_ctm(C3b[k], C2b[j], eTb[k], eTt[j], PU[dn], PL[up])
            eTr[l] = next_et(eTrb[k], R(Tn[k], _RIGHT), PU[iy], PL[dn])
            eTr[i] = next_et(eTrb[j], R(Tn[j], _RIGHT), PU[up], PL[iy])
    for iy0 in range(0, -LY, -1):  # Top_move
        iy = (iy0 + 1 + LY) % LY
        PU, PL = [None] * LX, [None] * LX
        for ix in range(LX):
            j = lat.index(ix, iy); k = lat.bottom(j); l = lat.left(k); i = lat.top(l)  # noqa: E702
            PU[ix], PL[ix] = P(C2[j], C1[i], eTr[j], eTl[i], eTt[i], eTt[j], R(Tn[j], _TOP), R(Tn[i], _TOP),
                               ud=(C2[j], C3[k], C4[l], C1[i], eTr[j], eTr[k], eTb[k], eTb[l], eTl[l], eTl[i],
                                   eTt[i], eTt[j], R(Tn[j], _TOP), R(Tn[k], _TOP), R(Tn[l], _TOP), R(Tn[i], _TOP)))
        C1b, C2b, eTtb = list(C1), list(C2), list(eTt)
        for ix in range(LX):
            j = lat.index(ix, iy); k = lat.bottom(j); l = lat.left(k); i = lat.top(l)  # noqa: E702
            rt, lf = (ix + 1) % LX, (ix - 1 + LX) % LX
            C2[k], C1[l] = next_ctm(C2b[j], C1b[i], eTr[j], eTl[i], PU[rt], PL[lf])
            eTt[k] = next_et(eTtb[j], R(Tn[j], _TOP), PU[ix], PL[rt])
            eTt[l] = next_et(eTtb[i], R(Tn[i], _TOP), PU[lf], PL[ix])
    for iy in range(LY):  # Bottom_move
        PU, PL = [None] * LX, [None] * LX
        for ix in range(LX):
            l = lat.index(ix, iy); i = lat.top(l); j = lat.right(i); k = lat.bottom(j)  # noqa: E702
            PU[ix], PL[ix] = P(C4[l], C3[k], eTl[l], eTr[k], eTb[k], eTb[l], R(Tn[l], _BOTTOM), R(Tn[k], _BOTTOM),
                               ud=(C4[l], C1[i], C2[j], C3[k], eTl[l], eTl[i], eTt[i], eTt[j], eTr[j], eTr[k],
                                   eTb[k], eTb[l], R(Tn[l], _BOTTOM), R(Tn[i], _BOTTOM), R(Tn[j], _BOTTOM),
                                   R(Tn[k], _BOTTOM)))
        C3b, C4b, eTbb = list(C3), list(C4), list(eTb)
        for ix in range(LX):
            l = lat.index(ix, iy); i = lat.top(l); j = lat.right(i); k = lat.bottom(j)  # noqa: E702
            rt, lf = (ix + 1) % LX, (ix - 1 + LX) % LX
            C4[i], C3[j] = next_ctm(C4b[l], C3b[k], eTl[l], eTr[k], PU[lf], PL[rt])
            eTb[i] = next_et(eTbb[l], R(Tn[l], _BOTTOM), PU[ix], PL[lf])
            eTb[j] = next_et(eTbb[k], R(Tn[k], _BOTTOM), PU[rt], PL[ix])


def contract_window(C, eTt, eTr, eTb, eTl, T, op):
    """``tenes_oracle.contract_window`` (contract_itps_ctm/ctm.cpp:45-87) in torch."""
    nrow, ncol = len(T), len(T[0])
    B = C[0]
    for c in range(ncol):
        B = td(B, eTt[c], [B.dim() - 1], [0])
        B = torch.movedim(B, B.dim() - 3, B.dim() - 1)
    B = td(B, C[1], [B.dim() - 1], [0])
    for r in range(nrow):
        B = td(eTl[r], B, [1], [0])
        for c in range(ncol):
            t = T[r][c]
            pos = 1 + 2 * c
            n = B.dim()
            B = torch.movedim(B, [pos, pos + 1, pos + 2, pos + 3], [n - 4, n - 3, n - 2, n - 1])
            B = td(B, t, [n - 4, n - 2], [0, 1])
            if op[r][c] is not None:
                B = td(B, op[r][c], [B.dim() - 1], [0])
            n = B.dim()
            B = td(B, t, [n - 5, n - 4, n - 1], [0, 1, 4])
            n = B.dim()
            B = B.permute(*(list(range(n - 4)) + [n - 3, n - 1, n - 4, n - 2]))
            B = torch.movedim(B, [n - 4, n - 3, n - 2, n - 1], [pos, pos + 1, pos + 2, pos + 3])
        n = B.dim()
        B = td(B, eTr[r], [n - 1, n - 3, n - 2], [0, 2, 3])
    X = td(C[3], B, [1], [0])
    for c in range(ncol):
        X = td(eTb[c], X, [1, 2, 3], [0, 1, 2])
    return td(X, C[2], [0, X.dim() - 1], [1, 0])


def window_value(env, Tn, lat: O.Lattice, term) -> torch.Tensor:
    """<prod ops> on the window of ``term`` (keys as tenes_b200.grad.WindowTerm:
    source, nrow, ncol, source_row, source_col, ops {(row, col): op})."""
    nrow, ncol = term["nrow"], term["ncol"]
    sr, sc = term["source_row"], term["source_col"]
    idx = [[lat.other(term["source"], c - sc, sr - r) for c in range(ncol)] for r in range(nrow)]
    C = [env["C1"][idx[0][0]], env["C2"][idx[0][ncol - 1]], env["C3"][idx[nrow - 1][ncol - 1]],
         env["C4"][idx[nrow - 1][0]]]
    T = [[Tn[idx[r][c]] for c in range(ncol)] for r in range(nrow)]
    ops = [[None] * ncol for _ in range(nrow)]
    for (r, c), o in term["ops"].items():
        ops[r][c] = torch.as_tensor(o, dtype=torch.float64)
    return contract_window(C, [env["eTt"][idx[0][c]] for c in range(ncol)],
                           [env["eTr"][idx[r][ncol - 1]] for r in range(nrow)],
                           [env["eTb"][idx[nrow - 1][c]] for c in range(ncol)],
                           [env["eTl"][idx[r][0]] for r in range(nrow)], T, ops)


def energy(Tn: Sequence[torch.Tensor], terms, chi: int, iterations: int, lat: O.Lattice,
           cutoff: float = 1e-12, eps: float = 1e-12, corner: bool = True) -> torch.Tensor:
    """E = sum_t coeff_t <ops_t> / <1>_t after ``iterations`` CTMRG sweeps from
    the initial environment of Tn (the norm of a window shared by every term on
    the same window, as twosite_obs.cpp:160-181 caches it)."""
    env = init_env(Tn, chi, lat)
    for _ in range(iterations):
        sweep(env, Tn, chi, lat, cutoff, eps, corner)
    norms: Dict[Tuple[int, ...], torch.Tensor] = {}
    E = torch.zeros((), dtype=torch.float64)
    for t in terms:
        key = (t["source"], t["nrow"], t["ncol"], t["source_row"], t["source_col"])
        if key not in norms:
            norms[key] = window_value(env, Tn, lat, dict(t, ops={}))
        E = E + t["coeff"] * window_value(env, Tn, lat, t) / norms[key]
    return E


def energy_and_grad(Tn_np: Sequence, terms, chi: int, iterations: int, lat: O.Lattice,
                    cutoff: float = 1e-12, eps: float = 1e-12, corner: bool = True) -> Tuple[float, List]:
    Tn = [torch.tensor(t, dtype=torch.float64, requires_grad=True) for t in Tn_np]
    E = energy(Tn, terms, chi, iterations, lat, cutoff, eps, corner)
    g = torch.autograd.grad(E, Tn)
    return float(E.detach()), [x.numpy() for x in g]
