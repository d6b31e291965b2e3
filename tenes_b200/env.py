"""Python mirror of TeNeS's iTPS environment interface on top of the C ABI.

``Environment`` owns one libtenes_gpu context (device-resident site tensors,
simple-update weights and CTM environment) and exposes the reference's
operations under the reference's names:

=====================================  =============================================
reference (src/iTPS/...)               here
=====================================  =============================================
core::Calc_CTM_Environment (ctm.cpp)   ``Environment.calc_ctm_environment``
core::Left/Right/Top/Bottom_move        ``Environment.move``
core::Check_Convergence_CTM             ``Environment.check_convergence``
core::Simple_update_bond / tensordot    ``Environment.simple_update``
Contract_one_site_iTPS_CTM              ``Environment.contract_one_site``
Contract_two_sites_*_op12_iTPS_CTM      ``Environment.contract_bond_op12``
=====================================  =============================================
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from ._lib import check, dptr


@dataclass
class CTMParams:
    """[parameter.ctm] / [parameter.simple_update] knobs (PEPS_Parameters)."""
    chi: int = 2
    inverse_projector_cut: float = 1e-12
    ctm_convergence_epsilon: float = 1e-6
    max_ctm_iteration: int = 100
    projector_corner: bool = True
    use_rsvd: bool = False
    rsvd_oversampling_factor: float = 2.0
    rsvd_oversample_abs: int = -1
    rsvd_power_iters: int = 2
    rsvd_seed: int = 0
    inverse_lambda_cut: float = 1e-12
    mixed: bool = False
    cuda_graph: bool = True
    svd_solver: int = 0
    # an iTPO (finite-temperature density operator): site tensors
    # (D,D,D,D,d,d), single-layer CTMRG, density contractions
    density: bool = False

    def to_c(self) -> _lib.Params:
        p = _lib.Params()
        for f in self.__dataclass_fields__:
            setattr(p, f, int(getattr(self, f)) if isinstance(getattr(self, f), bool) else getattr(self, f))
        return p


ENV_NAMES = ("C1", "C2", "C3", "C4", "eTt", "eTr", "eTb", "eTl")


class Environment:
    """Device-resident iTPS + CTM environment of one unit cell."""

    def __init__(self, LX: int, LY: int, physical_dims: Sequence[int],
                 virtual_dims: Sequence[Sequence[int]], params: CTMParams, is_complex: bool,
                 skew: int = 0, device: int = 0):
        self.lib = _lib.load()
        self.LX, self.LY, self.skew = LX, LY, skew
        self.N = LX * LY
        self.pdim = [int(x) for x in physical_dims]
        self.vdim = [[int(x) for x in v] for v in virtual_dims]
        self.params = params
        self.is_complex = bool(is_complex)
        self.dtype = np.complex128 if is_complex else np.float64
        pd = (C.c_int * self.N)(*self.pdim)
        vd = (C.c_int * (4 * self.N))(*[x for v in self.vdim for x in v])
        self._keep = (pd, vd)
        desc = _lib.LatticeDesc(LX, LY, skew, pd, vd)
        self._cp = params.to_c()
        h = C.c_void_p()
        check(self.lib.tg_ctx_create(C.byref(desc), C.byref(self._cp), int(is_complex), device, C.byref(h)))
        self.ctx = h

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.tg_ctx_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ------------------------------------------------------------- tensors
    def site_shape(self, i: int) -> Tuple[int, ...]:
        v = self.vdim[i]
        if self.params.density:
            return (v[0], v[1], v[2], v[3], self.pdim[i], self.pdim[i])
        return (v[0], v[1], v[2], v[3], self.pdim[i])

    def env_shape(self, which: int, i: int) -> Tuple[int, ...]:
        chi = self.params.chi
        if which < 4:
            return (chi, chi)
        leg = {4: 1, 5: 2, 6: 3, 7: 0}[which]
        d = self.vdim[i][leg]
        return (chi, chi, d, 1 if self.params.density else d)

    def set_site_tensor(self, i: int, T: np.ndarray) -> None:
        a = _lib.as_host(T, self.is_complex)
        if a.shape != self.site_shape(i):
            raise ValueError(f"site {i}: shape {a.shape} != {self.site_shape(i)}")
        check(self.lib.tg_set_site_tensor(self.ctx, i, dptr(a.view(np.float64))))

    def get_site_tensor(self, i: int, out: Optional[np.ndarray] = None) -> np.ndarray:
        """Site tensor i; into `out` (C-contiguous, of the tensor's shape and dtype) when given."""
        a = self._out(out, self.site_shape(i))
        check(self.lib.tg_get_site_tensor(self.ctx, i, dptr(a.view(np.float64))))
        return a

    def _out(self, out: Optional[np.ndarray], shape) -> np.ndarray:
        if out is None:
            return np.empty(shape, dtype=self.dtype)
        if out.shape != tuple(shape) or out.dtype != self.dtype or not out.flags["C_CONTIGUOUS"]:
            raise ValueError(f"out: needs a C-contiguous {self.dtype} array of shape {tuple(shape)}")
        return out

    def set_lambda(self, i: int, leg: int, lam: np.ndarray) -> None:
        a = np.ascontiguousarray(lam, dtype=np.float64)
        if a.shape != (self.vdim[i][leg],):
            raise ValueError("lambda length mismatch")
        check(self.lib.tg_set_lambda(self.ctx, i, leg, dptr(a)))

    def get_lambda(self, i: int, leg: int) -> np.ndarray:
        a = np.empty(self.vdim[i][leg], dtype=np.float64)
        check(self.lib.tg_get_lambda(self.ctx, i, leg, dptr(a)))
        return a

    def set_env(self, which: int, i: int, T: np.ndarray) -> None:
        a = _lib.as_host(T, self.is_complex)
        if a.shape != self.env_shape(which, i):
            raise ValueError(f"{ENV_NAMES[which]}[{i}]: shape {a.shape} != {self.env_shape(which, i)}")
        check(self.lib.tg_set_env(self.ctx, which, i, dptr(a.view(np.float64))))

    def get_env(self, which: int, i: int, out: Optional[np.ndarray] = None) -> np.ndarray:
        """Environment tensor `which` (ENV_NAMES) of site i; into `out` when given."""
        a = self._out(out, self.env_shape(which, i))
        check(self.lib.tg_get_env(self.ctx, which, i, dptr(a.view(np.float64))))
        return a

    # --------------------------------------------------------------- CTMRG
    def init_env(self) -> None:
        check(self.lib.tg_ctm_init(self.ctx))

    def move(self, direction: int, line: int) -> None:
        """0 = Left_move, 1 = Right_move, 2 = Top_move, 3 = Bottom_move."""
        check(self.lib.tg_ctm_move(self.ctx, direction, line))

    def sweep(self) -> None:
        check(self.lib.tg_ctm_sweep(self.ctx))

    def check_convergence(self) -> Tuple[bool, float]:
        conv = C.c_int()
        sig = C.c_double()
        check(self.lib.tg_ctm_check_convergence(self.ctx, C.byref(conv), C.byref(sig)))
        return bool(conv.value), sig.value

    def calc_ctm_environment(self, initialize: bool = True) -> Tuple[int, bool, float]:
        it = C.c_int()
        conv = C.c_int()
        sig = C.c_double()
        check(self.lib.tg_ctm_run(self.ctx, int(initialize), C.byref(it), C.byref(conv), C.byref(sig)))
        return it.value, bool(conv.value), sig.value

    def projector_svd_stats(self) -> dict:
        """Counters of the exact truncated SVD of the full-SVD projectors."""
        out = (C.c_int64 * 4)()
        check(self.lib.tg_projector_svd_stats(self.ctx, out))
        return {"solves": out[0], "iterations": out[1], "checks": out[2], "dense": out[3]}

    def corner_spectrum(self, which: int, i: int) -> np.ndarray:
        a = np.empty(self.params.chi, dtype=np.float64)
        check(self.lib.tg_corner_spectrum(self.ctx, which, i, dptr(a)))
        return a

    # --------------------------------------------------------- observables
    def contract_one_site(self, i: int, op: np.ndarray) -> complex:
        o = np.ascontiguousarray(op, dtype=self.dtype)
        out = np.zeros(2)
        check(self.lib.tg_measure_onesite(self.ctx, i, dptr(o.view(np.float64)), dptr(out)))
        return complex(out[0], out[1])

    def contract_bond_op12(self, source: int, dx: int, dy: int, op12: np.ndarray) -> complex:
        o = np.ascontiguousarray(op12, dtype=self.dtype)
        out = np.zeros(2)
        check(self.lib.tg_measure_bond_op12(self.ctx, source, dx, dy, dptr(o.view(np.float64)), dptr(out)))
        return complex(out[0], out[1])

    def contract_bond_rdm(self, source: int, dx: int, dy: int) -> np.ndarray:
        """Unnormalised two-site reduced density matrix of a nearest-neighbour
        bond, legs (source, target, source', target'): <op12> = sum(op12 * rdm),
        norm = einsum('abab', rdm)."""
        from .input import LatticeSpec
        target = LatticeSpec(self.LX, self.LY, self.skew, self.pdim, self.vdim, [], []).other(source, dx, dy)
        shape = (self.pdim[source], self.pdim[target]) * 2
        out = np.zeros(int(np.prod(shape)) * (2 if self.is_complex else 1))
        check(self.lib.tg_measure_bond_rdm(self.ctx, source, dx, dy, dptr(out)))
        if self.params.density:
            # R[(p_s,q_s),(p_t,q_t)] -> rdm[p_s,p_t,q_s,q_t], the same contraction rule
            ds, dt = self.pdim[source], self.pdim[target]
            return out.view(self.dtype).reshape(ds, ds, dt, dt).transpose(0, 2, 1, 3).copy()
        return out.view(self.dtype).reshape(shape)

    def correlation_strip(self, left: int, vertical: bool, r_max: int, left_op: np.ndarray, right_ops) -> np.ndarray:
        """<O_left O_right>/<1> at distances 1..r_max to the right (vertical:
        up) of `left` through the strip contraction (tg_measure_correlation).
        right_ops(site) -> list of that site's right operators (the same
        count for every site).  Returns a complex (r_max, nright) array."""
        lists = [list(right_ops(i)) for i in range(self.N)]
        nright = len(lists[0])
        if any(len(l) != nright for l in lists) or nright == 0:
            raise ValueError("correlation_strip: the same positive number of right operators on every site")
        for i, l in enumerate(lists):
            for o in l:
                if np.shape(o) != (self.pdim[i],) * 2:
                    raise ValueError(f"correlation_strip: operator of shape {np.shape(o)} on site {i} "
                                     f"(physical dimension {self.pdim[i]})")
        if np.shape(left_op) != (self.pdim[left],) * 2:
            raise ValueError(f"correlation_strip: left operator of shape {np.shape(left_op)} on site {left}")
        flat = np.concatenate([np.ascontiguousarray(o, dtype=self.dtype).reshape(-1) for l in lists for o in l])
        flat = np.ascontiguousarray(flat, dtype=self.dtype)
        lop = np.ascontiguousarray(left_op, dtype=self.dtype)
        out = np.zeros(2 * r_max * nright)
        check(self.lib.tg_measure_correlation(self.ctx, left, int(bool(vertical)), r_max, dptr(lop.view(np.float64)),
                                              nright, dptr(flat.view(np.float64)), dptr(out)))
        return (out[0::2] + 1j * out[1::2]).reshape(r_max, nright)

    def contract_window(self, source: int, nrow: int, ncol: int, source_row: int, source_col: int,
                        ops: Optional[dict] = None) -> complex:
        """Contract_RxC_iTPS_CTM: <prod ops> on an nrow x ncol window (unnormalised).
        ops maps (row, col) -> d x d operator; identity elsewhere."""
        ops = ops or {}
        keys = sorted(ops)
        rows = (C.c_int * max(len(keys), 1))(*[k[0] for k in keys])
        cols = (C.c_int * max(len(keys), 1))(*[k[1] for k in keys])
        flat = np.concatenate([np.ascontiguousarray(ops[k], dtype=self.dtype).reshape(-1) for k in keys]) \
            if keys else np.zeros(1, dtype=self.dtype)
        flat = np.ascontiguousarray(flat, dtype=self.dtype)
        out = np.zeros(2)
        check(self.lib.tg_measure_window(self.ctx, source, nrow, ncol, source_row, source_col, len(keys), rows,
                                         cols, dptr(flat.view(np.float64)), dptr(out)))
        return complex(out[0], out[1])

    def energy_grad(self, terms, iterations: int, checkpoint_every: int = 5, svd_broadening: float = 1e-12,
                    grad: bool = True):
        """E = sum_t coeff_t <ops_t>/<1>_t after ``iterations`` CTMRG sweeps from
        the initial environment of the current site tensors, and dE/dTn per
        site (None when ``grad`` is False).  ``terms`` are window terms as
        built by ``tenes_b200.grad`` (dicts with source, nrow, ncol,
        source_row, source_col, ops {(row, col): d x d real operator}, coeff).
        The context's environment is left unchanged."""
        if self.is_complex:
            raise ValueError("energy_grad: real site tensors only")
        arr = (_lib.WindowTerm * len(terms))()
        keep = []
        for q, t in enumerate(terms):
            keys = sorted(t["ops"])
            rows = (C.c_int * max(len(keys), 1))(*[k[0] for k in keys])
            cols = (C.c_int * max(len(keys), 1))(*[k[1] for k in keys])
            flat = np.ascontiguousarray(
                np.concatenate([np.asarray(t["ops"][k], dtype=np.float64).reshape(-1) for k in keys])
                if keys else np.zeros(1), dtype=np.float64)
            keep.append((rows, cols, flat))
            arr[q] = _lib.WindowTerm(t["source"], t["nrow"], t["ncol"], t["source_row"], t["source_col"],
                                     len(keys), rows, cols, dptr(flat), float(t["coeff"]))
        E = np.zeros(1)
        sizes = [int(np.prod(self.site_shape(i))) for i in range(self.N)]
        g = np.zeros(sum(sizes)) if grad else None
        check(self.lib.tg_energy_grad(self.ctx, len(terms), arr, int(iterations), int(checkpoint_every),
                                      float(svd_broadening), dptr(E), dptr(g) if grad else None))
        if not grad:
            return float(E[0]), None
        out, off = [], 0
        for i, n in enumerate(sizes):
            out.append(g[off:off + n].reshape(self.site_shape(i)))
            off += n
        return float(E[0]), out

    def tm_eigenvalues(self, direction: int, fixed: int, num_eigvals: int = 4, maxdim_dense: int = 200,
                       arnoldi_maxdim: int = 50, arnoldi_restartdim: int = 20, arnoldi_maxiter: int = 1,
                       arnoldi_rtol: float = 1e-10) -> np.ndarray:
        """TransferMatrix::eigenvalues (transfer_matrix.cpp:84-142)."""
        out = np.zeros(2 * num_eigvals)
        nev = C.c_int()
        check(self.lib.tg_tm_eigenvalues(self.ctx, direction, fixed, num_eigvals, maxdim_dense, arnoldi_maxdim,
                                         arnoldi_restartdim, arnoldi_maxiter, arnoldi_rtol, dptr(out),
                                         C.byref(nev)))
        v = out[: 2 * nev.value]
        return v[0::2] + 1j * v[1::2]

    # ------------------------------------------------------- simple update
    def _check_op(self, source: int, source_leg: int, op: np.ndarray) -> None:
        """A one-site op must be (d, d) and a bond op (d_s, d_t, d_s, d_t) for the
        sites' physical dimensions (the library keeps them fixed)."""
        d = self.pdim[source]
        if source_leg < 0:
            want = (d, d)
        else:
            from .input import LatticeSpec
            t = LatticeSpec(self.LX, self.LY, self.skew, self.pdim, self.vdim, [], []).other(
                source, *((-1, 0), (0, 1), (1, 0), (0, -1))[source_leg])
            want = (d, self.pdim[t], d, self.pdim[t])
        if tuple(np.shape(op)) != want:
            raise ValueError(f"operator of shape {tuple(np.shape(op))} on site {source} leg {source_leg}: "
                             f"{want} expected")

    def simple_update(self, source: int, source_leg: int, op: np.ndarray) -> None:
        """iTPS::simple_update(EvolutionOperator) (src/iTPS/simple_update.cpp:25-46)."""
        self._check_op(source, source_leg, op)
        o = _lib.as_host(op, self.is_complex)
        if source_leg < 0:
            check(self.lib.tg_su_onesite(self.ctx, source, dptr(o.view(np.float64))))
        else:
            check(self.lib.tg_su_bond(self.ctx, source, source_leg, dptr(o.view(np.float64))))

    def simple_update_many(self, steps) -> None:
        """A sequence of (source, source_leg, op) simple-update steps in its
        order, in one library call (tg_su_bonds): runs of bond steps on
        disjoint site pairs go to the device together."""
        steps = list(steps)
        if not steps:
            return
        hosts = []
        for source, leg, op in steps:
            self._check_op(source, leg, op)
            hosts.append(np.ascontiguousarray(_lib.as_host(op, self.is_complex)))
        n = len(steps)
        src = (C.c_int * n)(*[int(x[0]) for x in steps])
        legs = (C.c_int * n)(*[int(x[1]) if x[1] >= 0 else -1 for x in steps])
        ptrs = (C.c_void_p * n)(*[h.ctypes.data for h in hosts])
        check(self.lib.tg_su_bonds(self.ctx, n, src, legs, ptrs))

    def full_update_bond(self, source: int, source_leg: int, op: np.ndarray, inverse_env_cut: float = 1e-12,
                         inverse_precision: float = 1e-12, convergence_epsilon: float = 1e-6,
                         max_iteration: int = 100, gauge_fix: bool = True) -> Tuple[int, bool]:
        """core::Full_update_bond of the bond (source, source_leg) in the
        current environment (src/iTPS/full_update.cpp:30-120); the site
        tensors are replaced, the environment is not moved.  Returns the
        least-squares iterations and whether they converged."""
        self._check_op(source, source_leg, op)
        o = _lib.as_host(op, self.is_complex)
        fp = _lib.FuParams(float(inverse_env_cut), float(inverse_precision), float(convergence_epsilon),
                           int(max_iteration), int(bool(gauge_fix)))
        it, conv = C.c_int(), C.c_int()
        check(self.lib.tg_fu_bond(self.ctx, source, source_leg, dptr(o.view(np.float64)), C.byref(fp),
                                  C.byref(it), C.byref(conv)))
        return it.value, bool(conv.value)

    def fix_local_gauge(self, maxiter: int = 100, eps: float = 1e-2) -> Tuple[int, float]:
        """iTPS::fix_local_gauge (src/iTPS/simple_update.cpp:49-101): sweeps of
        core::fix_local_gauge over the bonds until every boundary tensor is
        within eps of the identity (at most maxiter sweeps).  Returns the
        sweeps done and the last score."""
        n, sc = C.c_int(), C.c_double()
        check(self.lib.tg_su_fix_gauge(self.ctx, int(maxiter), float(eps), C.byref(n), C.byref(sc)))
        return n.value, sc.value

    def init_tensors(self, seed: int, initial_dirs: Sequence[Sequence[float]],
                     noises: Sequence[float]) -> None:
        """iTPS::initialize_tensors (src/iTPS/tensors.cpp:38-137)."""
        flat = np.ascontiguousarray([x for d in initial_dirs for x in d] or [0.0], dtype=np.float64)
        lens = (C.c_int * self.N)(*[len(d) for d in initial_dirs])
        nz = np.ascontiguousarray(noises, dtype=np.float64)
        check(self.lib.tg_init_tensors(self.ctx, int(seed), dptr(flat), lens, dptr(nz)))

    def sync(self) -> None:
        check(self.lib.tg_sync(self.ctx))


    def stream_handle(self) -> int:
        """cudaStream_t of the context (for events / ordering)."""
        h = C.c_void_p()
        check(self.lib.tg_ctx_stream(self.ctx, C.byref(h)))
        return int(h.value or 0)


def kernel_launch_count() -> int:
    return int(_lib.load().tg_kernel_launch_count())


PROFILE_KINDS = ("gemm_dmma", "permute", "normalize", "jacobi_spectrum", "factorisations", "other",
                 "gemm_tcgen05")


def profile_enable(on: bool) -> None:
    check(_lib.load().tg_profile_enable(int(on)))


def profile_reset() -> None:
    check(_lib.load().tg_profile_reset())


def profile_query(kind: int):
    """(launches, device_ms, flops, bytes) summed since the last reset."""
    n = C.c_uint64()
    ms, fl, by = C.c_double(), C.c_double(), C.c_double()
    check(_lib.load().tg_profile_query(kind, C.byref(n), C.byref(ms), C.byref(fl), C.byref(by)))
    return int(n.value), ms.value, fl.value, by.value
