"""Drop-in driver for TeNeS's iTPS ground-state, time-evolution and
finite-temperature runs on the GPU path: ``python -m tenes_b200 input.toml``
in place of ``tenes input.toml``.

Mirrors the reference's driver (src/iTPS/main.cpp:141-199, iTPS.cpp,
optimize.cpp:24-37, simple_update.cpp:103-138, time_evolution.cpp:21-90,
finite_temperature.cpp:22-86, measure.cpp:30-144) and its output files
(onesite_obs.cpp:125-200, twosite_obs.cpp:288-340, multisite_obs.cpp:250-300,
correlation_length.cpp:57-125, density.cpp:30-228, measure.cpp:81-107).  All
tensor work goes through the C ABI of libtenes_gpu; this layer holds the
reference's host-side bookkeeping only.  In finite-temperature mode the
context holds the density operator (tg_params.density) and the same
measurement calls are the density contractions.

Out of scope (raises InputError): the mean-field environment.
Long-range correlation functions ([correlation]) are measured through window
contractions up to r = 3 and through the strip contraction beyond.
Tensor checkpoints (tensor_save / tensor_load) are written and read by
saveload.py.
"""

from __future__ import annotations

import math
import os
import sys
import time as _time
from typing import Dict, List, Optional, Tuple

import numpy as np

from .env import CTMParams, Environment
from .input import Input, InputError, load_input
from .saveload import load_tensors, save_tensors


def _fmt(x: float) -> str:
    return f"{x:.17e}"


def _g(x) -> str:
    """A number as C++'s default ostream formatting prints it (%g, 6 digits)."""
    return format(x, "g") if isinstance(x, float) else str(int(x))


def write_parameters(path: str, p, lattice) -> None:
    """parameters.dat: PEPS_Parameters::save (PEPS_Parameters.cpp:220-300),
    SquareLattice::save appended (SquareLattice.cpp:139-150) and the start
    time (iTPS.cpp:145-150), line for line.  The reference's switch over the
    calculation mode falls through from "time evolution" into "finite
    temperature" (no break, PEPS_Parameters.cpp:282-287), so a time-evolution
    run lists both; the file keeps that."""
    import datetime
    b = lambda v: "true" if v else "false"  # noqa: E731
    lst = lambda v: "[" + ", ".join(_g(x) for x in v) + "]"  # noqa: E731
    mode = {"ground_state": "ground state\n", "time_evolution": "time evolution\nfinite temperature\n",
            "finite_temperature": "finite temperature\n"}[p.calcmode]
    lines = [
        f"simple_num_step = {lst(p.num_simple_step)}",
        f"simple_tau = {lst([float(x) for x in p.tau_simple_step])}",
        f"simple_inverse_lambda_cutoff = {_g(float(p.Inverse_lambda_cut))}",
        f"simple_gauge_fix = {int(bool(p.Simple_Gauge_Fix))}",
        f"simple_gauge_maxiter = {int(p.Simple_Gauge_maxiter)}",
        f"simple_gauge_convergence_epsilon = {_g(float(p.Simple_Gauge_Convergence_Epsilon))}",
        "",
        f"full_num_step = {lst(p.num_full_step)}",
        f"full_inverse_projector_cutoff = {_g(float(p.Inverse_projector_cut))}",
        f"full_inverse_precision = {_g(float(p.Full_Inverse_precision))}",
        f"full_convergence_epsilon = {_g(float(p.Full_Convergence_Epsilon))}",
        f"full_iteration_max = {int(p.Full_max_iteration)}",
        f"full_gauge_fix = {b(p.Full_Gauge_Fix)}",
        f"full_fastfullupdate = {b(p.Full_Use_FastFullUpdate)}",
        "",
        f"ctm_dimension = {int(p.CHI)}",
        f"ctm_inverse_projector_cutoff = {_g(float(p.Inverse_Env_cut))}",
        f"ctm_convergence_epsilon = {_g(float(p.CTM_Convergence_Epsilon))}",
        f"ctm_iteration_max = {int(p.Max_CTM_Iteration)}",
        f"ctm_projector_corner = {b(p.CTM_Projector_corner)}",
        f"use_rsvd = {b(p.Use_RSVD)}",
        f"rsvd_oversampling_factor = {_g(float(p.RSVD_Oversampling_factor))}",
        f"meanfield_env = {b(p.MeanField_Env)}",
        "",
    ]
    text = "\n".join(lines) + "\n" + "mode = " + mode + "simple\n"
    text += (f"Lcor = {int(getattr(p, 'Lcor', 0))}\nseed = {int(p.seed)}\nis_real = {int(bool(p.is_real))}\n"
             f"iszero_tol = {_g(float(p.iszero_tol))}\nmeasure = {int(bool(p.to_measure))}\n"
             f"tensor_load_dir = {p.tensor_load_dir}\ntensor_save_dir = {p.tensor_save_dir}\n"
             f"outdir = {p.outdir}\n")
    text += f"\nLsub = [ {lattice.LX} , {lattice.LY} ]\nskew = {lattice.skew}\n"
    text += f"\nstart_datetime =  {datetime.datetime.now().astimezone().isoformat(timespec='seconds')}\n"
    with open(path, "w") as f:
        f.write(text)


class ITPS:
    """iTPS<tensor> (src/iTPS/iTPS.hpp:97-234) over a device-resident Environment."""

    def __init__(self, inp: Input, device: int = 0, mixed: bool = False, print_level: int = 1):
        p = inp.params
        self.density = p.calcmode == "finite_temperature"  # an iTPO (iTPS.cpp:176-180)
        if p.MeanField_Env:
            raise InputError("the mean-field environment is not part of this library")
        self.inp = inp
        self.p = p
        self.print_level = print_level
        ls = inp.lattice
        self.LX, self.LY, self.N = ls.LX, ls.LY, ls.LX * ls.LY
        self.is_real = inp.is_real
        cp = CTMParams(chi=p.CHI, inverse_projector_cut=p.Inverse_projector_cut,
                       ctm_convergence_epsilon=p.CTM_Convergence_Epsilon,
                       max_ctm_iteration=p.Max_CTM_Iteration, projector_corner=p.CTM_Projector_corner,
                       use_rsvd=p.Use_RSVD, rsvd_oversampling_factor=p.RSVD_Oversampling_factor,
                       inverse_lambda_cut=p.Inverse_lambda_cut, mixed=mixed, density=self.density)
        self.env = Environment(ls.LX, ls.LY, ls.physical_dims, ls.virtual_dims, cp, not self.is_real,
                               skew=ls.skew, device=device)
        for up in list(inp.simple_updates) + list(inp.full_updates):
            d = ls.physical_dims[up.source_site]
            if up.is_onesite():
                ok = up.op.shape == (d, d)
            else:
                dt = ls.physical_dims[ls.other(up.source_site, *((-1, 0), (0, 1), (1, 0), (0, -1))[up.source_leg])]
                ok = up.op.shape == (d, dt, d, dt)
            if not ok:
                raise InputError(f"evolution operator on site {up.source_site} has dimensions {list(up.op.shape)}: "
                                 "operators that change a site's physical dimension along the sequence (as "
                                 "next-nearest-neighbour gates do) are not supported by this library")
        if p.tensor_save_dir:  # iTPS.cpp:161-173
            os.makedirs(p.tensor_save_dir, exist_ok=True)
        if p.tensor_load_dir:  # initialize_tensors: the checkpoint replaces the random start (tensors.cpp:130-135)
            load_tensors(self.env, p.tensor_load_dir, p.CHI, print_level)
        else:
            self.env.init_tensors(p.seed, ls.initial_dirs, ls.noises)
        self.outdir = p.outdir
        os.makedirs(self.outdir, exist_ok=True)
        write_parameters(os.path.join(self.outdir, "parameters.dat"), p, ls)
        n1 = self._names(inp.onesite, "onesite", False)
        n2 = self._names(inp.twosite, "twosite", False)
        nm = self._names(inp.multisite, "multisite", True)
        width = max([len("Energy")] + [len(s) for s in n1 + n2 + nm])
        self.names1, self.names2, self.namesm = ([s.ljust(width) for s in n] for n in (n1, n2, nm))
        self._first: Dict[str, bool] = {}
        self.t_su = self.t_fu = self.t_env = self.t_obs = 0.0
        self.t0 = _time.perf_counter()
        dmax = max(max(v) for v in ls.virtual_dims)  # iTPS.cpp:120-136
        if self.density:
            if p.CHI < dmax and print_level > 0:
                print("WARNING: CTM may be too small (chi < D) for iTPO (finite_temperature mode)", file=sys.stderr)
        elif p.CHI < dmax ** 2 and print_level > 0:
            print("WARNING: CTM may be too small (chi < D*D) for iTPS", file=sys.stderr)

    @staticmethod
    def _names(ops, kind: str, default_name: bool) -> List[str]:
        """Group names (iTPS.cpp:310-415): one name per group, an error when a
        group carries two; only multisite groups get a generated default name."""
        if not ops:
            return []
        names = [""] * (max(o.group for o in ops) + 1)
        for o in ops:
            name = o.name or f"{kind}[{o.group}]"
            if not names[o.group]:
                names[o.group] = name if default_name else o.name
            elif names[o.group] != (name if default_name else o.name):
                raise InputError(f"{kind} operator group {o.group} has two different names: "
                                 f"{name} and {names[o.group]}")
        return names

    def _op(self, a: np.ndarray) -> np.ndarray:
        return a.real.copy() if self.is_real else a

    # ----------------------------------------------------- simple update
    def simple_update_step(self, group: int = 0) -> None:
        """One Trotter step: every op of `group` in input order (simple_update.cpp:113-119),
        then the local gauge fixing when simple_update.gauge_fix is set."""
        self.env.simple_update_many((up.source_site, up.source_leg, self._op(up.op))
                                    for up in self.inp.simple_updates if up.group == group)
        if self.p.Simple_Gauge_Fix:  # simple_update.cpp:121-124, time_evolution.cpp:59-62
            self.env.fix_local_gauge(self.p.Simple_Gauge_maxiter, self.p.Simple_Gauge_Convergence_Epsilon)

    def optimize(self) -> None:
        """optimize() (optimize.cpp:24-37): simple update, then full update."""
        t = _time.perf_counter()
        nsteps = self.p.num_simple_step[0]
        for _ in range(nsteps):
            self.simple_update_step(0)
        self.env.sync()
        self.t_su += _time.perf_counter() - t
        if self.p.num_full_step[0] > 0:
            self.full_update()

    # ------------------------------------------------------ full update
    # moves after a bond update of the fast full update: (direction, site
    # whose column / row) for the source and the target (full_update.cpp:122-148);
    # directions 0 left, 1 right, 2 top, 3 bottom
    _FAST_MOVES = {0: ((1, "s", "x"), (0, "t", "x")), 1: ((3, "s", "y"), (2, "t", "y")),
                   2: ((0, "s", "x"), (1, "t", "x")), 3: ((2, "s", "y"), (3, "t", "y"))}

    def full_update_op(self, up) -> None:
        """iTPS::full_update(EvolutionOperator) (full_update.cpp:30-149)."""
        if up.is_onesite():
            self.env.simple_update(up.source_site, -1, self._op(up.op))
            return
        p = self.p
        it, conv = self.env.full_update_bond(up.source_site, up.source_leg, self._op(up.op),
                                             p.Inverse_Env_cut, p.Full_Inverse_precision,
                                             p.Full_Convergence_Epsilon, p.Full_max_iteration, p.Full_Gauge_Fix)
        if not conv and self.print_level > 0:
            print(f"warning: Full update iteration was not conveged! count= {it}")
        if not p.Full_Use_FastFullUpdate:
            self.update_ctm()
            return
        target = self._other(up.source_site, *((-1, 0), (0, 1), (1, 0), (0, -1))[up.source_leg])
        for direction, who, axis in self._FAST_MOVES[up.source_leg]:
            site = up.source_site if who == "s" else target
            line = site % self.LX if axis == "x" else site // self.LX
            self.env.move(direction, line)

    def full_update(self) -> None:
        """iTPS::full_update() (full_update.cpp:151-186): a full CTMRG, then
        every full-update operator of group 0 in input order, num_step times."""
        t = _time.perf_counter()
        self.update_ctm()
        for _ in range(self.p.num_full_step[0]):
            for up in self.inp.full_updates:
                if up.group == 0:
                    self.full_update_op(up)
        self.env.sync()
        self.t_fu += _time.perf_counter() - t

    # ------------------------------------------------------ environment
    def update_ctm(self) -> Tuple[int, bool, float]:
        t = _time.perf_counter()
        it, conv, sig = self.env.calc_ctm_environment(True)
        self.t_env += _time.perf_counter() - t
        if not conv and self.print_level > 0:
            print(f"Warning: CTM did not converge! count, sig_max = {it} {sig}")
        return it, conv, sig

    # ------------------------------------------------------- observables
    def measure_onesite(self):
        """measure_onesite (onesite_obs.cpp:35-123)."""
        ng = len(self.names1)
        vals = [[complex("nan")] * self.N for _ in range(ng)]
        norm = []
        for i in range(self.N):
            d = self.inp.lattice.physical_dims[i]
            norm.append(self.env.contract_one_site(i, np.eye(d)))
        for o in self.inp.onesite:
            v = self.env.contract_one_site(o.source_site, self._op(o.op))
            vals[o.group][o.source_site] = o.coeff * v / norm[o.source_site]
        self._norm_warnings(norm, strict=False)
        return vals, norm

    def _norm_warnings(self, norms, strict: bool) -> None:
        if not norms or self.print_level <= 0:
            return
        re_min = min(n.real for n in norms)
        im_max = max(abs(n.imag) for n in norms)
        if (re_min <= 0.0) if not strict else (re_min < 0.0):
            print(f"WARNING: Norm is negative [min(real(NORM)) = {re_min}].", file=sys.stderr)
        if im_max > 1e-6:
            print(f"WARNING: Norm is not real [max(abs(imag(NORM))) = {im_max} > 1e-6].", file=sys.stderr)

    def _site_op(self, site: int, group: int) -> np.ndarray:
        for o in self.inp.onesite:
            if o.source_site == site and o.group == group:
                return self._op(o.op)
        raise InputError(f"no onesite operator of group {group} on site {site}")

    def measure_twosite(self):
        """measure_twosite (twosite_obs.cpp:31-260)."""
        lat_other = self._other
        ng = len(self.names2)
        ret: List[Dict] = [dict() for _ in range(ng)]
        norms: Dict = {}
        for o in self.inp.twosite:
            dx, dy = o.dx[0], o.dy[0]
            ncol, nrow = abs(dx) + 1, abs(dy) + 1
            if ncol > 4 or nrow > 4:
                print("Warning: now version of TeNeS does not support too long-ranged operator", file=sys.stderr)
                continue
            sc, tc = (0, ncol - 1) if dx >= 0 else (ncol - 1, 0)
            sr, tr = (nrow - 1, 0) if dy >= 0 else (0, nrow - 1)
            origin = lat_other(o.source_site, -sc, sr)  # site at (row 0, col 0)
            bottom_left = lat_other(origin, 0, -(nrow - 1))
            key = (bottom_left, nrow - 1, ncol - 1)
            if key not in norms:
                norms[key] = self.env.contract_window(o.source_site, nrow, ncol, sr, sc)
            norm = norms[key]
            if not o.ops_indices:
                op = self._op(o.op)
                if nrow * ncol == 2:
                    value = self.env.contract_bond_op12(o.source_site, dx, dy, op)
                else:
                    sh = op.shape
                    U, s, VT = np.linalg.svd(op.transpose(0, 2, 1, 3).reshape(sh[0] * sh[2], -1),
                                             full_matrices=False)
                    U = U.reshape(sh[0], sh[2], -1)
                    VT = VT.reshape(-1, sh[1], sh[3])
                    value = 0.0
                    for si in range(len(s)):
                        value += s[si] * self.env.contract_window(
                            o.source_site, nrow, ncol, sr, sc,
                            {(sr, sc): self._op(U[:, :, si]), (tr, tc): self._op(VT[si])})
            else:
                tgt = lat_other(o.source_site, dx, dy)
                value = self.env.contract_window(o.source_site, nrow, ncol, sr, sc,
                                                 {(sr, sc): self._site_op(o.source_site, o.ops_indices[0]),
                                                  (tr, tc): self._site_op(tgt, o.ops_indices[1])})
            ret[o.group][(o.source_site, dx, dy)] = o.coeff * value / norm
        self._norm_warnings(list(norms.values()), strict=True)
        return ret, norms

    def measure_multisite(self):
        """measure_multisite (multisite_obs.cpp:31-232)."""
        ng = len(self.namesm)
        ret: List[Dict] = [dict() for _ in range(ng)]
        norms: Dict = {}
        for o in self.inp.multisite:
            mindx, maxdx = min(0, *o.dx), max(0, *o.dx)
            mindy, maxdy = min(0, *o.dy), max(0, *o.dy)
            ncol, nrow = maxdx - mindx + 1, maxdy - mindy + 1
            if ncol > 4 or nrow > 4:
                print("Warning: now version of TeNeS does not support too long-ranged operator", file=sys.stderr)
                continue
            if not o.ops_indices:
                raise InputError("Empty op.ops_indices is not supported for multisites observable")
            sc, sr = -mindx, maxdy
            origin = self._other(o.source_site, -sc, sr)
            key = (self._other(origin, 0, -(nrow - 1)), nrow - 1, ncol - 1)
            if key not in norms:
                norms[key] = self.env.contract_window(o.source_site, nrow, ncol, sr, sc)
            ops = {(sr, sc): self._site_op(o.source_site, o.ops_indices[0])}
            for n, (dx, dy) in enumerate(zip(o.dx, o.dy)):
                tgt = self._other(o.source_site, dx, dy)
                ops[(sr - dy, sc + dx)] = self._site_op(tgt, o.ops_indices[n + 1])
            value = self.env.contract_window(o.source_site, nrow, ncol, sr, sc, ops)
            ret[o.group][(o.source_site, tuple(o.dx), tuple(o.dy))] = o.coeff * value / norms[key]
        self._norm_warnings(list(norms.values()), strict=True)
        return ret

    # ------------------------------------------- long-range correlations
    # Up to r = 3 (and about 2 GB of boundary tensor) a correlation is read
    # from the window that spans the two sites; longer strips go through the
    # strip contraction (tg_measure_correlation), linear in r.
    MAX_WINDOW_R = 3
    MAX_WINDOW_BYTES = 2 << 30

    def _site_op_or_none(self, site: int, group: int):
        for o in self.inp.onesite:
            if o.source_site == site and o.group == group:
                return self._op(o.op)
        return None

    def measure_correlation(self):
        """measure_correlation_ctm (correlation_function.cpp:42-220): for every
        site and every (left, right) one-site operator group pair of
        [correlation], <O_left O_right> / <1> at horizontal and vertical
        distances 1 .. r_max, in the reference's order.  Short strips are read
        from windows (the window over the two sites with the operators at its
        ends, over the same window without operators); longer ones from the
        StartCorrelation / Transfer / FinishCorrelation strip."""
        cp = self.inp.corparam
        nl = len(self.names1)
        dmax = max(max(v) for v in self.inp.lattice.virtual_dims)
        use_windows = (cp.r_max <= self.MAX_WINDOW_R
                       and 16 * self.p.CHI ** 2 * dmax ** (2 * (cp.r_max + 1)) <= self.MAX_WINDOW_BYTES)
        r_ops: List[List[int]] = [[] for _ in range(nl)]
        for lop, rop in cp.operators:
            if not (0 <= lop < nl and 0 <= rop < nl):
                raise InputError(f"correlation operator index out of range: ({lop}, {rop})")
            r_ops[lop].append(rop)
        out = []
        for left in range(self.N):
            for lop in range(nl):
                if not r_ops[lop]:
                    continue
                Ol = self._site_op_or_none(left, lop)
                if Ol is None:
                    continue
                for horizontal in (True, False):
                    if use_windows:
                        vals = self._correlation_windows(left, horizontal, cp.r_max, Ol, r_ops[lop])
                    else:
                        def ops_of(site, rops=r_ops[lop]):
                            d = self.inp.lattice.physical_dims[site]
                            return [self._site_op_or_none(site, q) if self._site_op_or_none(site, q) is not None
                                    else np.zeros((d, d)) for q in rops]
                        strip = self.env.correlation_strip(left, not horizontal, cp.r_max, Ol, ops_of)
                        vals = []
                        site = left
                        for r in range(cp.r_max):
                            site = self._other(site, 1, 0) if horizontal else self._other(site, 0, 1)
                            vals.append([strip[r][k] if self._site_op_or_none(site, q) is not None else None
                                         for k, q in enumerate(r_ops[lop])])
                    for r in range(1, cp.r_max + 1):
                        for k, rop in enumerate(r_ops[lop]):
                            v = vals[r - 1][k]
                            if v is not None:
                                out.append((left, r if horizontal else 0, 0 if horizontal else r, lop, rop, v))
        return out

    def _correlation_windows(self, left, horizontal, r_max, Ol, rops):
        vals = []
        site = left
        for r in range(1, r_max + 1):
            site = self._other(site, 1, 0) if horizontal else self._other(site, 0, 1)
            if horizontal:
                geo, pl, pr = (1, r + 1, 0, 0), (0, 0), (0, r)
            else:
                geo, pl, pr = (r + 1, 1, r, 0), (r, 0), (0, 0)
            norm = self.env.contract_window(left, *geo)
            row = []
            for rop in rops:
                Or = self._site_op_or_none(site, rop)
                row.append(None if Or is None else self.env.contract_window(left, *geo, {pl: Ol, pr: Or}) / norm)
            vals.append(row)
        return vals

    def save_correlation(self, cors, time, prefix):
        """save_correlation (correlation_function.cpp:349-395)."""
        cols = self._time_header(time) + ["left_op", "left_site", "right_op", "right_dx", "right_dy", "real",
                                          "imag"]
        hdr = self._cols(cols)
        hdr.append("# The names of operators are the following: ")
        hdr += [f"# {i}: {n}" for i, n in enumerate(self.names1)]
        with self._open(prefix + "correlation.dat", hdr) as f:
            for left, dx, dy, lop, rop, v in cors:
                t = f"{_fmt(time)} " if time is not None else ""
                f.write(f"{t}{lop} {left} {rop} {dx} {dy} {_fmt(v.real)} {_fmt(v.imag)} \n")

    def measure_transfer_matrix(self):
        """measure_transfer_matrix_eigenvalues (correlation_length.cpp:24-55)."""
        tp = self.inp.tm_params
        res = []
        for d in (0, 1):
            W = self.LY if d == 0 else self.LX
            for fixed in range(W):
                ev = self.env.tm_eigenvalues(d, fixed, tp.num_eigvals, tp.maxdim_dense_eigensolver,
                                             tp.arnoldi_maxdim, tp.arnoldi_restartdim, tp.arnoldi_maxiter,
                                             tp.arnoldi_rtol)
                res.append((d, fixed, ev))
        return res

    def _other(self, i: int, dx: int, dy: int) -> int:
        return self.inp.lattice.other(i, dx, dy)

    # ----------------------------------------------------------- writers
    def _open(self, name: str, header: List[str]):
        path = os.path.join(self.outdir, name)
        if not self._first.get(name):
            self._first[name] = True
            with open(path, "w") as f:
                f.write("\n".join(header) + "\n\n")
        return open(path, "a")

    def _time_header(self, time: Optional[float]) -> List[str]:
        if time is None:
            return []
        return ["time" if self.p.calcmode == "time_evolution" else "inverse temperature"]

    @staticmethod
    def _cols(cols: List[str]) -> List[str]:
        out = ["# The meaning of each column is the following: "]
        out += [f"# ${i + 1}: {c}" for i, c in enumerate(cols)]
        return out

    def save_onesite(self, vals, norm, time, prefix):
        hdr = self._cols(self._time_header(time) + ["op_group", "site_index", "real", "imag"])
        hdr += ["# The names of op_group are the following: "]
        hdr += [f"# {g}: {n}" for g, n in enumerate(self.names1)] + ["# -1: norm"]
        with self._open(prefix + "onesite_obs.dat", hdr) as f:
            tp = "" if time is None else _fmt(time) + " "
            for g, row in enumerate(vals):
                for i, v in enumerate(row):
                    if not math.isnan(v.real):
                        f.write(f"{tp}{g} {i} {_fmt(v.real)} {_fmt(v.imag)}\n")
            for i, v in enumerate(norm):
                f.write(f"{tp}-1 {i} {_fmt(v.real)} {_fmt(v.imag)}\n")

    def save_twosite(self, ret, norms, time, prefix):
        hdr = self._cols(self._time_header(time) + ["op_group", "source_site", "dx", "dy", "real", "imag"])
        hdr += ["# The names of op_group are the following: "]
        hdr += [f"# {g}: {n}" for g, n in enumerate(self.names2)] + ["# -1: norm"]
        with self._open(prefix + "twosite_obs.dat", hdr) as f:
            tp = "" if time is None else _fmt(time) + " "
            for g, d in enumerate(ret):
                for (s, dx, dy), v in sorted(d.items()):
                    f.write(f"{tp}{g} {s} {dx} {dy} {_fmt(v.real)} {_fmt(v.imag)}\n")
            # norm keys are Bond{bottom-left site, nrow - 1, ncol - 1} (twosite_obs.cpp:166)
            for (s, a, b), v in sorted(norms.items()):
                f.write(f"{tp}-1 {s} {a} {b} {_fmt(v.real)} {_fmt(v.imag)}\n")

    def save_multisite(self, ret, time, prefix):
        nsites_of = {}
        for o in self.inp.multisite:
            if nsites_of.setdefault(o.group, len(o.dx) + 1) != len(o.dx) + 1:
                raise InputError(f"multisite operator group {o.group} mixes different numbers of sites")
        for nsites in sorted(set(nsites_of.values())):
            cols = self._time_header(time) + ["op_group", "source_site"]
            for k in range(1, nsites):
                cols += [f"dx[{k}]", f"dy[{k}]"]
            hdr = self._cols(cols + ["real", "imag"]) + ["# The names of op_group are the following: "]
            hdr += [f"# {g}: {n}" for g, n in enumerate(self.namesm) if nsites_of.get(g) == nsites]
            with self._open(prefix + f"multisite_obs_{nsites}.dat", hdr) as f:
                tp = "" if time is None else _fmt(time) + " "
                for g, d in enumerate(ret):
                    for (s, dxs, dys), v in sorted(d.items()):
                        if len(dxs) + 1 != nsites:
                            continue
                        pos = " ".join(f"{a} {b}" for a, b in zip(dxs, dys))
                        f.write(f"{tp}{g} {s} {pos} {_fmt(v.real)} {_fmt(v.imag)}\n")

    def save_correlation_length(self, res, time, prefix):
        hdr = ["# The meaning of each column is the following: "]
        idx = 1
        if time is not None:
            hdr.append(f"# ${idx}: time")
            idx += 1
        hdr += [f"# ${idx}: direction 0: +x, 1: +y", f"# ${idx + 1}: y (dir=0) or x (dir=1) coorinates",
                f"# ${idx + 2}: correlation length xi = 1/e_1 ",
                f"# ${idx + 3}-: eigenvalues e_i = -log|t_i/t_0|",
                "#      where i > 0 and t_i is i-th largest eigenvalue of T"]
        with self._open(prefix + "correlation_length.dat", hdr) as f:
            tp = "" if time is None else _fmt(time) + " "
            lat = self.inp.lattice
            for (d, x, ev) in res:
                if len(ev) == 1:
                    f.write(f"{tp}{d} {x} {_fmt(0.0)}\n")
                    continue
                L = lat.LX if d == 0 else self._ly_noskew()
                with np.errstate(divide="ignore", invalid="ignore"):
                    e = np.abs(np.asarray(ev)) / abs(ev[0])
                    xi = -L / np.log(e[1])
                    es = -np.log(e[1:]) / L
                f.write(f"{tp}{d} {x} {_fmt(xi)} " + " ".join(_fmt(v) for v in es) + "\n")

    def _ly_noskew(self) -> int:
        ls = self.inp.lattice
        if ls.skew == 0:
            return ls.LY
        s = ls.skew % ls.LX
        return ls.LY * ((ls.LX * s // math.gcd(ls.LX, s)) // s)

    def save_density(self, vals, two, multi, time, prefix):
        nsites = sum(1 for d in self.inp.lattice.physical_dims if d > 1)
        # sites without an operator of a group hold NaN and make that group's sum NaN, as in
        # the reference; energy compares the width-padded names (density.cpp:61-72)
        loc = [sum((row[i] for i in range(self.N) if self.inp.lattice.physical_dims[i] > 1), 0j)
               for row in vals]
        tw = [sum(d.values(), 0j) for d in two]
        mu = [sum(d.values(), 0j) for d in multi]
        energy = sum(loc[g].real for g, n in enumerate(self.names1) if n == "site_hamiltonian")
        energy += sum(tw[g].real for g, n in enumerate(self.names2) if n == "bond_hamiltonian")
        inv = 1.0 / nsites
        energy *= inv
        cnt1 = {o.group for o in self.inp.onesite}
        cnt2 = {o.group for o in self.inp.twosite}
        cntm = {o.group for o in self.inp.multisite}
        path = os.path.join(self.outdir, prefix + "density.dat")

        def num(v: float) -> str:
            return (" " if v >= 0.0 else "") + _fmt(v)

        if time is not None:
            if not self._first.get("density"):
                self._first["density"] = True
                hdr = self._cols(self._time_header(time) + ["observable ID", "real", "imag"])
                hdr += ["# The meaning of observable IDs are the following: ", "# 0: Energy"]
                k = 1
                for names, cnt in ((self.names1, cnt1), (self.names2, cnt2), (self.namesm, cntm)):
                    for g, n in enumerate(names):
                        if g in cnt:
                            hdr.append(f"# {k}: {n}")
                            k += 1
                with open(path, "w") as f:
                    f.write("\n".join(hdr) + "\n\n")
            with open(path, "a") as f:
                f.write(f"{_fmt(time)} 0 {num(energy)}  {_fmt(0.0)}\n")
                k = 1
                for arr, names, cnt in ((loc, self.names1, cnt1), (tw, self.names2, cnt2),
                                        (mu, self.namesm, cntm)):
                    for g, n in enumerate(names):
                        if g in cnt:
                            v = complex(arr[g]) * inv
                            f.write(f"{_fmt(time)} {k} {num(v.real)} {num(v.imag)}\n")
                            k += 1
        else:
            width = len((self.names1 + self.names2 + self.namesm + ["Energy"])[0])
            with open(path, "w") as f:
                f.write(f"{'Energy'.ljust(width)} = {num(energy)}  {_fmt(0.0)}\n")
                for arr, names, cnt in ((loc, self.names1, cnt1), (tw, self.names2, cnt2),
                                        (mu, self.namesm, cntm)):
                    for g, n in enumerate(names):
                        if g in cnt:
                            v = complex(arr[g]) * inv
                            f.write(f"{n} = {num(v.real)} {num(v.imag)}\n")
        return energy

    # ----------------------------------------------------------- measure
    def measure(self, time: Optional[float] = None, prefix: str = ""):
        """iTPS::measure (measure.cpp:30-79)."""
        self.update_ctm()
        t = _time.perf_counter()
        vals, norm = self.measure_onesite()
        self.save_onesite(vals, norm, time, prefix)
        two, norms = self.measure_twosite()
        self.save_twosite(two, norms, time, prefix)
        multi = self.measure_multisite()
        if self.inp.multisite:
            self.save_multisite(multi, time, prefix)
        if self.inp.corparam.r_max > 0:
            self.save_correlation(self.measure_correlation(), time, prefix)
        # measure_density skips the transfer matrix at beta = 0, where it is
        # degenerate (measure.cpp:133-139)
        if self.inp.tm_params.to_calculate and not (self.density and time == 0.0):
            self.save_correlation_length(self.measure_transfer_matrix(), time, prefix)
        energy = self.save_density(vals, two, multi, time, prefix)
        self.t_obs += _time.perf_counter() - t
        return energy

    def time_evolution(self) -> None:
        """iTPS::time_evolution (time_evolution.cpp:21-90) with the group
        checks of iTPS.cpp:217-306: simple-update steps when
        simple_update.num_step > 0, else full-update steps (each followed by
        the fast full update's moves or a full CTMRG, as in the ground state)."""
        p = self.p
        if p.num_simple_step[0] > 0 and p.num_full_step[0] > 0:
            raise InputError("While mode is not ground state calculation,\n"
                             "       simple update and full update are both required.")
        su = p.num_simple_step[0] > 0
        kind = "simple" if su else "full"
        ups = self.inp.simple_updates if su else self.inp.full_updates
        groups = {u.group for u in ups}
        ngroups = max(groups) + 1 if groups else 1
        for g in range(ngroups):
            if groups and g not in groups:
                raise InputError(f"no {kind} update with group number {g}")

        def per_group(v: List, what: str) -> List:
            if len(v) == ngroups:
                return list(v)
            if len(v) == 1:
                return list(v) * ngroups
            raise InputError(f"size of {what} {len(v)} is not equal to the number of {kind} update groups.")

        nss = per_group(p.num_simple_step if su else p.num_full_step, "num_step")
        tau = per_group(p.tau_simple_step if su else p.tau_full_step, "tau")
        mi = list(p.measure_interval)
        while len(mi) < ngroups:
            mi.append(mi[-1])
        t = 0.0
        self.measure(t, "TE_")
        for g in range(ngroups):
            for step in range(nss[g]):
                t0 = _time.perf_counter()
                if su:
                    self.simple_update_step(g)
                else:
                    for up in ups:
                        if up.group == g:
                            self.full_update_op(up)
                self.env.sync()
                if su:
                    self.t_su += _time.perf_counter() - t0
                else:
                    self.t_fu += _time.perf_counter() - t0
                t += tau[g]
                if (step + 1) % mi[g] == 0:
                    self.measure(t, "TE_")
            if nss[g] % mi[g] != 0:
                self.measure(t, "TE_")

    def finite_temperature(self) -> None:
        """iTPS::finite_temperature (finite_temperature.cpp:22-86): imaginary-time
        simple-update steps on the density operator, beta += 2 tau per step,
        measure_density (measure.cpp:110-144) at beta = 0, every
        measure_interval steps and after the last step of a group."""
        p = self.p
        ups = self.inp.simple_updates
        groups = {u.group for u in ups}
        ngroups = max(groups) + 1 if groups else 1
        for g in range(ngroups):
            if groups and g not in groups:
                raise InputError(f"no simple update with group number {g}")

        def per_group(v: List, what: str) -> List:
            if len(v) == ngroups:
                return list(v)
            if len(v) == 1:
                return list(v) * ngroups
            raise InputError(f"size of {what} {len(v)} is not equal to the number of simple update groups.")

        nss = per_group(p.num_simple_step, "num_step")
        tau = per_group(p.tau_simple_step, "tau")
        mi = list(p.measure_interval)
        while len(mi) < ngroups:
            mi.append(mi[-1])
        beta = 0.0
        self.measure(beta, "FT_")
        for g in range(ngroups):
            for step in range(nss[g]):
                t0 = _time.perf_counter()
                self.simple_update_step(g)
                self.env.sync()
                self.t_su += _time.perf_counter() - t0
                beta += 2.0 * tau[g]
                if mi[g] > 0 and (step + 1) % mi[g] == 0:
                    self.measure(beta, "FT_")
            if mi[g] == 0 or nss[g] % mi[g] != 0:
                self.measure(beta, "FT_")

    def summary(self) -> None:
        """summary() (measure.cpp:81-107): time.dat."""
        with open(os.path.join(self.outdir, "time.dat"), "w") as f:
            f.write(f"time all           = {_time.perf_counter() - self.t0}\n")
            f.write(f"time simple update = {self.t_su}\n")
            f.write(f"time full update   = {self.t_fu}\n")
            f.write(f"time environment  = {self.t_env}\n")
            f.write(f"time observable    = {self.t_obs}\n")


def run_status(path: str, print_level: int = 1, device: int = 0) -> Tuple[int, str]:
    """The body of the C entry point tenes_gpu_main: run() with every error
    turned into a tg_status code and a message, nothing raised (the
    reference's tenes_itps_main lets its exceptions propagate,
    src/iTPS/main.cpp:33-39; a C caller cannot catch them)."""
    from ._lib import TG_E_INPUT, TG_E_LOAD, TG_E_RUNTIME, TGError
    from .saveload import LoadError
    try:
        run(path, device=device, print_level=print_level)
        return 0, ""
    except InputError as e:
        code, msg = TG_E_INPUT, f"input error: {e}"
    except LoadError as e:
        code, msg = TG_E_LOAD, f"load error: {e}"
    except TGError as e:
        code, msg = e.code, str(e)
    except (OSError, FileNotFoundError) as e:
        code, msg = TG_E_INPUT, f"input error: {e}"
    except Exception as e:  # noqa: BLE001 -- every failure becomes a status code
        code, msg = TG_E_RUNTIME, f"{type(e).__name__}: {e}"
    if print_level > 0:
        print(f"ERROR: {msg}", file=sys.stderr)
    return code, msg


def run(path: str, device: int = 0, mixed: bool = False, print_level: int = 1,
        outdir: Optional[str] = None) -> ITPS:
    """tenes_itps_main for one expert input file; `outdir` overrides
    parameter.general.output."""
    inp = load_input(path)
    if outdir is not None:
        inp.params.outdir = outdir
    it = ITPS(inp, device=device, mixed=mixed, print_level=print_level)
    # run_groundstate / run_timeevolution (main.cpp:141-177): the checkpoint
    # is written after the optimisation, before the measurement
    if inp.params.calcmode == "time_evolution":
        it.time_evolution()
        save_tensors(it.env, inp.params.tensor_save_dir, inp.params.CHI, print_level)
    elif inp.params.calcmode == "finite_temperature":  # run_finitetemperature (main.cpp:180-198)
        it.finite_temperature()
        save_tensors(it.env, inp.params.tensor_save_dir, inp.params.CHI, print_level)
    else:
        it.optimize()
        save_tensors(it.env, inp.params.tensor_save_dir, inp.params.CHI, print_level)
        if inp.params.to_measure:
            it.measure()
    it.summary()
    return it
