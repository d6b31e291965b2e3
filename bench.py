"""CTMRG throughput on B200: sweeps/s of the iTPS corner-transfer-matrix
environment (one sweep = Left, Right, Top, Bottom moves of
core::Calc_CTM_Environment, src/iTPS/core/ctm.cpp:1203-1243) and the time to
a converged environment, mixed precision against the FP64 path.

Workload (default): spin-1/2 antiferromagnetic Heisenberg model, 2x2 unit
cell, D=6, chi=72, site tensors from 300 seeded simple-update steps at
tau=0.01 run through the library itself, Neel initial state + noise 1e-2
(seed 11).  Data are synthetic; the reference publishes no benchmark suite.
`value` is the chosen form: 3xTF32 tcgen05 contractions with FP64 rSVD
projectors (k = chi+10, q = 2).  `time_to_converge` runs the chosen form, the
FP64 rSVD path and the FP64 full-SVD path (the reference's default projector)
from the same tensors until the energy per site moves by <= 1e-7 per sweep.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N>1 runs N independent replicas (one per GPU, different seeds; the CTMRG of
one unit cell does not shard) and reports the summed sweeps/s.
"""

from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

CONFIGS = {
    # name: (D, chi, su_steps, description)
    "c3": (6, 72, 300, "afh_square_2x2_D6_chi72_fp64"),
    "c2": (4, 32, 200, "afh_square_2x2_D4_chi32_fp64"),
    "c1": (2, 10, 100, "afh_square_2x2_D2_chi10_fp64"),
}
TAU = 0.01
SEED = 11
L2_BYTES = 126 * 1024 * 1024


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ------------------------------------------------------------------ workload
def lattice_spec(D):
    LX = LY = 2
    N = LX * LY
    pd = [2] * N
    vd = [[D] * 4 for _ in range(N)]
    # Neel pattern: sublattice A up, B down (parity of x + y)
    dirs = [[1.0, 0.0] if ((i % LX) + (i // LX)) % 2 == 0 else [0.0, 1.0] for i in range(N)]
    noises = [1e-2] * N
    return LX, LY, pd, vd, dirs, noises


def bonds(LX, LY):
    N = LX * LY
    return [(s, 2) for s in range(N)] + [(s, 1) for s in range(N)]


def heisenberg_op():
    from tenes_b200.std_ops import evolution_twosite, heisenberg_bond, real_if_close
    return real_if_close(evolution_twosite(heisenberg_bond(1.0), TAU))


# ------------------------------------------------------------------ our arm
def ctm_params(cfg, projector, precision="fp64"):
    from tenes_b200.env import CTMParams
    D, chi, _, _ = CONFIGS[cfg]
    mixed = precision == "mixed"
    if projector == "rsvd":
        # rSVD projectors, oversampling chi+10, 2 power iterations
        return CTMParams(chi=chi, max_ctm_iteration=1, use_rsvd=True, rsvd_oversample_abs=10,
                         rsvd_power_iters=2, mixed=mixed)
    return CTMParams(chi=chi, max_ctm_iteration=1, mixed=mixed)


def make_env(cfg, seed, device, projector="svd", su_steps=None, precision="fp64"):
    from tenes_b200.env import Environment
    D, chi, su_default, _ = CONFIGS[cfg]
    su_steps = su_default if su_steps is None else su_steps
    LX, LY, pd, vd, dirs, noises = lattice_spec(D)
    env = Environment(LX, LY, pd, vd, ctm_params(cfg, projector, precision), False, device=device)
    env.init_tensors(seed, dirs, noises)
    op = heisenberg_op()
    t0 = time.perf_counter()
    for _ in range(su_steps):
        for (s, leg) in bonds(LX, LY):
            env.simple_update(s, leg, op)
    log(f"[bench] {su_steps} simple-update steps in {time.perf_counter() - t0:.1f}s")
    env.init_env()
    return env


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(rows)}


def fp64_peak_tflops(device):
    """Measured FP64 dense GEMM peak of this GPU (cuBLAS DGEMM 8192^3)."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=device)
    b = torch.randn(n, n, dtype=torch.float64, device=device)
    for _ in range(2):
        a @ b
    torch.cuda.synchronize(device)
    best = 1e30
    for _ in range(3):
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record()
        a @ b
        e.record()
        torch.cuda.synchronize(device)
        best = min(best, s.elapsed_time(e))
    del a, b
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def traffic_from_profile(cfg, family):
    """DRAM bytes per launch of the product family's dominant shape from the
    committed ncu summary (profiles/roofline_traffic_<cfg>.md, a line
    `<family>: traffic_bytes_per_launch = X`), if any."""
    path = os.path.join(ROOT, "profiles", f"roofline_traffic_{cfg}.md")
    if not os.path.exists(path):
        return None
    m = re.search(family + r":\s*traffic_bytes_per_launch\s*=\s*([0-9.eE+]+)", open(path).read())
    return float(m.group(1)) if m else None


def bond_energy(env):
    """Energy per site: <S.S> over the horizontal and vertical bond of every
    site, each normalised by the same contraction with the identity
    (Contract_two_sites_*_op12 / norm, twosite_obs.cpp:180-225), both read
    from the bond's reduced density matrix (one contraction per bond)."""
    from tenes_b200.std_ops import heisenberg_bond, real_if_close
    h = real_if_close(heisenberg_bond(1.0))
    tot = 0.0
    for s in range(env.N):
        for dx, dy in ((1, 0), (0, 1)):
            rho = env.contract_bond_rdm(s, dx, dy)
            tot += (np.sum(h * rho) / np.einsum("abab->", rho)).real
    return tot / env.N


def prepare_tensors(cfg, seed, device, su_steps=None):
    """Site tensors from the seeded simple update, run by the library."""
    env = make_env(cfg, seed, device, "svd", su_steps, "fp64")
    T = [env.get_site_tensor(i) for i in range(env.N)]
    env.close()
    return T


def env_for(cfg, T, device, projector, precision, max_iter=1):
    from tenes_b200.env import Environment
    D, chi, _, _ = CONFIGS[cfg]
    LX, LY, pd, vd, _, _ = lattice_spec(D)
    p = ctm_params(cfg, projector, precision)
    p.max_ctm_iteration = max_iter
    env = Environment(LX, LY, pd, vd, p, False, device=device)
    for i, t in enumerate(T):
        env.set_site_tensor(i, t)
    env.init_env()
    return env


def converge(cfg, T, device, projector, precision, tol=1e-7, max_sweeps=40):
    """Time to a converged environment: sweeps until the energy per site
    changes by at most `tol` between successive sweeps (energy evaluations
    included in the wall time); the sweep at which the reference's own
    corner-spectrum criterion (eps = 1e-6, ctm.cpp:815-969) first holds is
    recorded too."""
    env = env_for(cfg, T, device, projector, precision)
    env.sync()
    t0 = time.perf_counter()
    e_prev, n, ref_conv, conv = None, 0, None, False
    e = float("nan")
    per_sweep = []  # (sweep, convergence check, energy) seconds
    while n < max_sweeps:
        ts = time.perf_counter()
        env.sweep()
        n += 1
        tc = time.perf_counter()
        c, _ = env.check_convergence()
        if c and ref_conv is None:
            ref_conv = n
        te = time.perf_counter()
        e = bond_energy(env)
        tz = time.perf_counter()
        per_sweep.append([round(tc - ts, 4), round(te - tc, 4), round(tz - te, 4)])
        if e_prev is not None and abs(e - e_prev) <= tol:
            conv = True
            break
        e_prev = e
    secs = time.perf_counter() - t0
    env.close()
    # host-side stalls (capture, allocator, other jobs on a shared machine) show
    # up as outliers of single sweeps; sweeps x the median sweep is the steady
    # rate's estimate of the same wall time
    med = statistics.median(sum(x) for x in per_sweep) if per_sweep else 0.0
    return {"sweeps": n, "seconds": secs, "seconds_sweeps_x_median": n * med, "converged": conv,
            "energy_per_site": e, "last_delta_e": (abs(e - e_prev) if e_prev is not None else None),
            "sweeps_to_corner_spectrum_eps_1e-6": ref_conv,
            "seconds_per_sweep_sweep_check_energy": per_sweep}


def max_over_ranks(ms, device, world):
    """The largest of the ranks' times (all-reduce MAX over the process
    group); unchanged for a single rank."""
    if world <= 1:
        return ms
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(world, steps, total_ms):
    """Whole-job sweeps/s of `world` independent replicas that each ran
    `steps` sweeps in at most `total_ms`."""
    return world * steps / (total_ms * 1e-3)


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from tenes_b200.env import (PROFILE_KINDS, kernel_launch_count, profile_enable, profile_query,
                                profile_reset)
    device = local_rank
    torch.cuda.set_device(device)
    T = prepare_tensors(args.config, SEED + rank, device, args.su_steps)
    env = env_for(args.config, T, device, args.projector, args.precision)
    stream = torch.cuda.ExternalStream(env.stream_handle(), device=device)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=device)

    for _ in range(args.warmup):
        env.sweep()
    if args.profile_sweep:
        # one sweep inside cudaProfilerStart/Stop for `ncu --profile-from-start off`
        torch.cuda.synchronize(device)
        torch.cuda.profiler.start()
        env.sweep()
        env.sync()
        torch.cuda.profiler.stop()
    times = []
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(device)
    clocks = Clocks(device)
    clocks.start()
    if args.profile_timed:
        profile_enable(True)
        profile_reset()
    l0 = kernel_launch_count()
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)  # L2 flush outside the timed window
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record(stream)
        env.sweep()
        e.record(stream)
        e.synchronize()
        times.append(s.elapsed_time(e))
    launches = kernel_launch_count() - l0
    torch.cuda.synchronize(device)
    ck = clocks.stop()
    timed_breakdown = None
    if args.profile_timed:
        timed_breakdown = {PROFILE_KINDS[k]: round(profile_query(k)[1] / args.steps, 3)
                           for k in range(len(PROFILE_KINDS))}
        profile_enable(False)
    total_ms = max_over_ranks(sum(times), device, world)
    if world > 1:
        dist.barrier()
    ms_per_step = total_ms / args.steps
    value = replica_rate(world, args.steps, total_ms)

    # ---- end to end through the C ABI with host buffers (set Tn + env, sweep, get env)
    # page-locked host buffers (allocated and filled outside the timed region)
    def pinned_copy(x):
        t = torch.empty(x.shape, dtype=torch.float64 if x.dtype == np.float64 else torch.complex128, pin_memory=True)
        v = t.numpy()
        v[...] = x
        return t, v
    keep_alive = []
    host_T = []
    for i in range(env.N):
        t, v = pinned_copy(env.get_site_tensor(i))
        keep_alive.append(t)
        host_T.append(v)
    host_env = [[None] * env.N for _ in range(8)]
    for w in range(8):
        for i in range(env.N):
            t, v = pinned_copy(env.get_env(w, i))
            keep_alive.append(t)
            host_env[w][i] = v
    h2d = sum(t.nbytes for t in host_T) + sum(t.nbytes for ws in host_env for t in ws)
    e2e_ms = 0.0
    for _ in range(args.steps):
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record(stream)
        for i, Ti in enumerate(host_T):
            env.set_site_tensor(i, Ti)
        for w in range(8):
            for i in range(env.N):
                env.set_env(w, i, host_env[w][i])
        env.sweep()
        for w in range(8):
            for i in range(env.N):
                env.get_env(w, i, out=host_env[w][i])
        e.record(stream)
        e.synchronize()
        e2e_ms += s.elapsed_time(e)
    e2e_ms = max_over_ranks(e2e_ms, device, world)
    e2e = {"value": replica_rate(world, args.steps, e2e_ms), "unit": "sweeps/s",
           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": sum(t.nbytes for ws in host_env for t in ws),
           "host_buffers": "page-locked; per step: 4 site tensors + 32 environment tensors up through "
                           "tg_set_site_tensor / tg_set_env, one tg_ctm_sweep, 32 environment tensors down "
                           "through tg_get_env"}

    # ---- per-family device time of one instrumented sweep (roofline of the dominant product kernel)
    profile_enable(True)
    profile_reset()
    env.sweep()
    env.sync()
    fam = {PROFILE_KINDS[k]: profile_query(k) for k in range(len(PROFILE_KINDS))}
    profile_enable(False)
    env.close()
    peaks = measured_peaks()
    if fam["gemm_tcgen05"][1] >= fam["gemm_dmma"][1]:
        n_g, ms_g, fl_g, _ = fam["gemm_tcgen05"]
        issued = 3.0 * fl_g  # three TF32 products per multiply-add
        peak = peaks.get("bf16_tflops_sustained", 1411.5) / 2.0
        roof = {"bound": "tensor", "kernel": "gemm_tma_kernel (tcgen05 kind::tf32, 3 products; split/pack included)",
                "achieved": issued / (ms_g * 1e-3) / 1e12 if ms_g > 0 else 0.0, "peak": peak,
                "peak_source": "MEASURED_PEAKS.json bf16_tflops_sustained / 2 (dense TF32 rate, of measured)",
                "algorithmic_tflops": fl_g / (ms_g * 1e-3) / 1e12 if ms_g > 0 else 0.0}
    else:
        n_g, ms_g, fl_g, _ = fam["gemm_dmma"]
        peak = fp64_peak_tflops(device) if rank == 0 else None
        roof = {"bound": "tensor", "kernel": "gemm_kernel (FP64 DMMA m8n8k4)",
                "achieved": fl_g / (ms_g * 1e-3) / 1e12 if ms_g > 0 else 0.0, "peak": peak,
                "peak_source": "measured in-run: cuBLAS DGEMM 8192^3 FP64 (MEASURED_PEAKS.json has no FP64 entry)"}
    roof.update({"unit": "TFLOP/s", "frac": (roof["achieved"] / roof["peak"]) if roof["peak"] else None,
                 "traffic": traffic_from_profile(args.config, "gemm_tcgen05" if "tcgen05" in roof["kernel"]
                                                 else "gemm_dmma"),
                 "traffic_note": "DRAM bytes of one launch of the family's dominant shape (the rSVD range-finder "
                                 "product 2592 x 82 x 2592), from profiles/roofline_traffic_<config>.md",
                 "launches_per_sweep": n_g,
                 "avg_launch_us": 1e3 * ms_g / max(n_g, 1), "flops_per_launch": fl_g / max(n_g, 1),
                 "sweep_breakdown_ms": {k: round(v[1], 3) for k, v in fam.items()}})

    # ---- time to a converged environment: the chosen form against the FP64 plain path
    conv = None
    if args.converge != "none":
        conv = {"criterion": "|E/site(sweep t) - E/site(sweep t-1)| <= 1e-7 (energy evaluations timed too)"}
        conv["mixed_rsvd"] = converge(args.config, T, device, "rsvd", "mixed")
        conv["fp64_rsvd"] = converge(args.config, T, device, "rsvd", "fp64")
        if args.converge == "full":
            conv["fp64_full_svd"] = converge(args.config, T, device, "svd", "fp64", max_sweeps=30)
        base = conv.get("fp64_full_svd") or conv["fp64_rsvd"]
        conv["speedup_mixed_vs_fp64_full_svd"] = (conv["fp64_full_svd"]["seconds"] / conv["mixed_rsvd"]["seconds"]
                                                  if "fp64_full_svd" in conv else None)
        conv["speedup_mixed_vs_fp64_rsvd"] = conv["fp64_rsvd"]["seconds"] / conv["mixed_rsvd"]["seconds"]
        conv["abs_delta_e_mixed_vs_fp64"] = abs(conv["mixed_rsvd"]["energy_per_site"] - base["energy_per_site"])
    return {"value": value, "ms_per_step": ms_per_step, "e2e": e2e, "roofline": roof,
            "clocks": ck, "gpu_launches": launches, "sweep_ms": [round(t, 3) for t in times],
            "timed_breakdown_ms": timed_breakdown, "converge": conv}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


# -------------------------------------------------------- CPU oracle (reference arm)
def oracle_sample(cfg, rank=0):
    """Time one Left_move of the CPU oracle on the same workload; one sweep is
    4*LX... = 8 moves of this size for a 2x2 cell."""
    from oracle import tenes_oracle as O
    D, chi, su_steps, _ = CONFIGS[cfg]
    LX, LY, pd, vd, dirs, noises = lattice_spec(D)
    lat = O.Lattice(LX, LY)
    lat.physical_dims = pd
    lat.virtual_dims = vd
    lat.initial_dirs = dirs
    lat.noises = noises
    Tn = O.initialize_tensors(lat, SEED + rank, True)
    lam = [[np.ones(D) for _ in range(4)] for _ in range(lat.N_UNIT)]
    p = O.Params(CHI=chi)
    op = heisenberg_op()
    for _ in range(su_steps):
        for (s, leg) in bonds(LX, LY):
            tg = lat.neighbor(s, leg)
            a, b, lc = O.simple_update_bond(Tn[s], Tn[tg], lam[s], lam[tg], op, leg, p)
            lam[s][leg] = lc
            lam[tg][(leg + 2) % 4] = lc
            Tn[s], Tn[tg] = a, b
    env = O.init_env(Tn, p, lat)
    return lat, Tn, p, env


def time_oracle_move(lat, Tn, p, env):
    from oracle import tenes_oracle as O
    t0 = time.perf_counter()
    O.left_move(env, Tn, 0, p, lat)
    return time.perf_counter() - t0


def moves_per_sweep(lat):
    return 2 * lat.LX_noskew + 2 * lat.LY_noskew


def run_reference(args, rank, world):
    if rank != 0:
        return None
    lat, Tn, p, env = oracle_sample(args.config)
    for _ in range(args.warmup):
        time_oracle_move(lat, Tn, p, env)
    tot = 0.0
    for _ in range(args.steps):
        tot += time_oracle_move(lat, Tn, p, env)
    per_sweep = tot / args.steps * moves_per_sweep(lat)
    v = 1.0 / per_sweep
    cores = os.cpu_count()
    D, chi, _, name = CONFIGS[args.config]
    return {"metric": "ctmrg_sweeps_per_s", "value": v, "unit": "sweeps/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_sweep * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": name, "D": D, "chi": chi, "unit_cell": "2x2", "projector": "full SVD"},
            "cpu_baseline": {"value": v, "unit": "sweeps/s", "cores": cores, "kind": "port",
                             "sample": "one Left_move (2 projector rows, full SVD) of the CPU oracle per step, "
                                       f"x{moves_per_sweep(lat)} moves per sweep"},
            "e2e": {"value": v, "unit": "sweeps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# J1-J2 gradient workload: 2x2 cell, d = 2, D = 3, chi = 36, J2 = 0.5, site
# tensors i.i.d. normal(0, 1), 25 CTMRG sweeps checkpointed every 5
GRAD = dict(D=3, chi=36, iterations=25, checkpoint_every=5, J1=1.0, J2=0.5, fd_step=1e-5)


def grad_problem(seed):
    from tenes_b200.grad import j1j2_terms
    rng = np.random.default_rng(seed)
    D = GRAD["D"]
    Tn = [rng.standard_normal((D, D, D, D, 2)) for _ in range(4)]
    return Tn, j1j2_terms(4, GRAD["J1"], GRAD["J2"])


def grad_env(Tn, mixed):
    from tenes_b200.env import CTMParams, Environment
    D = GRAD["D"]
    env = Environment(2, 2, [2] * 4, [[D] * 4 for _ in range(4)],
                      CTMParams(chi=GRAD["chi"], max_ctm_iteration=1, mixed=mixed), False)
    for i, t in enumerate(Tn):
        env.set_site_tensor(i, t)
    return env


def run_grad(args):
    """Gradient evaluations/s of the J1-J2 energy (hand-written adjoint
    through the sweeps and the projector SVDs), the central-difference check
    on seeded entries, and the mixed-precision (3xTF32 moves) arm."""
    from tenes_b200.env import kernel_launch_count
    Tn, terms = grad_problem(SEED)
    it, ck = args.grad_iters, GRAD["checkpoint_every"]

    def timed(env, grad=True):
        t0 = time.perf_counter()
        out = env.energy_grad(terms, it, ck, grad=grad)
        return out, time.perf_counter() - t0

    from tenes_b200.env import profile_enable, profile_query, profile_reset
    env = grad_env(Tn, False)
    env.energy_grad(terms, 1, ck)  # warm-up (library and solver initialisation)
    l0 = kernel_launch_count()
    times = []
    for _ in range(args.steps):
        (E, g), dt = timed(env)
        times.append(dt)
    launches = (kernel_launch_count() - l0) // max(args.steps, 1)
    profile_enable(True)
    profile_reset()
    _, t_fwd = timed(env, grad=False)
    kinds = ["gemm_dmma", "permute", "normalize", "spectrum", "factorisations", "other", "gemm_tcgen05"]
    breakdown = {k: round(profile_query(q)[1], 3) for q, k in enumerate(kinds)}
    profile_enable(False)
    gmax = max(float(np.abs(x).max()) for x in g)
    rng = np.random.default_rng(SEED + 1)
    errs, h = [], GRAD["fd_step"]
    for _ in range(args.grad_fd):
        site = int(rng.integers(4))
        idx = tuple(int(rng.integers(n)) for n in Tn[site].shape)
        vals = []
        for sgn in (1, -1):
            T = Tn[site].copy()
            T[idx] += sgn * h
            env.set_site_tensor(site, T)
            vals.append(env.energy_grad(terms, it, ck, grad=False)[0])
        env.set_site_tensor(site, Tn[site])
        fd = (vals[0] - vals[1]) / (2 * h)
        errs.append(abs(fd - g[site][idx]) / max(abs(fd), abs(g[site][idx]), 1e-3 * gmax))
    env.close()
    envm = grad_env(Tn, True)
    envm.energy_grad(terms, 1, ck)
    tm = []
    for _ in range(args.steps):
        (Em, gm), dt = timed(envm)
        tm.append(dt)
    envm.close()
    gv = np.concatenate([x.reshape(-1) for x in g])
    gmv = np.concatenate([x.reshape(-1) for x in gm])
    med, medm = float(np.median(times)), float(np.median(tm))
    return {"metric": "gradient_evaluations_per_s", "value": 1.0 / med, "unit": "evals/s", "n_gpus": 1,
            "steps": args.steps, "warmup": 1, "ms_per_step": 1e3 * med, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (site tensors i.i.d. normal(0,1), seeded)",
            "config": {"workload": "j1j2_square_2x2_D3_chi36_J2_0.5_fp64", "D": GRAD["D"], "chi": GRAD["chi"],
                       "iterations": it, "checkpoint_every": ck, "projector": "full SVD",
                       "timing": "host wall clock around tg_energy_grad (synchronous call)"},
            "energy_per_site": E, "seconds_energy_only": t_fwd, "gpu_launches": int(launches),
            "energy_only_breakdown_ms": breakdown,
            "fd_check": {"entries": args.grad_fd, "step": h, "max_rel_err": max(errs) if errs else None},
            "mixed": {"value": 1.0 / medm, "unit": "evals/s", "energy_per_site": Em,
                      "abs_delta_e": abs(Em - E),
                      "grad_rel_err": float(np.linalg.norm(gmv - gv) / np.linalg.norm(gv))}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c3", choices=sorted(CONFIGS))
    ap.add_argument("--projector", default="rsvd", choices=["svd", "rsvd"],
                    help="svd: full SVD (reference default); rsvd: k = chi+10, 2 power iterations")
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"],
                    help="mixed: 3xTF32 tcgen05 contractions, FP64 projector algebra")
    ap.add_argument("--converge", default="full", choices=["full", "fast", "none"],
                    help="time-to-converge arms: full = mixed rSVD, FP64 rSVD and FP64 full SVD; "
                         "fast = without the FP64 full-SVD arm")
    ap.add_argument("--su-steps", type=int, default=None,
                    help="override the simple-update steps that prepare the tensors (profiling runs)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-timed", action="store_true",
                    help="CUDA-event profile of the library kernels during the timed sweeps (diagnostic)")
    ap.add_argument("--profile-sweep", action="store_true",
                    help="wrap one extra sweep in cudaProfilerStart/Stop (for ncu)")
    ap.add_argument("--grad", action="store_true",
                    help="gradient evaluations/s of the J1-J2 energy (D=3, chi=36) with the FD check")
    ap.add_argument("--grad-iters", type=int, default=GRAD["iterations"])
    ap.add_argument("--grad-fd", type=int, default=32, help="entries checked by central differences")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    if args.grad:
        print(json.dumps(run_grad(args)), flush=True)
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        out = run_reference(args, rank, world)
        if out is not None:
            print(json.dumps(out), flush=True)
        return

    import torch
    import torch.distributed as dist
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    res = run_ours(args, rank, world, local_rank)
    if rank == 0:
        D, chi, su, name = CONFIGS[args.config]
        cpu = None
        if not args.no_cpu_baseline:
            lat, Tn, p, env = oracle_sample(args.config)
            t = time_oracle_move(lat, Tn, p, env)
            v = 1.0 / (t * moves_per_sweep(lat))
            cpu = {"value": v, "unit": "sweeps/s", "cores": os.cpu_count(), "kind": "port",
                   "sample": f"one Left_move of the CPU oracle (numpy FP64, full SVD), x{moves_per_sweep(lat)} "
                             "moves per sweep"}
        line = {"metric": "ctmrg_sweeps_per_s", "value": res["value"], "unit": "sweeps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if args.precision == "fp64" else "tf32x3+f64",
                "data": "synthetic (seeded simple-update tensors of the workload's shapes)",
                "config": {"workload": f"{name}_{args.precision}_{args.projector}", "precision": args.precision,
                           "D": D, "chi": chi, "unit_cell": "2x2", "su_steps": su,
                           "projector": ("full SVD (reference default)" if args.projector == "svd"
                                         else "rSVD k=chi+10, q=2"), "parallelism": f"replicas{world}",
                           "l2": "flushed between timed sweeps (252 MB write outside the timed window)"},
                "roofline": res["roofline"], "cpu_baseline": cpu, "e2e": res["e2e"],
                "clocks": res["clocks"], "gpu_launches": res["gpu_launches"], "sweep_ms": res["sweep_ms"]}
        if res["converge"] is not None:
            line["time_to_converge"] = res["converge"]
        if res["timed_breakdown_ms"] is not None:
            line["timed_breakdown_ms"] = res["timed_breakdown_ms"]
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
