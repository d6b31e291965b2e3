"""CTMRG throughput on B200: sweeps/s of the iTPS corner-transfer-matrix
environment (one sweep = Left, Right, Top, Bottom moves of
core::Calc_CTM_Environment, src/iTPS/core/ctm.cpp:1203-1243) and the time to
a converged environment, FP64 and mixed precision.

Workload (default c3): spin-1/2 antiferromagnetic Heisenberg model, 2x2 unit
cell, D=6, chi=72, site tensors from 300 seeded simple-update steps at
tau=0.01 run through the library itself from a Neel initial state + noise
1e-2 (iTPS::initialize_tensors, seed 11).  Data are synthetic; the reference
publishes no benchmark suite.

`value` is the FP64 path with rSVD projectors (k = chi+10, q = 2), the same
arithmetic and the same algorithm as the reference arm (`--impl reference`:
the FP64 CPU oracle with the same projectors, on all host cores).  Beside it
the line reports the mixed form (3xTF32 tcgen05 contractions, FP64 projector
algebra) at the same projectors, the FP64 full-SVD path (the reference's
default projector), the time to a converged environment of all three, and
each arm's energy per site against the FP64 oracle run from the same site
tensors.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    python bench.py --ft     # iTPO: single-layer CTMRG, density simple update, FT_TFI_square run
    python bench.py --grad   # energy gradient of the J1-J2 model (adjoint CTMRG)

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

# name: workload of one 2x2 unit cell
#   afh: J (SxSx + SySy + SzSz), Neel + noise 1e-2 through initialize_tensors
#   tfi: -SzSz bonds and a -hx Sx field (one-site evolution operators), site
#        tensors i.i.d. uniform[-1, 1] from the seed, each scaled to max |entry| = 1
CONFIGS = {
    "c3": dict(model="afh", D=6, chi=72, su_steps=300, name="afh_square_2x2_D6_chi72"),
    "c2": dict(model="afh", D=4, chi=32, su_steps=200, name="afh_square_2x2_D4_chi32"),
    "c1": dict(model="tfi", D=2, chi=10, su_steps=1000, name="tfi_square_2x2_D2_chi10_hx1"),
    # Kitaev honeycomb on the brick wall, 4x4, complex, per-bond D from {3, 4, 5} (seeded), one vertical
    # leg of every site of dimension 1, chi = 48; site tensors i.i.d. uniform[-1, 1] (real and imaginary
    # parts); 40 CTMRG sweeps; energy per site and plaquette flux
    "c5": dict(model="kitaev", D=5, dims=(3, 4, 5), chi=48, su_steps=0, sweeps=40,
               name="kitaev_brickwall_4x4_D345_chi48_h0.05"),
}
HX = 1.0
KITAEV_H = 0.05  # [111] field: -h (Sx + Sy + Sz) on every site
TAU = 0.01
SEED = 11
L2_BYTES = 126 * 1024 * 1024
RSVD_OVERSAMPLE, RSVD_POWER = 10, 2


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


def brick_wall_dims(LX=4, LY=4, seed=5, dims=(3, 4, 5)):
    """Virtual dimensions [site][left, up, right, bottom] of the honeycomb
    lattice on the brick wall: every horizontal bond present, a vertical bond
    only above the sites of odd x + y (the others have an up leg of dimension
    1, so their left / right moves take the identity projector,
    ctm.cpp:303-317); each present bond's dimension drawn from `dims`."""
    rng = np.random.default_rng(seed)
    N = LX * LY
    right = lambda i: (i % LX + 1) % LX + (i // LX) * LX  # noqa: E731
    top = lambda i: i % LX + ((i // LX + 1) % LY) * LX  # noqa: E731
    vd = [[0] * 4 for _ in range(N)]
    for i in range(N):
        vd[i][2] = vd[right(i)][0] = int(rng.choice(dims))
    for i in range(N):
        x, y = i % LX, i // LX
        vd[i][1] = vd[top(i)][3] = int(rng.choice(dims)) if (x + y) % 2 == 1 else 1
    return vd


def cell(cfg):
    """(LX, LY, physical dims, virtual dims, initial directions, noises, complex) of a workload."""
    c = CONFIGS[cfg]
    if c["model"] == "kitaev":
        vd = brick_wall_dims(dims=c["dims"])
        return 4, 4, [2] * 16, vd, [[0.0, 0.0] for _ in range(16)], [0.0] * 16, True
    LX, LY, pd, vd, dirs, noises = lattice_spec(c["D"])
    return LX, LY, pd, vd, dirs, noises, False


def random_complex_tensors(vd, seed):
    """Site tensors with real and imaginary parts i.i.d. uniform[-1, 1]."""
    rng = np.random.default_rng(seed)
    out = []
    for v in vd:
        sh = (v[0], v[1], v[2], v[3], 2)
        out.append(rng.uniform(-1.0, 1.0, sh) + 1j * rng.uniform(-1.0, 1.0, sh))
    return out


def kitaev_bond_list(vd, LX=4, LY=4):
    """(site, dx, dy, Pauli-pair index) of every Kitaev bond: x and y bonds
    alternate along the rows (x to the right of an even-parity site), z bonds
    on the present vertical legs; the bond term is -K S^a S^a with K = 1."""
    out = []
    for i in range(LX * LY):
        x, y = i % LX, i // LX
        out.append((i, 1, 0, 0 if (x + y) % 2 == 0 else 1))
        if vd[i][1] > 1:
            out.append((i, 0, 1, 2))
    return out


def spin_half():
    sx = np.array([[0.0, 0.5], [0.5, 0.0]], dtype=complex)
    sy = np.array([[0.0, -0.5j], [0.5j, 0.0]])
    sz = np.array([[0.5, 0.0], [0.0, -0.5]], dtype=complex)
    return sx, sy, sz


def hexagons(LX=4, LY=4):
    """Bottom-left sites of the hexagons of the cell (odd x + y) and the Pauli
    operator of each of the six sites on the 2 x 3 window -- the one of the
    site's bond that leaves the hexagon: bottom row x, z, y; top row y, z, x."""
    S = spin_half()
    ops = {(1, 0): 2 * S[0], (1, 1): 2 * S[2], (1, 2): 2 * S[1], (0, 0): 2 * S[1], (0, 1): 2 * S[2], (0, 2): 2 * S[0]}
    return [i for i in range(LX * LY) if ((i % LX) + (i // LX)) % 2 == 1], ops


def kitaev_observables(env, vd):
    """Energy per site (-K S^a S^a on every bond from the bond's reduced
    density matrix, -h (Sx + Sy + Sz) on every site) and the mean plaquette
    flux W_p = <prod_j sigma_j> over the cell's hexagons (2 x 3 windows)."""
    S = spin_half()
    tot = 0.0
    for (s, dx, dy, a) in kitaev_bond_list(vd):
        rho = env.contract_bond_rdm(s, dx, dy)
        h = -np.einsum("ac,bd->abcd", S[a], S[a])
        tot += (np.sum(h * rho) / np.einsum("abab->", rho)).real
    f = S[0] + S[1] + S[2]
    for s in range(env.N):
        tot -= KITAEV_H * (env.contract_one_site(s, f) / env.contract_one_site(s, np.eye(2))).real
    starts, ops = hexagons()
    flux = [(env.contract_window(s, 2, 3, 1, 0, ops) / env.contract_window(s, 2, 3, 1, 0)).real for s in starts]
    return tot / env.N, float(np.mean(flux))


def bonds(LX, LY):
    N = LX * LY
    return [(s, 2) for s in range(N)] + [(s, 1) for s in range(N)]


def heisenberg_op():
    from tenes_b200.std_ops import evolution_twosite, heisenberg_bond, real_if_close
    return real_if_close(evolution_twosite(heisenberg_bond(1.0), TAU))


def su_ops(cfg):
    """(bond evolution operator, one-site evolution operator or None)."""
    from tenes_b200.std_ops import evolution_onesite, evolution_twosite, ising_bond, real_if_close, spin_ops
    if CONFIGS[cfg]["model"] == "afh":
        return heisenberg_op(), None
    _, Sx, _ = spin_ops(0.5)
    return (real_if_close(evolution_twosite(ising_bond(1.0), TAU)),
            real_if_close(evolution_onesite(-HX * Sx, TAU)))


def bond_hamiltonian(cfg):
    from tenes_b200.std_ops import heisenberg_bond, ising_bond, real_if_close
    return real_if_close(heisenberg_bond(1.0) if CONFIGS[cfg]["model"] == "afh" else ising_bond(1.0))


def uniform_tensors(D, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(4):
        t = rng.uniform(-1.0, 1.0, (D, D, D, D, 2))
        out.append(t / np.abs(t).max())
    return out


# ------------------------------------------------------------------ our arm
def ctm_params(cfg, projector, precision="fp64"):
    from tenes_b200.env import CTMParams
    chi = CONFIGS[cfg]["chi"]
    mixed = precision == "mixed"
    if projector == "rsvd":
        # rSVD projectors, oversampling chi+10, 2 power iterations
        return CTMParams(chi=chi, max_ctm_iteration=1, use_rsvd=True, rsvd_oversample_abs=RSVD_OVERSAMPLE,
                         rsvd_power_iters=RSVD_POWER, mixed=mixed)
    return CTMParams(chi=chi, max_ctm_iteration=1, mixed=mixed)


def make_env(cfg, seed, device, projector="svd", su_steps=None, precision="fp64"):
    from tenes_b200.env import Environment
    c = CONFIGS[cfg]
    D = c["D"]
    su_steps = c["su_steps"] if su_steps is None else su_steps
    LX, LY, pd, vd, dirs, noises, cx = cell(cfg)
    env = Environment(LX, LY, pd, vd, ctm_params(cfg, projector, precision), cx, device=device)
    if c["model"] == "afh":
        env.init_tensors(seed, dirs, noises)
    elif c["model"] == "kitaev":
        for i, t in enumerate(random_complex_tensors(vd, seed)):
            env.set_site_tensor(i, t)
    else:
        for i, t in enumerate(uniform_tensors(D, seed)):
            env.set_site_tensor(i, t)
    op, op1 = su_ops(cfg) if su_steps else (None, None)
    step = [(s, leg, op) for (s, leg) in bonds(LX, LY)]
    if op1 is not None:
        step += [(s, -1, op1) for s in range(env.N)]
    t0 = time.perf_counter()
    for _ in range(su_steps):
        env.simple_update_many(step)  # one library call a step
    env.sync()
    env.su_seconds = time.perf_counter() - t0
    log(f"[bench] {su_steps} simple-update steps in {env.su_seconds:.2f}s")
    env.init_env()
    return env


def su_rate_gpu(cfg, seed, device, steps=None):
    """Simple-update steps/s of the library (one step = every bond of the
    cell, plus the one-site operators of the Ising field), host wall clock
    around a synchronised loop from the seeded start."""
    env = make_env(cfg, seed, device, "svd", steps, "fp64")
    n = CONFIGS[cfg]["su_steps"] if steps is None else steps
    rate = n / env.su_seconds
    env.close()
    return rate


def su_rate_oracle(cfg, seed, steps):
    """The same for the CPU oracle (core::Simple_update_bond restated), on a
    sample of `steps` steps."""
    from oracle import tenes_oracle as O
    c = CONFIGS[cfg]
    D = c["D"]
    lat = oracle_lattice(cfg)
    Tn = O.initialize_tensors(lat, seed, True) if c["model"] == "afh" else uniform_tensors(D, seed)
    lam = [[np.ones(D) for _ in range(4)] for _ in range(lat.N_UNIT)]
    p = O.Params()
    op, op1 = su_ops(cfg)
    t0 = time.perf_counter()
    for _ in range(steps):
        for (s, leg) in bonds(lat.LX, lat.LY):
            tg = lat.neighbor(s, leg)
            a, b, lc = O.simple_update_bond(Tn[s], Tn[tg], lam[s], lam[tg], op, leg, p)
            lam[s][leg] = lc
            lam[tg][(leg + 2) % 4] = lc
            Tn[s], Tn[tg] = a, b
        if op1 is not None:
            for s in range(lat.N_UNIT):
                Tn[s] = np.tensordot(Tn[s], op1, ([4], [0]))
    return steps / (time.perf_counter() - t0)


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


def bond_energy(env, cfg="c3"):
    """Energy per site: the bond Hamiltonian over the horizontal and vertical
    bond of every site, each normalised by the same contraction with the
    identity (Contract_two_sites_*_op12 / norm, twosite_obs.cpp:180-225), both
    read from the bond's reduced density matrix (one contraction per bond);
    for the Ising workload plus the field term -hx <Sx> of every site."""
    if CONFIGS[cfg]["model"] == "kitaev":
        return kitaev_observables(env, cell(cfg)[3])[0]
    h = bond_hamiltonian(cfg)
    tot = 0.0
    for s in range(env.N):
        for dx, dy in ((1, 0), (0, 1)):
            rho = env.contract_bond_rdm(s, dx, dy)
            tot += (np.sum(h * rho) / np.einsum("abab->", rho)).real
    if CONFIGS[cfg]["model"] == "tfi":
        sx = np.array([[0.0, 0.5], [0.5, 0.0]])
        for s in range(env.N):
            tot -= HX * (env.contract_one_site(s, sx) / env.contract_one_site(s, np.eye(2))).real
    return tot / env.N


def prepare_tensors(cfg, seed, device, su_steps=None):
    """Site tensors from the seeded simple update, run by the library, and
    the simple update's steps/s."""
    env = make_env(cfg, seed, device, "svd", su_steps, "fp64")
    T = [env.get_site_tensor(i) for i in range(env.N)]
    n = CONFIGS[cfg]["su_steps"] if su_steps is None else su_steps
    rate = n / env.su_seconds if env.su_seconds > 0 else None
    env.close()
    return T, rate


def env_for(cfg, T, device, projector, precision, max_iter=1):
    from tenes_b200.env import Environment
    LX, LY, pd, vd, _, _, cx = cell(cfg)
    p = ctm_params(cfg, projector, precision)
    p.max_ctm_iteration = max_iter
    env = Environment(LX, LY, pd, vd, p, cx, device=device)
    for i, t in enumerate(T):
        env.set_site_tensor(i, t)
    env.init_env()
    return env


def converge(cfg, T, device, projector, precision, tol=1e-7, max_sweeps=40):
    """Time to a converged environment: sweeps until the energy per site
    changes by at most `tol` between successive sweeps (energy evaluations
    included in the wall time).  The sweeps go on, up to `max_sweeps`, until
    the reference's own corner-spectrum criterion (eps = 1e-6,
    ctm.cpp:815-969; the library's check after every sweep) holds as well,
    and the sweep and time at which each criterion first held are reported."""
    env = env_for(cfg, T, device, projector, precision)
    env.sync()
    t0 = time.perf_counter()
    e_prev, n, ref_conv, ref_secs, conv, secs, n_conv, e_conv = None, 0, None, None, False, None, None, None
    e = float("nan")
    per_sweep = []  # (sweep, convergence check, energy) seconds
    energies = []
    while n < max_sweeps:
        ts = time.perf_counter()
        env.sweep()
        n += 1
        tc = time.perf_counter()
        c, _ = env.check_convergence()
        te = time.perf_counter()
        e = bond_energy(env, cfg)
        tz = time.perf_counter()
        energies.append(e)
        per_sweep.append([round(tc - ts, 4), round(te - tc, 4), round(tz - te, 4)])
        if c and ref_conv is None:
            ref_conv, ref_secs = n, tz - t0
        if not conv and e_prev is not None and abs(e - e_prev) <= tol:
            conv, secs, n_conv, e_conv = True, tz - t0, n, e
        if conv and ref_conv is not None:
            break
        e_prev = e
    if not conv:
        secs, n_conv, e_conv = time.perf_counter() - t0, n, e
    env.close()
    # host-side stalls (capture, allocator, other jobs on a shared machine) show
    # up as outliers of single sweeps; sweeps x the median sweep is the steady
    # rate's estimate of the same wall time
    med = statistics.median(sum(x) for x in per_sweep[:n_conv]) if per_sweep else 0.0
    return {"sweeps": n_conv, "seconds": secs, "seconds_sweeps_x_median": n_conv * med, "converged": conv,
            "energy_per_site": e_conv,
            "last_delta_e": abs(energies[n_conv - 1] - energies[n_conv - 2]) if n_conv >= 2 else None,
            "sweeps_to_corner_spectrum_eps_1e-6": ref_conv, "seconds_to_corner_spectrum_eps_1e-6": ref_secs,
            "sweeps_run": n, "energy_per_sweep": energies, "seconds_per_sweep_sweep_check_energy": per_sweep}


def kitaev_run(cfg, T, device, projector, precision="fp64"):
    """The Kitaev workload's run: a fixed number of sweeps from the initial
    environment, timed on the host around synchronised sweeps, then the energy
    per site and the mean plaquette flux."""
    n = CONFIGS[cfg]["sweeps"]
    env = env_for(cfg, T, device, projector, precision)
    env.sync()
    t0 = time.perf_counter()
    for _ in range(n):
        env.sweep()
    env.sync()
    secs = time.perf_counter() - t0
    e, w = kitaev_observables(env, cell(cfg)[3])
    env.close()
    return {"sweeps": n, "seconds": secs, "sweeps_per_s": n / secs, "energy_per_site": e, "plaquette_flux": w}


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


def timed_sweeps(env, steps, warmup, stream, flush):
    """Device time (ms) of each of `steps` sweeps after `warmup` untimed ones:
    CUDA events on the context's stream, an L2 flush before each."""
    import torch
    for _ in range(warmup):
        env.sweep()
    env.sync()
    times = []
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)  # L2 flush outside the timed window
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record(stream)
        env.sweep()
        e.record(stream)
        e.synchronize()
        times.append(s.elapsed_time(e))
    return times


def sweep_profile(env):
    """Per-family device time of one instrumented sweep: {family: (launches, ms, flops, bytes)}."""
    from tenes_b200.env import PROFILE_KINDS, profile_enable, profile_query, profile_reset
    profile_enable(True)
    profile_reset()
    env.sweep()
    env.sync()
    fam = {PROFILE_KINDS[k]: profile_query(k) for k in range(len(PROFILE_KINDS))}
    profile_enable(False)
    return fam


def roofline_fp64(fam, peak_tflops, cfg):
    """FP64 DMMA products (gemm_kernel, gemm_narrow_kernel, gemm_group_kernel,
    skinny_kernel): compute-bound at intensity >> the FP64 ridge (~6 flop/B),
    so the roof is the measured DGEMM rate."""
    n_g, ms_g, fl_g, by_g = fam["gemm_dmma"]
    ach = fl_g / (ms_g * 1e-3) / 1e12 if ms_g > 0 else 0.0
    return {"bound": "tensor", "kernel": "gemm_kernel + gemm_narrow_kernel + gemm_group_kernel + skinny_kernel "
                                         "(FP64 DMMA m8n8k4)",
            "achieved": ach, "peak": peak_tflops, "unit": "TFLOP/s",
            "frac": ach / peak_tflops if peak_tflops else None,
            "peak_source": "measured in-run: cuBLAS DGEMM 8192^3 FP64 (MEASURED_PEAKS.json has no FP64 entry)",
            "traffic": traffic_from_profile(cfg, "gemm_dmma"),
            "hbm_gbs_algorithmic": by_g / (ms_g * 1e-3) / 1e9 if ms_g > 0 else 0.0,
            "launches_per_sweep": n_g, "avg_launch_us": 1e3 * ms_g / max(n_g, 1),
            "flops_per_launch": fl_g / max(n_g, 1),
            "sweep_breakdown_ms": {k: round(v[1], 3) for k, v in fam.items()}}


def roofline_tcgen05(fam, peaks, cfg):
    """3xTF32 tcgen05 products with their split pass: the dominant shape (the
    rSVD range finder, 2592 x 82 x 2592 at c3) has 55 issued flop/B, below
    the TF32 ridge (~107), so the binding roof is HBM; the tensor-pipe
    fraction is reported beside it."""
    n_g, ms_g, fl_g, by_g = fam["gemm_tcgen05"]
    hbm = peaks.get("hbm_gbs", 6650.0)
    tf32 = peaks.get("bf16_tflops_sustained", 1411.5) / 2.0
    gbs = by_g / (ms_g * 1e-3) / 1e9 if ms_g > 0 else 0.0
    issued = 3.0 * fl_g / (ms_g * 1e-3) / 1e12 if ms_g > 0 else 0.0
    return {"bound": "hbm", "kernel": "gemm_tma_kernel (tcgen05 kind::tf32, 3 products) + split_pack_kernel",
            "achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm if hbm else None,
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)",
            "tensor_tflops_issued": issued, "tensor_peak": tf32, "tensor_frac": issued / tf32,
            "traffic": traffic_from_profile(cfg, "gemm_tcgen05"),
            "launches_per_sweep": n_g, "avg_launch_us": 1e3 * ms_g / max(n_g, 1),
            "sweep_breakdown_ms": {k: round(v[1], 3) for k, v in fam.items()}}


def run_ours(args, rank, world, local_rank):
    import torch
    from tenes_b200.env import kernel_launch_count
    device = local_rank
    torch.cuda.set_device(device)
    cfg = args.config
    kit = CONFIGS[cfg]["model"] == "kitaev"
    T, su_rate = prepare_tensors(cfg, SEED + rank, device, args.su_steps)
    su = {} if kit else {cfg: {"gpu_steps_per_s": su_rate}}
    if not args.quick and cfg != "c1":
        su["c1"] = {"gpu_steps_per_s": su_rate_gpu("c1", SEED + rank, device)}
    env = env_for(cfg, T, device, args.projector, args.precision)
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
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize(device)
    clocks = Clocks(device)
    clocks.start()
    l0 = kernel_launch_count()
    times = timed_sweeps(env, args.steps, 0, stream, flush)
    launches = kernel_launch_count() - l0
    torch.cuda.synchronize(device)
    ck = clocks.stop()
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

    # ---- roofline of this arm's dominant product family (one instrumented sweep)
    fam = sweep_profile(env)
    env.close()
    peaks = measured_peaks()
    dgemm = fp64_peak_tflops(device)
    if args.precision == "mixed":
        roof = roofline_tcgen05(fam, peaks, cfg)
    else:
        roof = roofline_fp64(fam, dgemm, cfg)

    # ---- the other arms from the same tensors (device-timed sweeps, same flush)
    arms = {}
    if not args.quick:
        for tag, proj, prec, k in (("mixed_rsvd", "rsvd", "mixed", args.steps), ("fp64_rsvd", "rsvd", "fp64",
                                   args.steps), ("fp64_full_svd", "svd", "fp64", min(args.steps, 3))):
            if kit and prec == "mixed":
                continue  # the tensor-core form takes real tensors only
            if proj == args.projector and prec == args.precision:
                arms[tag] = {"sweeps_per_s": value / world, "ms_per_sweep": ms_per_step, "headline": True}
                continue
            e2 = env_for(cfg, T, device, proj, prec)
            st2 = torch.cuda.ExternalStream(e2.stream_handle(), device=device)
            tt = timed_sweeps(e2, k, 3 if proj == "rsvd" else 1, st2, flush)
            f2 = sweep_profile(e2)
            e2.close()
            arms[tag] = {"sweeps_per_s": 1e3 * len(tt) / sum(tt), "ms_per_sweep": sum(tt) / len(tt),
                         "sweeps_timed": len(tt),
                         "roofline": roofline_tcgen05(f2, peaks, cfg) if prec == "mixed"
                         else roofline_fp64(f2, dgemm, cfg)}
        if "mixed_rsvd" in arms and "fp64_rsvd" in arms:
            arms["speedup_mixed_vs_fp64_same_projector"] = (arms["mixed_rsvd"]["sweeps_per_s"]
                                                            / arms["fp64_rsvd"]["sweeps_per_s"])

    # ---- time to a converged environment: mixed and FP64 at the same projector, and FP64 full SVD
    conv = None
    if args.converge != "none" and kit:
        conv = {"criterion": f"{CONFIGS[cfg]['sweeps']} sweeps from the initial environment (fixed count)",
                "fp64_rsvd": kitaev_run(cfg, T, device, "rsvd")}
        if args.converge == "full":
            conv["fp64_full_svd"] = kitaev_run(cfg, T, device, "svd")
    elif args.converge != "none":
        conv = {"criterion": "|E/site(sweep t) - E/site(sweep t-1)| <= 1e-7 (energy evaluations timed too)"}
        conv["mixed_rsvd"] = converge(cfg, T, device, "rsvd", "mixed")
        conv["fp64_rsvd"] = converge(cfg, T, device, "rsvd", "fp64")
        if args.converge == "full":
            conv["fp64_full_svd"] = converge(cfg, T, device, "svd", "fp64", max_sweeps=30)
        conv["speedup_mixed_vs_fp64_rsvd"] = conv["fp64_rsvd"]["seconds"] / conv["mixed_rsvd"]["seconds"]
        conv["speedup_mixed_vs_fp64_full_svd"] = (conv["fp64_full_svd"]["seconds"] / conv["mixed_rsvd"]["seconds"]
                                                  if "fp64_full_svd" in conv else None)
        conv["abs_delta_e_mixed_vs_fp64_rsvd"] = abs(conv["mixed_rsvd"]["energy_per_site"]
                                                     - conv["fp64_rsvd"]["energy_per_site"])
    return {"value": value, "ms_per_step": ms_per_step, "e2e": e2e, "roofline": roof, "arms": arms,
            "clocks": ck, "gpu_launches": launches, "sweep_ms": [round(t, 3) for t in times],
            "converge": conv, "tensors": T, "simple_update": su}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


# -------------------------------------------------------- CPU oracle (reference arm)
def oracle_lattice(cfg):
    from oracle import tenes_oracle as O
    LX, LY, pd, vd, dirs, noises, _ = cell(cfg)
    lat = O.Lattice(LX, LY)
    lat.physical_dims = pd
    lat.virtual_dims = vd
    lat.initial_dirs = dirs
    lat.noises = noises
    return lat


def oracle_params(cfg, projector="rsvd"):
    from oracle import tenes_oracle as O
    chi = CONFIGS[cfg]["chi"]
    if projector == "rsvd":
        return O.Params(CHI=chi, Use_RSVD=True, rsvd_oversample_abs=RSVD_OVERSAMPLE, rsvd_power_iters=RSVD_POWER)
    return O.Params(CHI=chi)


def oracle_tensors(cfg, seed):
    """The workload's site tensors by the CPU oracle: its own seeded start and
    simple update (the same algorithm as the library's)."""
    from oracle import tenes_oracle as O
    c = CONFIGS[cfg]
    D = c["D"]
    lat = oracle_lattice(cfg)
    if c["model"] == "kitaev":
        return lat, random_complex_tensors(lat.virtual_dims, seed)
    Tn = O.initialize_tensors(lat, seed, True) if c["model"] == "afh" else uniform_tensors(D, seed)
    lam = [[np.ones(D) for _ in range(4)] for _ in range(lat.N_UNIT)]
    p = O.Params()
    op, op1 = su_ops(cfg)
    for _ in range(c["su_steps"]):
        for (s, leg) in bonds(lat.LX, lat.LY):
            tg = lat.neighbor(s, leg)
            a, b, lc = O.simple_update_bond(Tn[s], Tn[tg], lam[s], lam[tg], op, leg, p)
            lam[s][leg] = lc
            lam[tg][(leg + 2) % 4] = lc
            Tn[s], Tn[tg] = a, b
        if op1 is not None:
            for s in range(lat.N_UNIT):
                Tn[s] = np.tensordot(Tn[s], op1, ([4], [0]))
    return lat, Tn


def oracle_moves(lat):
    """The moves of one sweep in the order of ctm.cpp:1205-1228 (as O.sweep)."""
    from oracle import tenes_oracle as O
    LX, LY = lat.LX_noskew, lat.LY_noskew
    mv = [(O.left_move, ix) for ix in range(LX)]
    mv += [(O.right_move, (ix + 1 + LX) % LX) for ix in range(0, -LX, -1)]
    mv += [(O.top_move, (iy + 1 + LY) % LY) for iy in range(0, -LY, -1)]
    mv += [(O.bottom_move, iy) for iy in range(LY)]
    return mv


def oracle_kitaev(oe, Tn, lat):
    """Energy per site and mean plaquette flux of the oracle's environment
    (the same terms and windows as kitaev_observables)."""
    from oracle import tenes_oracle as O
    S = spin_half()
    one = np.einsum("ac,bd->abcd", np.eye(2), np.eye(2))
    tot = 0.0
    for (s, dx, dy, a) in kitaev_bond_list(lat.virtual_dims):
        h = -np.einsum("ac,bd->abcd", S[a], S[a])
        if dy == 0:
            l, r = s, lat.other(s, 1, 0)
            arg = (oe.C1[l], oe.C2[r], oe.C3[r], oe.C4[l], oe.eTt[l], oe.eTt[r], oe.eTr[r], oe.eTb[r], oe.eTb[l],
                   oe.eTl[l], Tn[l], Tn[r])
            tot += (O.contract_two_sites_horizontal_op12(*arg, h)
                    / O.contract_two_sites_horizontal_op12(*arg, one)).real
        else:
            t, b = lat.other(s, 0, 1), s
            arg = (oe.C1[t], oe.C2[t], oe.C3[b], oe.C4[b], oe.eTt[t], oe.eTr[t], oe.eTr[b], oe.eTb[b], oe.eTl[b],
                   oe.eTl[t], Tn[t], Tn[b])
            tot += (O.contract_two_sites_vertical_op12(*arg, h.transpose(1, 0, 3, 2))
                    / O.contract_two_sites_vertical_op12(*arg, one)).real
    f = S[0] + S[1] + S[2]
    for i in range(lat.N_UNIT):
        a = (oe.C1[i], oe.C2[i], oe.C3[i], oe.C4[i], oe.eTt[i], oe.eTr[i], oe.eTb[i], oe.eTl[i], Tn[i])
        tot -= KITAEV_H * (O.contract_one_site(*a, f) / O.contract_one_site(*a, np.eye(2))).real
    starts, ops = hexagons()
    flux = []
    for s in starts:
        _, Cs, eTt, eTr, eTb, eTl, T = O._window(oe, Tn, lat, s, 0, 1, 2, 3)
        grid = [[ops.get((r, c), np.eye(2)) for c in range(3)] for r in range(2)]
        flux.append((O.contract_window(Cs, eTt, eTr, eTb, eTl, T, grid)
                     / O.contract_window(Cs, eTt, eTr, eTb, eTl, T, [[np.eye(2)] * 3 for _ in range(2)])).real)
    return tot / lat.N_UNIT, float(np.mean(flux))


def oracle_energy(cfg, oe, Tn, lat):
    """Energy per site of the oracle's environment (op12 contractions / norm,
    twosite_obs.cpp; the Ising field through the one-site contraction)."""
    from oracle import tenes_oracle as O
    if CONFIGS[cfg]["model"] == "kitaev":
        return oracle_kitaev(oe, Tn, lat)[0]
    h = bond_hamiltonian(cfg)
    one = np.einsum("ac,bd->abcd", np.eye(2), np.eye(2))
    tot = 0.0
    for i in range(lat.N_UNIT):
        j = lat.right(i)
        a = (oe.C1[i], oe.C2[j], oe.C3[j], oe.C4[i], oe.eTt[i], oe.eTt[j], oe.eTr[j], oe.eTb[j], oe.eTb[i],
             oe.eTl[i], Tn[i], Tn[j])
        tot += (O.contract_two_sites_horizontal_op12(*a, h) / O.contract_two_sites_horizontal_op12(*a, one)).real
        j = lat.top(i)
        a = (oe.C1[j], oe.C2[j], oe.C3[i], oe.C4[i], oe.eTt[j], oe.eTr[j], oe.eTr[i], oe.eTb[i], oe.eTl[i],
             oe.eTl[j], Tn[j], Tn[i])
        tot += (O.contract_two_sites_vertical_op12(*a, h) / O.contract_two_sites_vertical_op12(*a, one)).real
    if CONFIGS[cfg]["model"] == "tfi":
        sx = np.array([[0.0, 0.5], [0.5, 0.0]])
        for i in range(lat.N_UNIT):
            a = (oe.C1[i], oe.C2[i], oe.C3[i], oe.C4[i], oe.eTt[i], oe.eTr[i], oe.eTb[i], oe.eTl[i], Tn[i])
            tot -= HX * (O.contract_one_site(*a, sx) / O.contract_one_site(*a, np.eye(2))).real
    return tot / lat.N_UNIT


def oracle_check(cfg, T, sweeps):
    """The FP64 CPU oracle with the headline's projectors (rSVD, k = chi+10,
    q = 2) from the GPU's own site tensors: `sweeps` sweeps, each move timed
    (the first sweep is the CPU baseline sample), then the energy per site."""
    from oracle import tenes_oracle as O
    lat = oracle_lattice(cfg)
    p = oracle_params(cfg)
    oe = O.init_env(T, p, lat)
    move_s = []
    for _ in range(sweeps):
        for fn, line in oracle_moves(lat):
            t0 = time.perf_counter()
            fn(oe, T, line, p, lat)
            move_s.append(time.perf_counter() - t0)
    if CONFIGS[cfg]["model"] == "kitaev":
        e, w = oracle_kitaev(oe, T, lat)
        return move_s, e, w
    return move_s, oracle_energy(cfg, oe, T, lat), None


def data_note(cfg):
    if CONFIGS[cfg]["model"] == "kitaev":
        return "synthetic (site tensors with i.i.d. uniform[-1, 1] real and imaginary parts, seeded)"
    return "synthetic (seeded simple-update tensors of the workload's shapes)"


def config_block(args, world):
    """The `config` object, identical in both arms for the same flags."""
    c = CONFIGS[args.config]
    kit = c["model"] == "kitaev"
    return {"workload": f"{c['name']}_{args.precision}_{args.projector}", "precision": args.precision,
            "D": "per bond from {3, 4, 5}, seeded; one vertical leg of 1 per site" if kit else c["D"],
            "chi": c["chi"], "unit_cell": "4x4" if kit else "2x2", "su_steps": c["su_steps"],
            "tensors": "complex128" if kit else "float64",
            "projector": ("full SVD (reference default)" if args.projector == "svd"
                          else f"rSVD k=chi+{RSVD_OVERSAMPLE}, q={RSVD_POWER}"),
            "parallelism": f"replicas{world}",
            "l2": "GPU arm: flushed between timed sweeps (252 MB write outside the timed window)"}


def run_reference(args, rank, world):
    """The reference arm: the FP64 CPU oracle (numpy, all host cores through
    BLAS/LAPACK) on the same workload and projectors.  Each step is one move;
    the steps walk through the moves of consecutive sweeps in the order of
    ctm.cpp:1205-1228, so every move of a sweep is timed and the sweeps/s is
    (steps / moves per sweep) / time."""
    if rank != 0:
        return None
    from oracle import tenes_oracle as O
    lat, Tn = oracle_tensors(args.config, SEED)
    p = oracle_params(args.config, args.projector)
    env = O.init_env(Tn, p, lat)
    moves = oracle_moves(lat)
    k = 0
    for _ in range(args.warmup):
        fn, line = moves[k % len(moves)]
        fn(env, Tn, line, p, lat)
        k += 1
    tot = 0.0
    for _ in range(args.steps):
        fn, line = moves[k % len(moves)]
        t0 = time.perf_counter()
        fn(env, Tn, line, p, lat)
        tot += time.perf_counter() - t0
        k += 1
    v = (args.steps / len(moves)) / tot
    cores = os.cpu_count()
    return {"metric": "ctmrg_sweeps_per_s", "value": v, "unit": "sweeps/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": data_note(args.config), "impl": "reference",
            "config": config_block(args, world),
            "step": f"one CTMRG move (1/{len(moves)} of a sweep), moves of consecutive sweeps in sweep order",
            "cpu_baseline": {"value": v, "unit": "sweeps/s", "cores": cores, "kind": "port",
                             "sample": f"{args.steps} consecutive moves of the FP64 CPU oracle "
                                       f"({args.steps / len(moves):.2f} sweeps) after {args.warmup} warm-up moves"},
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


def fd_summary(fds, h, gmax):
    """Central differences against the adjoint on the seeded entries: the
    relative error of each entry (no floor), the absolute error, and how many
    entries meet 1e-6 relative."""
    if not fds:
        return {"entries": 0}
    rel = [abs(f - g) / max(abs(f), abs(g), 1e-300) for f, g in fds]
    ab = [abs(f - g) for f, g in fds]
    return {"entries": len(fds), "step": h, "max_rel_err": max(rel), "median_rel_err": float(np.median(rel)),
            "entries_within_1e-6_rel": sum(r <= 1e-6 for r in rel), "max_abs_err": max(ab),
            "max_abs_grad": gmax, "min_abs_grad_checked": min(abs(g) for _, g in fds),
            "pairs_fd_adjoint": fds}


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
    fds, h = [], GRAD["fd_step"]
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
        fds.append((float(fd), float(g[site][idx])))
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
            "fd_check": fd_summary(fds, h, gmax),
            "mixed": {"value": 1.0 / medm, "unit": "evals/s", "energy_per_site": Em,
                      "abs_delta_e": abs(Em - E),
                      "grad_rel_err": float(np.linalg.norm(gmv - gv) / np.linalg.norm(gv))}}


# iTPO workload (finite temperature, ctm_single.cpp): TFI on the square
# lattice, bond -SzSz, field -hx Sx on the bonds' sites, density operator of
# a 2x2 cell from the identity at beta = 0 through FT["su_steps"] density
# simple-update steps at tau (beta = 2 tau per step).
FT = dict(D=8, chi=64, su_steps=200, tau=0.01, hx=1.0)


def ft_problem():
    """(lattice spec, Trotter step as (source, leg, op) triples, bond
    Hamiltonian) of the iTPO workload."""
    from tenes_b200.std_ops import evolution_onesite, evolution_twosite, ising_bond, real_if_close, spin_ops
    _, Sx, _ = spin_ops(0.5)
    op = real_if_close(evolution_twosite(ising_bond(1.0), FT["tau"]))
    op1 = real_if_close(evolution_onesite(-FT["hx"] * Sx, FT["tau"]))
    step = [(s, leg, op) for (s, leg) in bonds(2, 2)] + [(s, -1, op1) for s in range(4)]
    h = real_if_close(ising_bond(1.0))
    return step, h, Sx


def ft_env(device, T=None):
    from tenes_b200.env import CTMParams, Environment
    p = CTMParams(chi=FT["chi"], max_ctm_iteration=1, density=True)
    env = Environment(2, 2, [2] * 4, [[FT["D"]] * 4] * 4, p, False, device=device)
    if T is None:
        env.init_tensors(SEED, [[0.0]] * 4, [0.0] * 4)
    else:
        for i, t in enumerate(T):
            env.set_site_tensor(i, t)
    return env


def ft_energy(env, h, Sx):
    """E/site = <bond terms> + <-hx Sx> through the density contractions."""
    ident = np.einsum("ac,bd->abcd", np.eye(2), np.eye(2))
    e = 0.0
    for s in range(4):
        for dx, dy in ((1, 0), (0, 1)):
            e += (env.contract_bond_op12(s, dx, dy, h) / env.contract_bond_op12(s, dx, dy, ident)).real
        e -= FT["hx"] * (env.contract_one_site(s, Sx) / env.contract_one_site(s, np.eye(2))).real
    return e / 4


def run_ft(args):
    """Single-layer (iTPO) CTMRG sweeps/s at D=8, chi=64 with the
    reference-default full-SVD corner projectors, the density simple update's
    steps/s, the energy per site against the oracle, and the whole
    FT_TFI_square run (500 steps, 6 measurements) end to end through the
    front end."""
    import torch
    from oracle import tenes_density as Dn
    from oracle import tenes_oracle as O
    from tenes_b200.env import kernel_launch_count
    device = 0
    step, h, Sx = ft_problem()
    env = ft_env(device)
    t0 = time.perf_counter()
    for _ in range(FT["su_steps"]):
        env.simple_update_many(step)
    env.sync()
    su_s = time.perf_counter() - t0
    T = [env.get_site_tensor(i) for i in range(4)]
    env.init_env()
    stream = torch.cuda.ExternalStream(env.stream_handle())
    flush = torch.empty(int(256e6) // 4, dtype=torch.float32, device=f"cuda:{device}")
    l0 = kernel_launch_count()
    times = timed_sweeps(env, args.steps, args.warmup, stream, flush)
    launches = (kernel_launch_count() - l0) // max(args.steps + args.warmup, 1)
    n_sw = args.warmup + args.steps
    e_gpu = ft_energy(env, h, Sx)
    env.close()
    # the oracle: same tensors, the same number of sweeps; the first sweep is the CPU sample
    lat = O.Lattice(2, 2)
    lat.physical_dims = [2] * 4
    lat.virtual_dims = [[FT["D"]] * 4] * 4
    p = O.Params(CHI=FT["chi"], Max_CTM_Iteration=1)
    Ts = [Dn.single_tensor(t) for t in T]
    oe = Dn.init_env(Ts, lat)
    sw = []
    for _ in range(n_sw):
        t1 = time.perf_counter()
        Dn.sweep(oe, Ts, p, lat)
        sw.append(time.perf_counter() - t1)
    ident = np.einsum("ac,bd->abcd", np.eye(2), np.eye(2))
    e_or = 0.0
    for s in range(4):
        for dx, dy in ((1, 0), (0, 1)):
            e_or += (Dn.contract_op12(oe, T, lat, s, dx, dy, h) / Dn.contract_op12(oe, T, lat, s, dx, dy, ident)).real
        e = oe
        n1 = Dn.contract_one_site(e.C1[s], e.C2[s], e.C3[s], e.C4[s], e.eTt[s], e.eTr[s], e.eTb[s], e.eTl[s], T[s],
                                  np.eye(2))
        v1 = Dn.contract_one_site(e.C1[s], e.C2[s], e.C3[s], e.C4[s], e.eTt[s], e.eTr[s], e.eTb[s], e.eTl[s], T[s],
                                  Sx)
        e_or -= FT["hx"] * (v1 / n1).real
    e_or /= 4
    # density simple update on the CPU oracle: a sample of the same steps
    Tn_o = [t.copy() for t in T]
    lam = [[np.ones(FT["D"]) for _ in range(4)] for _ in range(4)]

    class Up:
        def __init__(self, s, l, o):
            self.source_site, self.source_leg, self.op = s, l, o

        def is_onesite(self):
            return self.source_leg < 0
    ups = [Up(s, l, o) for (s, l, o) in step]
    n_cpu = 5
    t1 = time.perf_counter()
    for _ in range(n_cpu):
        for up in ups:
            Dn.su_density(Tn_o, lam, lat, up, p)
    su_cpu = n_cpu / (time.perf_counter() - t1)
    # the reference's own FT_TFI_square input end to end, GPU front end and the oracle driver
    import shutil
    import tenes_b200.itps as itps
    from tests import _ft  # noqa: F401 -- the oracle's driver loop
    with tempfile.TemporaryDirectory() as td:
        shutil.copyfile(os.path.join(ROOT, "tests", "golden", "ft_tfi_square_input.toml"),
                        os.path.join(td, "in.toml"))
        t1 = time.perf_counter()
        itps.run(os.path.join(td, "in.toml"), print_level=0, outdir=os.path.join(td, "out"))
        run_gpu = time.perf_counter() - t1
    t1 = time.perf_counter()
    _ft.run("ft_tfi_square", lambda beta, inp, lat_, p_, one, two, multi, Tn: _ft.measure(inp, lat_, p_, one, two,
                                                                                            multi, Tn))
    run_cpu = time.perf_counter() - t1
    med = float(np.median(times))
    return {"metric": "itpo_ctmrg_sweeps_per_s", "value": 1e3 / med, "unit": "sweeps/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": med, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (the density operator after the seeded finite-temperature simple update)",
            "config": {"workload": f"itpo_tfi_square_2x2_D{FT['D']}_chi{FT['chi']}_beta{2 * FT['tau'] * FT['su_steps']:g}",
                       "projector": "full SVD corner (reference default)",
                       "l2": "flushed between timed sweeps (256 MB write outside the timed window)"},
            "sweep_ms": [round(t, 3) for t in times], "gpu_launches": int(launches),
            "cpu_baseline": {"value": 1.0 / sw[0], "unit": "sweeps/s", "cores": os.cpu_count(), "kind": "port",
                             "sample": "the first of the oracle's single-layer sweeps from the same tensors"},
            "energy_per_site": e_gpu, "oracle_energy_per_site": e_or, "abs_delta_e": abs(e_gpu - e_or),
            "sweeps_compared": n_sw,
            "density_simple_update": {"gpu_steps_per_s": FT["su_steps"] / su_s, "cpu_oracle_steps_per_s": su_cpu,
                                      "step": "8 bond + 4 one-site density updates (kron(op, conj(op)))"},
            "ft_tfi_square_run": {"gpu_seconds": run_gpu, "cpu_oracle_seconds": run_cpu,
                                  "what": "the reference's FT_TFI_square input: 500 density simple-update steps "
                                          "and 6 measurements (CTMRG chi=10, observables, correlations, "
                                          "correlation length)"}}


def run_gemm(spec):
    """One contraction kernel alone, through tg_bench_gemm: spec = M N K
    [layout] [prec] [iters]; layout 0: A row-major (M, K), B row-major (K, N);
    1: B column-major (the rSVD panel products); prec 0: FP64 DMMA, 1: 3xTF32
    on tcgen05.  Prints the average device time of one product and its
    algorithmic rate (2 M N K flop)."""
    import ctypes as C
    from tenes_b200 import _lib
    a = [int(x) for x in spec]
    M, N, K = a[:3]
    layout = a[3] if len(a) > 3 else 0
    prec = a[4] if len(a) > 4 else 0
    iters = a[5] if len(a) > 5 else 10
    lib = _lib.load()
    ms = C.c_double()
    _lib.check(lib.tg_bench_gemm(M, N, K, layout, prec, iters, C.byref(ms)))
    tf = 2.0 * M * N * K / (ms.value * 1e-3) / 1e12
    print(f"M={M} N={N} K={K} layout={layout} prec={prec}: {ms.value * 1e3:.1f} us  {tf:.1f} TFLOP/s", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c3", choices=sorted(CONFIGS))
    ap.add_argument("--projector", default="rsvd", choices=["svd", "rsvd"],
                    help="svd: full SVD (reference default); rsvd: k = chi+10, 2 power iterations")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="mixed: 3xTF32 tcgen05 contractions, FP64 projector algebra")
    ap.add_argument("--converge", default="full", choices=["full", "fast", "none"],
                    help="time-to-converge arms: full = mixed rSVD, FP64 rSVD and FP64 full SVD; "
                         "fast = without the FP64 full-SVD arm")
    ap.add_argument("--quick", action="store_true", help="headline and e2e only (no other arms)")
    ap.add_argument("--su-steps", type=int, default=None,
                    help="override the simple-update steps that prepare the tensors (profiling runs)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-sweep", action="store_true",
                    help="wrap one extra sweep in cudaProfilerStart/Stop (for ncu)")
    ap.add_argument("--grad", action="store_true",
                    help="gradient evaluations/s of the J1-J2 energy (D=3, chi=36) with the FD check")
    ap.add_argument("--grad-iters", type=int, default=GRAD["iterations"])
    ap.add_argument("--grad-fd", type=int, default=32, help="entries checked by central differences")
    ap.add_argument("--ft", action="store_true",
                    help="iTPO (finite temperature): single-layer CTMRG sweeps/s at D=8, chi=64, the density "
                         "simple update and the FT_TFI_square run")
    ap.add_argument("--gemm", nargs="+", metavar="M N K [layout prec iters]",
                    help="time one contraction kernel alone (tg_bench_gemm) and exit")
    args = ap.parse_args()
    if args.gemm:
        run_gemm(args.gemm)
        return
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    if args.grad:
        print(json.dumps(run_grad(args)), flush=True)
        return
    if args.ft:
        print(json.dumps(run_ft(args)), flush=True)
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
        c = CONFIGS[args.config]
        cpu = None
        oracle = None
        if not args.no_cpu_baseline:
            # The oracle from the GPU's own site tensors, as many sweeps as the
            # FP64 rSVD arm took to converge: its first sweep is the CPU
            # baseline sample, its energy pins every arm's energy.
            n_sw = res["converge"]["fp64_rsvd"]["sweeps"] if res["converge"] else 1
            move_s, e_or, w_or = oracle_check(args.config, res["tensors"], n_sw)
            per = len(oracle_moves(oracle_lattice(args.config)))
            first = sum(move_s[:per])
            cpu = {"value": 1.0 / first, "unit": "sweeps/s", "cores": os.cpu_count(), "kind": "port",
                   "sample": f"the first of {n_sw} consecutive sweeps ({per} moves) of the FP64 CPU oracle with "
                             f"the same projectors (rSVD k=chi+{RSVD_OVERSAMPLE}, q={RSVD_POWER}) from the same "
                             "site tensors"}
            oracle = {"sweeps": n_sw, "energy_per_site": e_or, "seconds_per_sweep": sum(move_s) / n_sw}
            if w_or is not None and res["converge"]:
                arm = res["converge"]["fp64_rsvd"]
                oracle["plaquette_flux"] = w_or
                oracle["abs_delta_e_fp64_rsvd"] = abs(arm["energy_per_site"] - e_or)
                oracle["abs_delta_flux_fp64_rsvd"] = abs(arm["plaquette_flux"] - w_or)
            elif res["converge"]:
                for tag in ("mixed_rsvd", "fp64_rsvd", "fp64_full_svd"):
                    arm = res["converge"].get(tag)
                    if arm and len(arm["energy_per_sweep"]) >= n_sw:
                        oracle[f"abs_delta_e_{tag}_at_sweep_{n_sw}"] = abs(arm["energy_per_sweep"][n_sw - 1] - e_or)
        line = {"metric": "ctmrg_sweeps_per_s", "value": res["value"], "unit": "sweeps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if args.precision == "fp64" else "tf32x3+f64",
                "data": data_note(args.config),
                "config": config_block(args, world),
                "roofline": res["roofline"], "cpu_baseline": cpu, "e2e": res["e2e"],
                "clocks": res["clocks"], "gpu_launches": res["gpu_launches"], "sweep_ms": res["sweep_ms"]}
        if res["arms"]:
            line["arms"] = res["arms"]
        if res["converge"] is not None:
            line["time_to_converge"] = res["converge"]
        if oracle is not None:
            line["fp64_oracle_check"] = oracle
        su = res["simple_update"]
        if not args.no_cpu_baseline and su:
            for c in su:
                # a bounded CPU sample: 1000 bond updates or so
                n = max(2, 1000 // (2 * 4 + (4 if CONFIGS[c]["model"] == "tfi" else 0)))
                su[c]["cpu_oracle_steps_per_s"] = su_rate_oracle(c, SEED, n)
                su[c]["cpu_oracle_sample_steps"] = n
                if su[c]["gpu_steps_per_s"]:
                    su[c]["speedup_gpu_vs_cpu_oracle"] = su[c]["gpu_steps_per_s"] / su[c]["cpu_oracle_steps_per_s"]
        if su:
            line["simple_update"] = {"step": "every bond of the 2x2 cell once (8 bond updates; the Ising workload also "
                                             "applies its 4 one-site field operators), tau = 0.01",
                                     "cpu_cores": os.cpu_count(), **su}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
