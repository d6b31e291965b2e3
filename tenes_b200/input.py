"""Reader for TeNeS's expert-format ``input.toml``.

Mirrors the keys, defaults and error behaviour of the reference loader
(src/iTPS/load_toml.cpp:247-662, defaults src/iTPS/PEPS_Parameters.cpp:30-77,
transfer-matrix defaults src/iTPS/transfer_matrix.hpp:38-45).  Produces plain
Python / numpy structures; nothing here touches the GPU.
"""

from __future__ import annotations

import tomllib
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np


class InputError(ValueError):
    """Malformed input file (tenes::input_error, src/exception.hpp:22-34)."""


@dataclass
class PEPSParameters:
    """PEPS_Parameters with the reference defaults (PEPS_Parameters.cpp:30-77)."""
    CHI: int = 2
    num_simple_step: List[int] = field(default_factory=lambda: [0])
    tau_simple_step: List[float] = field(default_factory=lambda: [0.0])
    measure_interval: List[int] = field(default_factory=lambda: [10])
    Inverse_lambda_cut: float = 1e-12
    Simple_Gauge_Fix: bool = False
    Simple_Gauge_maxiter: int = 100
    Simple_Gauge_Convergence_Epsilon: float = 1e-2
    Inverse_projector_cut: float = 1e-12
    CTM_Convergence_Epsilon: float = 1e-6
    Max_CTM_Iteration: int = 100
    CTM_Projector_corner: bool = True
    Use_RSVD: bool = False
    RSVD_Oversampling_factor: float = 2.0
    MeanField_Env: bool = False
    num_full_step: List[int] = field(default_factory=lambda: [0])
    tau_full_step: List[float] = field(default_factory=lambda: [0.0])
    Inverse_Env_cut: float = 1e-12
    Full_Inverse_precision: float = 1e-12
    Full_Convergence_Epsilon: float = 1e-6
    Full_max_iteration: int = 100
    Full_Gauge_Fix: bool = True
    Full_Use_FastFullUpdate: bool = True
    seed: int = 11
    is_real: bool = False
    iszero_tol: float = 0.0
    to_measure: bool = True
    outdir: str = "output"
    tensor_load_dir: str = ""
    tensor_save_dir: str = ""
    calcmode: str = "ground_state"  # ground_state | time_evolution | finite_temperature


@dataclass
class TransferMatrixParameters:
    """TransferMatrix_Parameters defaults (transfer_matrix.hpp:29-47)."""
    to_calculate: bool = True
    num_eigvals: int = 4
    maxdim_dense_eigensolver: int = 200
    arnoldi_maxdim: int = 50
    arnoldi_restartdim: int = 20
    arnoldi_maxiter: int = 1
    arnoldi_rtol: float = 1e-10


@dataclass
class CorrelationParameters:
    """[correlation] (CorrelationParameter, correlation_function.hpp:33-39;
    gen_corparam, load_toml.cpp:298-314): r_max and (left, right) one-site
    operator groups."""
    r_max: int = 0
    operators: List[Tuple[int, int]] = field(default_factory=list)


@dataclass
class LatticeSpec:
    """[tensor] section (load_toml.cpp:247-296)."""
    LX: int
    LY: int
    skew: int
    physical_dims: List[int]
    virtual_dims: List[List[int]]
    initial_dirs: List[List[float]]
    noises: List[float]

    def neighbors(self) -> List[List[int]]:
        """Neighbour table [left, top, right, bottom] of every site, skew
        boundary included (SquareLattice::calc_neighbors, SquareLattice.cpp:48-90)."""
        LX, LY, N = self.LX, self.LY, self.LX * self.LY
        nn = [[(ix - 1) % LX + iy * LX, ix + ((iy + 1) % LY) * LX, (ix + 1) % LX + iy * LX,
               ix + ((iy - 1) % LY) * LX] for iy in range(LY) for ix in range(LX)]
        skew = int(np.fmod(self.skew, LX))
        if skew != 0:
            for ix in range(LX):
                nn[ix][3] = int(np.fmod(ix + LX + skew, LX)) + (LY - 1) * LX
                nn[N + ix - LX][1] = int(np.fmod(ix + LX - skew, LX))
        return nn

    def other(self, i: int, dx: int, dy: int) -> int:
        """Site reached from i by dx steps right and dy steps up
        (SquareLattice::other, SquareLattice.cpp:116-137)."""
        nn = self.neighbors()
        for _ in range(abs(dx)):
            i = nn[i][2 if dx > 0 else 0]
        for _ in range(abs(dy)):
            i = nn[i][1 if dy > 0 else 3]
        return i


@dataclass
class Operator:
    """An observable (src/operator.hpp:26-169)."""
    name: str
    group: int
    source_site: int
    dx: List[int]
    dy: List[int]
    op: Optional[np.ndarray]
    ops_indices: List[int]
    coeff: complex


@dataclass
class EvolutionOperator:
    """exp(-tau H) piece (src/operator.hpp:174-192); source_leg < 0 = one-site."""
    source_site: int
    source_leg: int
    group: int
    op: np.ndarray

    def is_onesite(self) -> bool:
        return self.source_leg < 0


@dataclass
class Input:
    params: PEPSParameters
    lattice: LatticeSpec
    simple_updates: List[EvolutionOperator]
    full_updates: List[EvolutionOperator]
    onesite: List[Operator]
    twosite: List[Operator]
    multisite: List[Operator]
    tm_params: TransferMatrixParameters
    is_real: bool
    corparam: CorrelationParameters = field(default_factory=CorrelationParameters)


def _drop_comment(line: str) -> str:
    i = line.find("#")
    return line if i < 0 else line[:i]


def read_tensor(text: str, shape: Sequence[int], atol: float = 0.0) -> np.ndarray:
    """util::read_tensor (src/util/read_tensor.hpp:35-86): each line holds
    rank integer indices followed by the real and imaginary part."""
    A = np.zeros(tuple(shape), dtype=np.complex128)
    rank = len(shape)
    for raw in text.splitlines():
        fields = _drop_comment(raw).split()
        if not fields:
            continue
        if len(fields) != rank + 2:
            raise InputError("cannot parse tensor; the number of columns differs from tensor rank + 2")
        idx = tuple(int(f) for f in fields[:rank])
        re = float(fields[rank])
        im = float(fields[rank + 1])
        re = re if abs(re) >= atol else 0.0
        im = im if abs(im) >= atol else 0.0
        A[idx] = complex(re, im)
    return A


def _get(d, key, default=None):
    return d.get(key, default) if isinstance(d, dict) else default


def _as_list(v, conv):
    if isinstance(v, list):
        return [conv(x) for x in v]
    return [conv(v)]


def gen_param(param: dict) -> PEPSParameters:
    """gen_param (load_toml.cpp:330-407)."""
    p = PEPSParameters()
    g = param.get("general")
    if g is not None:
        p.is_real = bool(g.get("is_real", p.is_real))
        p.iszero_tol = float(g.get("iszero_tol", p.iszero_tol))
        p.to_measure = bool(g.get("measure", p.to_measure))
        p.outdir = str(g.get("output", p.outdir))
        p.tensor_load_dir = str(g.get("tensor_load", p.tensor_load_dir))
        p.tensor_save_dir = str(g.get("tensor_save", p.tensor_save_dir))
        mode = str(g.get("mode", "ground state"))
        if mode.startswith("ground"):
            p.calcmode = "ground_state"
        elif mode.startswith("time"):
            p.calcmode = "time_evolution"
        elif mode.startswith("finite"):
            p.calcmode = "finite_temperature"
        else:
            raise InputError("Invalid mode: " + mode)
        if "measure_interval" in g:
            p.measure_interval = _as_list(g["measure_interval"], int)
    s = param.get("simple_update")
    if s is not None:
        if "num_step" in s:
            p.num_simple_step = _as_list(s["num_step"], int)
        if "tau" in s:
            p.tau_simple_step = _as_list(s["tau"], float)
        p.Inverse_lambda_cut = float(s.get("lambda_cutoff", p.Inverse_lambda_cut))
        p.Simple_Gauge_Fix = bool(s.get("gauge_fix", p.Simple_Gauge_Fix))
        p.Simple_Gauge_maxiter = int(s.get("gauge_maxiter", p.Simple_Gauge_maxiter))
        p.Simple_Gauge_Convergence_Epsilon = float(s.get("gauge_convergence_epsilon",
                                                         p.Simple_Gauge_Convergence_Epsilon))
    f = param.get("full_update")
    if f is not None:
        if "num_step" in f:
            p.num_full_step = _as_list(f["num_step"], int)
        # the reference reads full_update.tau from the simple_update table
        # (load_toml.cpp:371); kept as is
        if s is not None and "tau" in s:
            p.tau_full_step = _as_list(s["tau"], float)
        p.Full_Inverse_precision = float(f.get("inverse_precision", p.Full_Inverse_precision))
        p.Full_Convergence_Epsilon = float(f.get("convergence_epsilon", p.Full_Convergence_Epsilon))
        p.Inverse_Env_cut = float(f.get("env_cutoff", p.Inverse_Env_cut))
        p.Full_max_iteration = int(f.get("iteration_max", p.Full_max_iteration))
        p.Full_Gauge_Fix = bool(f.get("gauge_fix", p.Full_Gauge_Fix))
        p.Full_Use_FastFullUpdate = bool(f.get("fastfullupdate", p.Full_Use_FastFullUpdate))
    c = param.get("ctm")
    if c is not None:
        p.CHI = int(c.get("dimension", p.CHI))
        p.Inverse_projector_cut = float(c.get("projector_cutoff", p.Inverse_projector_cut))
        p.CTM_Convergence_Epsilon = float(c.get("convergence_epsilon", p.CTM_Convergence_Epsilon))
        p.Max_CTM_Iteration = int(c.get("iteration_max", p.Max_CTM_Iteration))
        p.CTM_Projector_corner = bool(c.get("projector_corner", p.CTM_Projector_corner))
        p.Use_RSVD = bool(c.get("use_rsvd", p.Use_RSVD))
        p.RSVD_Oversampling_factor = float(c.get("rsvd_oversampling_factor", p.RSVD_Oversampling_factor))
        p.MeanField_Env = bool(c.get("meanfield_env", p.MeanField_Env))
        if p.RSVD_Oversampling_factor < 1.0:
            raise InputError("rsvd_oversampling_factor must be >= 1.0")
    r = param.get("random")
    if r is not None:
        p.seed = int(r.get("seed", p.seed))
    return p


def gen_lattice(t: dict) -> LatticeSpec:
    """gen_lattice (load_toml.cpp:247-296) plus SquareLattice::check_dims."""
    if "L_sub" not in t:
        raise InputError("cannot find L_sub in tensor")
    L = t["L_sub"]
    if isinstance(L, int):
        L = [L, L]
    LX, LY = int(L[0]), int(L[1])
    if LX <= 0:
        raise InputError("Lattice.X should be positive")
    if LY <= 0:
        raise InputError("Lattice.Y should be positive")
    skew = int(t.get("skew", 0))
    N = LX * LY
    pd = [-1] * N
    vd = [[-1] * 4 for _ in range(N)]
    dirs: List[List[float]] = [[0.0] for _ in range(N)]
    noises = [0.0] * N
    if "unitcell" not in t:
        raise InputError("cannot find unitcell in tensor")
    for site in t["unitcell"]:
        indices = [int(i) for i in site.get("index", [])]
        if not indices:
            indices = list(range(N))
        for i in indices:
            dirs[i] = [float(x) for x in site.get("initial_state", [0.0])]
            noises[i] = float(site.get("noise", 0.0))
            if "physical_dim" not in site:
                raise InputError("cannot find physical_dim in tensor.unitcell")
            pd[i] = int(site["physical_dim"])
            v = site.get("virtual_dim")
            if v is None:
                raise InputError("cannot find virtual_dim in tensor.unitcell")
            v = [int(x) for x in (v if isinstance(v, list) else [v])]
            if len(v) == 1:
                v = v * 4
            if len(v) != 4:
                raise InputError("The size of tensor.unitcell.virtual_dim must be 1 or 4.")
            vd[i] = v
    spec = LatticeSpec(LX, LY, skew, pd, vd, dirs, noises)
    return spec


def _read_bonds(text: str) -> List[Tuple[int, int, int]]:
    out = []
    for raw in text.splitlines():
        w = _drop_comment(raw).split()
        if not w:
            continue
        if len(w) < 3:
            raise InputError("A bond should have 3 integers")
        out.append((int(w[0]), int(w[1]), int(w[2])))
    return out


def _read_multisites(text: str):
    out = []
    for raw in text.splitlines():
        w = _drop_comment(raw).split()
        if not w:
            continue
        if len(w) < 5:
            raise InputError("A multisite should have at least 5 integers")
        if len(w) % 2 != 1:
            raise InputError("A multisite should have odd number of integers")
        dx = [int(w[i]) for i in range(1, len(w), 2)]
        dy = [int(w[i + 1]) for i in range(1, len(w), 2)]
        out.append((int(w[0]), dx, dy))
    return out


def load_operator(t: dict, nsites: int, nbody: int, atol: float, table: str) -> List[Operator]:
    """load_operator (load_toml.cpp:451-565)."""
    elements = t.get("elements")
    ops = t.get("ops")
    if elements is not None and ops is not None:
        raise InputError(f"Both elements and ops are defined in a section {table}")
    if nbody == 1 and elements is None:
        raise InputError(f"elements not found in a section {table}")
    A = None
    op_ind: List[int] = []
    if elements is not None:
        if nbody > 2:
            raise InputError("observable.multisite does not support elements")
        dim = t.get("dim")
        if dim is None:
            raise InputError(f"cannot find dim in {table}")
        if isinstance(dim, list):
            if len(dim) != nbody:
                raise InputError(f"operator is {nbody}-sites but dim has {len(dim)} integers")
            shape = [int(d) for d in dim]
        else:
            shape = [int(dim)] * nbody
        shape = shape + shape
        A = read_tensor(elements, shape, atol)
    elif ops is not None:
        op_ind = [int(i) for i in ops]
    else:
        raise InputError(f"Neither elements nor ops are not defined in a section {table}")
    if "group" not in t:
        raise InputError(f"cannot find group in {table}")
    group = int(t["group"])
    name = str(t.get("name", ""))
    coeff = complex(float(t.get("coeff", 1.0)), float(t.get("coeff_im", 0.0)))
    out = []
    if nbody == 1:
        sites = t.get("sites")
        if sites is None:
            raise InputError(f"cannot find sites in {table}")
        sites = [int(s) for s in sites] if isinstance(sites, list) else [int(sites)]
        if not sites:
            sites = list(range(nsites))
        for s in sites:
            out.append(Operator(name, group, s, [], [], A, [], coeff))
    elif nbody == 2:
        if "bonds" not in t:
            raise InputError(f"cannot find bonds in {table}")
        for (s, dx, dy) in _read_bonds(t["bonds"]):
            out.append(Operator(name, group, s, [dx], [dy], A, list(op_ind), coeff))
    else:
        if "multisites" not in t:
            raise InputError(f"cannot find multisites in {table}")
        for (s, dx, dy) in _read_multisites(t["multisites"]):
            out.append(Operator(name, group, s, dx, dy, A, list(op_ind), coeff))
    return out


def load_evolution(t: dict, atol: float, table: str) -> EvolutionOperator:
    """load_Evolution_operator (load_toml.cpp:604-638)."""
    dims = t.get("dimensions")
    if dims is None:
        raise InputError(f"cannot find dimensions in {table}")
    if "elements" not in t:
        raise InputError(f"cannot find elements in {table}")
    shape = [int(d) for d in dims]
    group = int(t.get("group", 0))
    A = read_tensor(t["elements"], shape, atol)
    if len(shape) == 2:
        return EvolutionOperator(int(t["site"]), -1, group, A)
    if len(shape) == 4:
        return EvolutionOperator(int(t["source_site"]), int(t["source_leg"]), group, A)
    raise InputError(f"{table}.dimensions should have 2 or 4 integers")


def _is_real(arrs: Sequence[Optional[np.ndarray]], tol: float) -> bool:
    """is_real (src/iTPS/main.cpp:73-135)."""
    for a in arrs:
        if a is not None and np.any(np.abs(a.imag) > tol):
            return False
    return True


def load_input(path: str) -> Input:
    """Parse an expert-format input file (tenes::itps::itps_main,
    src/iTPS/main.cpp:208-351)."""
    with open(path, "rb") as f:
        toml = tomllib.load(f)
    return load_input_dict(toml)


def load_input_dict(toml: dict) -> Input:
    param = toml.get("parameter", {})
    p = gen_param(param)
    if "tensor" not in toml:
        raise InputError("cannot find tensor section")
    lat = gen_lattice(toml["tensor"])
    N = lat.LX * lat.LY
    tol = p.iszero_tol
    evo = toml.get("evolution", {})
    su = [load_evolution(t, tol, "evolution.simple") for t in evo.get("simple", [])]
    fu = [load_evolution(t, tol, "evolution.full") for t in evo.get("full", [])]
    obs = toml.get("observable", {})
    one = [o for t in obs.get("onesite", []) for o in load_operator(t, N, 1, tol, "observable.onesite")]
    two = [o for t in obs.get("twosite", []) for o in load_operator(t, N, 2, tol, "observable.twosite")]
    multi = [o for t in obs.get("multisite", []) for o in load_operator(t, N, 3, tol, "observable.multisite")]
    tm = TransferMatrixParameters()
    cl = toml.get("correlation_length")
    if cl is not None:
        tm.to_calculate = bool(cl.get("measure", tm.to_calculate))
        tm.num_eigvals = int(cl.get("num_eigvals", tm.num_eigvals))
        tm.maxdim_dense_eigensolver = int(cl.get("maxdim_dense_eigensolver", tm.maxdim_dense_eigensolver))
        tm.arnoldi_maxdim = int(cl.get("arnoldi_maxdim", tm.arnoldi_maxdim))
        tm.arnoldi_restartdim = int(cl.get("arnoldi_restartdim", tm.arnoldi_restartdim))
        tm.arnoldi_maxiter = int(cl.get("arnoldi_maxiterations", tm.arnoldi_maxiter))
        tm.arnoldi_rtol = float(cl.get("arnoldi_rtol", tm.arnoldi_rtol))
    cp = CorrelationParameters()
    cor = toml.get("correlation")
    if cor is not None:
        if "r_max" not in cor:
            raise InputError("cannot find r_max in correlation")
        if "operators" not in cor:
            raise InputError("cannot find operators in correlation")
        cp.r_max = int(cor["r_max"])
        cp.operators = [(int(o[0]), int(o[1])) for o in cor["operators"]]
    real = p.is_real
    real = real and _is_real([e.op for e in su], tol) and _is_real([e.op for e in fu], tol)
    real = real and _is_real([o.op for o in one + two + multi], tol)
    if p.is_real and not real:
        raise InputError("TeNeS invoked in real tensor mode (parameter.general.is_real = true) "
                         "but some operators are complex.")
    return Input(p, lat, su, fu, one, two, multi, tm, real, cp)
