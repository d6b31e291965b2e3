"""Tensor checkpoints: iTPS::save_tensors / load_tensors
(src/iTPS/saveload_tensors.cpp:38-262) and resize_tensor (src/tensor.cpp:114-149).

The directory layout, the metadata file and the semantics follow the
reference:

* ``params.dat``: format version (1), N_UNIT, CHI, then one line per site with
  the four virtual dimensions and the physical dimension, each line followed
  by a ``# comment`` (saveload_tensors.cpp:45-58);
* ``T_i.dat``, ``Et_i.dat``, ``Er_i.dat``, ``Eb_i.dat``, ``El_i.dat``,
  ``C1_i.dat`` ... ``C4_i.dat`` for every site i (saveload_tensors.cpp:59-71);
* ``lambda_i.dat``: the simple-update weights of the four legs, one value per
  line (saveload_tensors.cpp:72-82);
* on load, every tensor is zero-extended / sliced to the current shapes, the
  weights of a leg are cut or zero-padded to its current dimension, N_UNIT or
  physical-dimension mismatches are errors, CHI and virtual-dimension
  mismatches are warnings (saveload_tensors.cpp:88-262).

The per-tensor files are this library's own text format: TeNeS writes them
through mptensor's ``Tensor::save``, which is not part of the reference tree.
A file is one header line ``# tenes_b200 tensor 1 <real|complex> <rank>
<d0> ... <d_{rank-1}>`` followed by the entries in row-major order, one per
line (``re im`` for complex), printed with 17 significant digits so that a
save / load round trip is exact.  The weights are printed the same way (the
reference prints them with the stream's default 6 digits; both read back).
"""

from __future__ import annotations

import os
import sys
from typing import List, Sequence, Tuple

import numpy as np

FORMAT_VERSION = 1
HEADER = "# tenes_b200 tensor 1"
# file stem -> index of Environment.get_env / set_env
ENV_FILES = (("Et", 4), ("Er", 5), ("Eb", 6), ("El", 7), ("C1", 0), ("C2", 1), ("C3", 2), ("C4", 3))


class LoadError(RuntimeError):
    """tenes::load_error: an unreadable or incompatible checkpoint."""


def write_tensor(path: str, a: np.ndarray) -> None:
    a = np.asarray(a)
    cplx = np.iscomplexobj(a)
    with open(path, "w") as f:
        f.write(f"{HEADER} {'complex' if cplx else 'real'} {a.ndim} {' '.join(str(d) for d in a.shape)}\n")
        flat = a.reshape(-1)
        if cplx:
            f.write("".join(f"{x.real:.17g} {x.imag:.17g}\n" for x in flat))
        else:
            f.write("".join(f"{x:.17g}\n" for x in flat))


def read_tensor(path: str) -> np.ndarray:
    if not os.path.exists(path):
        raise LoadError(f"{path} does not exist")
    with open(path) as f:
        head = f.readline().split()
        if " ".join(head[:4]) != HEADER or len(head) < 6:
            raise LoadError(f"{path} is not a tenes_b200 tensor file (tensors saved by TeNeS itself use "
                            "mptensor's own format, which this library does not read)")
        kind, rank = head[4], int(head[5])
        shape = tuple(int(x) for x in head[6:6 + rank])
        vals = np.array(f.read().split(), dtype=np.float64)
    n = int(np.prod(shape)) if shape else 1
    if kind == "complex":
        if vals.size != 2 * n:
            raise LoadError(f"{path}: {vals.size // 2} entries for shape {shape}")
        return (vals[0::2] + 1j * vals[1::2]).reshape(shape)
    if vals.size != n:
        raise LoadError(f"{path}: {vals.size} entries for shape {shape}")
    return vals.reshape(shape)


def resize_tensor(src: np.ndarray, shape: Sequence[int]) -> np.ndarray:
    """Zero-extend the legs shorter than ``shape`` and slice the longer ones
    (resize_tensor, tensor.cpp:114-149)."""
    if src.ndim != len(shape):
        raise LoadError(f"rank mismatch: {src.ndim} legs loaded, {len(shape)} expected")
    out = np.zeros(tuple(shape), dtype=src.dtype)
    common = tuple(slice(0, min(a, b)) for a, b in zip(src.shape, shape))
    out[common] = src[common]
    return out


def _drop_comment(line: str) -> str:
    return line.split("#", 1)[0].strip()


def save_tensors(env, save_dir: str, chi: int, print_level: int = 1) -> None:
    """iTPS::save_tensors (saveload_tensors.cpp:38-86) for the context's site
    tensors, environment and weights."""
    if not save_dir:
        return
    os.makedirs(save_dir, exist_ok=True)
    N = env.N
    with open(os.path.join(save_dir, "params.dat"), "w") as f:
        f.write(f"{FORMAT_VERSION} # Format_Version\n{N} # N_UNIT\n{chi} # CHI\n")
        for i in range(N):
            f.write(" ".join(str(d) for d in env.vdim[i]) + f" {env.pdim[i]} # Shape of Tn[{i}]\n")
    for i in range(N):
        write_tensor(os.path.join(save_dir, f"T_{i}.dat"), env.get_site_tensor(i))
        for stem, w in ENV_FILES:
            write_tensor(os.path.join(save_dir, f"{stem}_{i}.dat"), env.get_env(w, i))
        with open(os.path.join(save_dir, f"lambda_{i}.dat"), "w") as f:
            for leg in range(4):
                f.write("".join(f"{x:.17g}\n" for x in env.get_lambda(i, leg)))
    if print_level > 0:
        print(f"Tensors saved in {save_dir}")


def load_tensors(env, load_dir: str, chi: int, print_level: int = 1) -> None:
    """iTPS::load_tensors / load_tensors_v1 (saveload_tensors.cpp:88-214):
    site tensors, environment and weights from ``load_dir``, resized to the
    context's shapes."""
    if not os.path.isdir(load_dir):
        raise LoadError(f"{load_dir} does not exists.")
    pfile = os.path.join(load_dir, "params.dat")
    if not os.path.exists(pfile):
        raise LoadError(f"{pfile} is missing (format version 0 checkpoints are mptensor files, which this "
                        "library does not read)")
    with open(pfile) as f:
        lines = [ln for ln in f.read().splitlines()]
    version = int(_drop_comment(lines[0]))
    if version != FORMAT_VERSION:
        raise LoadError(f"ERROR: Unknown saved tensor format version: {version}")
    N = env.N
    loaded_N = int(_drop_comment(lines[1]))
    if loaded_N != N:
        raise LoadError(f"ERROR: N_UNIT is {N} but loaded N_UNIT has {loaded_N}")
    loaded_chi = int(_drop_comment(lines[2]))
    if loaded_chi != chi and print_level > 0:
        print(f"WARNING: parameters.ctm.dimension is {chi} but loaded tensors have CHI = {loaded_chi}")
    loaded_shape: List[Tuple[int, ...]] = []
    for i in range(N):
        sh = tuple(int(x) for x in _drop_comment(lines[3 + i]).split())
        for leg in range(4):
            if sh[leg] != env.vdim[i][leg] and print_level > 0:
                print(f"WARNING: virtual dimension of the leg {leg} of the tensor {i} is {env.vdim[i][leg]} "
                      f"but loaded tensor has {sh[leg]}")
        if sh[4] != env.pdim[i]:
            raise LoadError(f"ERROR: dimension of the physical bond of the tensor {i} is {env.pdim[i]} but "
                            f"loaded tensor has {sh[4]}")
        loaded_shape.append(sh)
    dtype = np.complex128 if env.is_complex else np.float64

    def load(stem: str, i: int, shape) -> np.ndarray:
        a = read_tensor(os.path.join(load_dir, f"{stem}_{i}.dat"))
        if len(shape) != a.ndim:
            raise LoadError(f"ERROR: rank mismatch in load_tensor: {stem}[{i}] has {len(shape)} legs, but "
                            f"loaded one has {a.ndim} legs.")
        if np.iscomplexobj(a) and not env.is_complex:
            if np.max(np.abs(a.imag), initial=0.0) > 0.0:
                raise LoadError(f"{stem}[{i}]: complex tensor loaded into a real calculation")
            a = a.real
        return resize_tensor(a.astype(dtype), shape)

    for i in range(N):
        env.set_site_tensor(i, load("T", i, env.site_shape(i)))
        for stem, w in ENV_FILES:
            env.set_env(w, i, load(stem, i, env.env_shape(w, i)))
        path = os.path.join(load_dir, f"lambda_{i}.dat")
        if not os.path.exists(path):
            raise LoadError(f"{path} does not exist")
        with open(path) as f:
            vals = [float(x) for x in f.read().split()]
        off = 0
        for leg in range(4):
            n = loaded_shape[i][leg]
            lam = np.zeros(env.vdim[i][leg])
            seg = vals[off:off + n]
            if len(seg) < n:
                raise LoadError(f"{path}: {len(vals)} weights, fewer than the loaded shapes need")
            m = min(n, env.vdim[i][leg])
            lam[:m] = seg[:m]
            off += n
            env.set_lambda(i, leg, lam)
    if print_level > 0:
        print(f"Tensors loaded from {load_dir}")
        sys.stdout.flush()
