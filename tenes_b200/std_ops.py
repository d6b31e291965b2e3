"""Spin operators and imaginary-time evolution operators, the input side of
the path (what tool/tenes_std.py writes into ``[[evolution.simple]]``).

Conventions follow the reference:
* spin-S operators in the S^z eigenbasis ordered m = S, S-1, ..., -S
  (tool/tenes_simple.py:624-657);
* a two-site operator is stored as op[a, b, c, d] = <a b| O |c d>, and the
  evolution operator of a bond is exp(-tau H_bond) (first-order Trotter,
  tool/tenes_std.py:893-957); a one-site operator is exp(-tau H_site)
  (tool/tenes_std.py:880-891).
"""

from __future__ import annotations

import numpy as np
import scipy.linalg


def spin_ops(S: float = 0.5):
    """(Sz, Sx, Sy) for spin S."""
    n = int(round(2 * S)) + 1
    m = S - np.arange(n)
    Sz = np.diag(m).astype(np.complex128)
    Sp = np.zeros((n, n), dtype=np.complex128)
    for i in range(1, n):
        Sp[i - 1, i] = np.sqrt(S * (S + 1) - m[i] * (m[i] + 1))
    Sm = Sp.conj().T
    Sx = 0.5 * (Sp + Sm)
    Sy = -0.5j * (Sp - Sm)
    return Sz, Sx, Sy


def two_site(A: np.ndarray, B: np.ndarray) -> np.ndarray:
    """A (x) B as op[a, b, c, d] = A[a, c] B[b, d]."""
    return np.einsum("ac,bd->abcd", A, B)


def heisenberg_bond(J: float = 1.0, Jz: float = None, S: float = 0.5) -> np.ndarray:
    """J (SxSx + SySy) + Jz SzSz as a (d, d, d, d) tensor."""
    Sz, Sx, Sy = spin_ops(S)
    Jz = J if Jz is None else Jz
    H = J * (two_site(Sx, Sx) + two_site(Sy, Sy)) + Jz * two_site(Sz, Sz)
    return H


def ising_bond(Jz: float = 1.0, S: float = 0.5) -> np.ndarray:
    """-Jz SzSz (transverse-field Ising bond)."""
    Sz, _, _ = spin_ops(S)
    return -Jz * two_site(Sz, Sz)


def evolution_twosite(H: np.ndarray, tau: float) -> np.ndarray:
    """exp(-tau H) of a two-site Hamiltonian (tool/tenes_std.py:893-957)."""
    d1, d2 = H.shape[0], H.shape[1]
    M = H.reshape(d1 * d2, d1 * d2)
    U = scipy.linalg.expm(-tau * M)
    return U.reshape(d1, d2, d1, d2)


def evolution_onesite(H: np.ndarray, tau: float) -> np.ndarray:
    """exp(-tau H) of a one-site Hamiltonian (tool/tenes_std.py:880-891)."""
    return scipy.linalg.expm(-tau * H)


def real_if_close(a: np.ndarray, tol: float = 1e-14) -> np.ndarray:
    return a.real.copy() if np.max(np.abs(a.imag), initial=0.0) <= tol else a
