"""Energy gradients of iTPS site tensors through the CTMRG environment.

No counterpart in the reference: TeNeS optimises site tensors by simple and
full update only.  This module is the tooling layer over the library's
adjoint (``tg_energy_grad``):

* ``two_site_terms`` / ``one_site_term`` turn operators into window terms,
  the form the adjoint evaluates -- a two-site operator becomes the products
  of its singular components on the window of its displacement, the way
  ``twosite_obs.cpp:223-243`` measures operators beyond nearest neighbours,
  with the window geometry of ``twosite_obs.cpp:95-110``;
* ``j1j2_terms`` is the energy per site of the J1-J2 Heisenberg model;
* ``CTMEnergy`` is a ``torch.autograd.Function`` whose forward runs the CTMRG
  sweeps and the energy on the GPU and whose backward is the library's
  hand-written reverse pass;
* ``optimize_lbfgs`` minimises the energy over the site tensors with
  ``torch.optim.LBFGS``.
"""

from __future__ import annotations

from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from .env import Environment
from .std_ops import heisenberg_bond, real_if_close

Term = Dict


def window_geometry(dx: int, dy: int) -> Tuple[int, int, int, int, int, int]:
    """(nrow, ncol, source_row, source_col, target_row, target_col) of the
    window spanning a displacement (dx right, dy up), row 0 on top
    (twosite_obs.cpp:95-110)."""
    nrow, ncol = abs(dy) + 1, abs(dx) + 1
    sc, tc = (0, ncol - 1) if dx >= 0 else (ncol - 1, 0)
    sr, tr = (nrow - 1, 0) if dy >= 0 else (0, nrow - 1)
    return nrow, ncol, sr, sc, tr, tc


def one_site_term(site: int, op: np.ndarray, coeff: float = 1.0) -> Term:
    return dict(source=site, nrow=1, ncol=1, source_row=0, source_col=0,
                ops={(0, 0): np.asarray(real_if_close(np.asarray(op)), dtype=np.float64)}, coeff=coeff)


def two_site_terms(source: int, dx: int, dy: int, op12: np.ndarray, coeff: float = 1.0) -> List[Term]:
    """<op12> between ``source`` and the site (dx, dy) away, as window terms:
    op12[a, b, a', b'] = sum_k A_k[a, a'] B_k[b, b'] from the SVD of op12 over
    legs (0, 2) | (1, 3) (twosite_obs.cpp:223-243), the singular value folded
    into A_k; components below 1e-14 of the largest are dropped."""
    if dx == 0 and dy == 0:
        raise ValueError("two_site_terms: the two sites must differ")
    op = np.asarray(real_if_close(np.asarray(op12)), dtype=np.float64)
    if np.iscomplexobj(op):
        raise ValueError("two_site_terms: real operators only")
    d1, d2 = op.shape[0], op.shape[1]
    U, s, Vh = np.linalg.svd(op.transpose(0, 2, 1, 3).reshape(d1 * d1, d2 * d2))
    nrow, ncol, sr, sc, tr, tc = window_geometry(dx, dy)
    terms = []
    for k in range(len(s)):
        if s[k] <= 1e-14 * s[0]:
            break
        terms.append(dict(source=source, nrow=nrow, ncol=ncol, source_row=sr, source_col=sc,
                          ops={(sr, sc): (U[:, k] * s[k]).reshape(d1, d1), (tr, tc): Vh[k].reshape(d2, d2)},
                          coeff=coeff))
    return terms


def j1j2_terms(n_sites: int, J1: float = 1.0, J2: float = 0.0, S: float = 0.5) -> List[Term]:
    """Energy per site of the J1-J2 Heisenberg model on the square lattice:
    (1/N) sum_i [J1 (S_i.S_{i+x} + S_i.S_{i+y}) + J2 (S_i.S_{i+x+y} + S_i.S_{i+x-y})]."""
    h = heisenberg_bond(1.0, S=S)
    terms: List[Term] = []
    for i in range(n_sites):
        for dx, dy in ((1, 0), (0, 1)):
            terms += two_site_terms(i, dx, dy, h, J1 / n_sites)
        if J2 != 0.0:
            for dx, dy in ((1, 1), (1, -1)):
                terms += two_site_terms(i, dx, dy, h, J2 / n_sites)
    return terms


class CTMEnergy(torch.autograd.Function):
    """E(Tn) through ``iterations`` CTMRG sweeps on the GPU; the backward is
    the library's reverse pass (``Environment.energy_grad``).  The site
    tensors are CPU float64 tensors; ``env`` is the Environment whose
    lattice, chi and precision are used (its site tensors are overwritten)."""

    @staticmethod
    def forward(ctx, env: Environment, terms, iterations: int, checkpoint_every: int, broadening: float,
                *Tn: torch.Tensor) -> torch.Tensor:
        for i, t in enumerate(Tn):
            env.set_site_tensor(i, t.detach().cpu().numpy().astype(np.float64))
        want = any(ctx.needs_input_grad[5:])
        E, g = env.energy_grad(terms, iterations, checkpoint_every, broadening, grad=want)
        ctx.grads = [torch.from_numpy(x.copy()) for x in g] if want else None
        ctx.nsites = len(Tn)
        return torch.tensor(E, dtype=torch.float64)

    @staticmethod
    def backward(ctx, gE: torch.Tensor):
        grads = tuple(gE * g for g in ctx.grads) if ctx.grads is not None else (None,) * ctx.nsites
        return (None, None, None, None, None) + grads


def energy(env: Environment, Tn: Sequence[torch.Tensor], terms, iterations: int, checkpoint_every: int = 5,
           broadening: float = 1e-12) -> torch.Tensor:
    return CTMEnergy.apply(env, terms, iterations, checkpoint_every, broadening, *Tn)


def optimize_lbfgs(env: Environment, Tn0: Sequence[np.ndarray], terms, iterations: int, steps: int,
                   checkpoint_every: int = 5, broadening: float = 1e-12, lr: float = 1.0, history: int = 10,
                   callback: Optional[Callable[[int, float], None]] = None):
    """``steps`` L-BFGS steps (strong-Wolfe line search) on the site tensors.
    Returns the optimised tensors and the energy after every step."""
    params = [torch.tensor(np.asarray(t, dtype=np.float64), requires_grad=True) for t in Tn0]
    opt = torch.optim.LBFGS(params, lr=lr, max_iter=1, history_size=history, line_search_fn="strong_wolfe")

    def closure():
        opt.zero_grad()
        E = energy(env, params, terms, iterations, checkpoint_every, broadening)
        E.backward()
        return E

    energies = []
    for step in range(steps):
        E = float(opt.step(closure))
        energies.append(E)
        if callback is not None:
            callback(step, E)
    return [p.detach().numpy().copy() for p in params], energies
