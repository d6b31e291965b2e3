"""CPU stand-in for tenes_b200.env.Environment built on the oracle.

Test infrastructure only: it lets the front-end's driver loop and writers run
here (no GPU) against the golden output files.  The product never imports it."""
import numpy as np

from oracle import tenes_density as D
from oracle import tenes_oracle as O


class OracleEnvironment:
    def __init__(self, LX, LY, physical_dims, virtual_dims, params, is_complex, skew=0, device=0):
        self.lat = O.Lattice(LX, LY, skew)
        self.lat.physical_dims = list(physical_dims)
        self.lat.virtual_dims = [list(v) for v in virtual_dims]
        self.N = LX * LY
        self.is_complex = is_complex
        self.p = O.Params(CHI=params.chi, Inverse_projector_cut=params.inverse_projector_cut,
                          CTM_Convergence_Epsilon=params.ctm_convergence_epsilon,
                          Max_CTM_Iteration=params.max_ctm_iteration,
                          CTM_Projector_corner=params.projector_corner, Use_RSVD=params.use_rsvd,
                          RSVD_Oversampling_factor=params.rsvd_oversampling_factor,
                          Inverse_lambda_cut=params.inverse_lambda_cut)
        self.env = None
        self.lam = [[np.ones(v[l]) for l in range(4)] for v in virtual_dims]
        # an iTPO (finite temperature) runs through oracle/tenes_density.py
        self.density = bool(getattr(params, "density", False))

    # accessors of tenes_b200.env.Environment (checkpoints)
    @property
    def pdim(self):
        return self.lat.physical_dims

    @property
    def vdim(self):
        return self.lat.virtual_dims

    def site_shape(self, i):
        v = self.lat.virtual_dims[i]
        d = self.lat.physical_dims[i]
        return (v[0], v[1], v[2], v[3], d, d) if self.density else (v[0], v[1], v[2], v[3], d)

    def env_shape(self, which, i):
        chi = self.p.CHI
        if which < 4:
            return (chi, chi)
        d = self.lat.virtual_dims[i][{4: 1, 5: 2, 6: 3, 7: 0}[which]]
        return (chi, chi, d, d)

    def _env_or_zeros(self):
        if self.env is None:
            dt = np.complex128 if self.is_complex else np.float64
            names = ("C1", "C2", "C3", "C4", "eTt", "eTr", "eTb", "eTl")
            self.env = O.Env(*[[np.zeros(self.env_shape(w, i), dtype=dt) for i in range(self.N)]
                               for w in range(len(names))])
        return self.env

    def get_site_tensor(self, i):
        return np.array(self.Tn[i], copy=True)

    def set_site_tensor(self, i, T):
        if not hasattr(self, "Tn"):
            self.Tn = [None] * self.N
        assert tuple(T.shape) == self.site_shape(i)
        self.Tn[i] = np.array(T, dtype=np.complex128 if self.is_complex else np.float64)

    def get_env(self, which, i):
        names = ("C1", "C2", "C3", "C4", "eTt", "eTr", "eTb", "eTl")
        return np.array(getattr(self._env_or_zeros(), names[which])[i], copy=True)

    def set_env(self, which, i, T):
        names = ("C1", "C2", "C3", "C4", "eTt", "eTr", "eTb", "eTl")
        assert tuple(T.shape) == self.env_shape(which, i)
        getattr(self._env_or_zeros(), names[which])[i] = np.array(T)

    def get_lambda(self, i, leg):
        return np.array(self.lam[i][leg], copy=True)

    def set_lambda(self, i, leg, lam):
        assert len(lam) == self.lat.virtual_dims[i][leg]
        self.lam[i][leg] = np.array(lam, dtype=np.float64)

    def init_tensors(self, seed, initial_dirs, noises):
        self.lat.initial_dirs = [list(d) for d in initial_dirs]
        self.lat.noises = list(noises)
        if self.density:
            self.Tn = D.initial_density(self.lat, not self.is_complex)
            return
        self.Tn = O.initialize_tensors(self.lat, seed, not self.is_complex)

    def fix_local_gauge(self, maxiter=100, eps=1e-2):
        if self.density:
            flat = [t.reshape(t.shape[:4] + (-1,)) for t in self.Tn]
            r = O.fix_local_gauge(flat, self.lam, self.lat, self.p, maxiter, eps)
            self.Tn = [f.reshape(t.shape) for f, t in zip(flat, self.Tn)]
            return r
        return O.fix_local_gauge(self.Tn, self.lam, self.lat, self.p, maxiter, eps)

    def simple_update(self, source, leg, op):
        if self.density:
            class _Up:
                pass
            up = _Up()
            up.source_site, up.source_leg, up.op = source, leg, op
            up.is_onesite = lambda: leg < 0
            D.su_density(self.Tn, self.lam, self.lat, up, self.p)
            return
        if leg < 0:
            self.Tn[source] = np.tensordot(self.Tn[source], op, ([4], [0]))
            return
        tg = self.lat.neighbor(source, leg)
        a, b, lc = O.simple_update_bond(self.Tn[source], self.Tn[tg], self.lam[source], self.lam[tg], op, leg,
                                        self.p)
        self.lam[source][leg] = lc
        self.lam[tg][(leg + 2) % 4] = lc
        self.Tn[source], self.Tn[tg] = a, b

    def simple_update_many(self, steps):
        for source, leg, op in steps:
            self.simple_update(source, leg, op)

    def sync(self):
        pass

    def full_update_bond(self, source, leg, op, inverse_env_cut=1e-12, inverse_precision=1e-12,
                         convergence_epsilon=1e-6, max_iteration=100, gauge_fix=True):
        import dataclasses
        p = dataclasses.replace(self.p, Inverse_Env_cut=inverse_env_cut, Full_Inverse_precision=inverse_precision,
                                Full_Convergence_Epsilon=convergence_epsilon, Full_max_iteration=max_iteration,
                                Full_Gauge_Fix=gauge_fix)
        tg = self.lat.neighbor(source, leg)
        args = O.full_update_env_args(self.env, source, leg, self.lat)
        r = O._FU_ROT[leg]
        a, b, it, conv = O.full_update_bond_horizontal(*args, self.Tn[source].transpose(r),
                                                       self.Tn[tg].transpose(r), op, p)
        k = O._FU_BACK[leg]
        self.Tn[source], self.Tn[tg] = a.transpose(k), b.transpose(k)
        return it, conv

    def correlation_strip(self, left, vertical, r_max, left_op, right_ops):
        if self.density:
            return np.array(D.correlation_strip(self.env, self.Tn, self.lat, left, vertical, r_max, left_op,
                                                right_ops))
        return np.array(O.correlation_strip(self.env, self.Tn, self.lat, left, vertical, r_max, left_op,
                                            right_ops))

    def move(self, direction, line):
        fn = (O.left_move, O.right_move, O.top_move, O.bottom_move)[direction]
        fn(self.env, self.Tn, line, self.p, self.lat)

    def calc_ctm_environment(self, initialize=True):
        calc = D.calc_ctm_environment if self.density else O.calc_ctm_environment
        self.env, it, conv, sig = calc(self.Tn, self.p, self.lat)
        return it, conv, sig

    def contract_one_site(self, i, op):
        e = self.env
        f = D.contract_one_site if self.density else O.contract_one_site
        return complex(f(e.C1[i], e.C2[i], e.C3[i], e.C4[i], e.eTt[i], e.eTr[i], e.eTb[i],
                                           e.eTl[i], self.Tn[i], op))

    def contract_bond_op12(self, source, dx, dy, op):
        e, lat, Tn = self.env, self.lat, self.Tn
        if self.density:
            return D.contract_op12(e, Tn, lat, source, dx, dy, op)
        if dy == 0:
            sc = 0 if dx >= 0 else 1
            l, r = lat.other(source, -sc, 0), lat.other(source, 1 - sc, 0)
            o = op if l == source else op.transpose(1, 0, 3, 2)
            return complex(O.contract_two_sites_horizontal_op12(
                e.C1[l], e.C2[r], e.C3[r], e.C4[l], e.eTt[l], e.eTt[r], e.eTr[r], e.eTb[r], e.eTb[l], e.eTl[l],
                Tn[l], Tn[r], o))
        sr = 1 if dy >= 0 else 0
        t, b = lat.other(source, 0, sr), lat.other(source, 0, sr - 1)
        o = op if t == source else op.transpose(1, 0, 3, 2)
        return complex(O.contract_two_sites_vertical_op12(
            e.C1[t], e.C2[t], e.C3[b], e.C4[b], e.eTt[t], e.eTr[t], e.eTr[b], e.eTb[b], e.eTl[b], e.eTl[t],
            Tn[t], Tn[b], o))

    def contract_window(self, source, nrow, ncol, source_row, source_col, ops=None):
        ops = ops or {}
        if self.density:
            return D.window_value(self.env, self.Tn, self.lat, source, nrow, ncol, source_row, source_col, ops)
        idx, Cs, eTt, eTr, eTb, eTl, T = O._window(self.env, self.Tn, self.lat, source, source_col, source_row,
                                                    nrow, ncol)
        grid = [[ops.get((r, c), np.eye(self.lat.physical_dims[idx[r][c]])) for c in range(ncol)]
                for r in range(nrow)]
        return complex(O.contract_window(Cs, eTt, eTr, eTb, eTl, T, grid))

    def tm_eigenvalues(self, direction, fixed, num_eigvals=4, maxdim_dense=200, arnoldi_maxdim=50,
                       arnoldi_restartdim=20, arnoldi_maxiter=1, arnoldi_rtol=1e-10):
        tp = O.TMParams(num_eigvals, maxdim_dense, arnoldi_maxdim, arnoldi_restartdim, arnoldi_maxiter,
                        arnoldi_rtol)
        if self.density:
            return D.tm_eigenvalues(self.env, self.lat, direction, fixed, tp)
        return O.tm_eigenvalues(self.env, self.lat, direction, fixed, tp)
