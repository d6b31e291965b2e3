"""Pin the iTPO (finite-temperature) oracle against the reference's own
finite-temperature runs, test/data/output_FT_TFI_square (2x2 cell, D = 3,
chi = 10, 10 CTMRG iterations, complex) and test/data/output_FT_Kitaev (2x1
skewed cell, D = 4 with a unit leg, chi = 5): the density simple update, the
single-layer CTMRG and every observable file (FT_density, FT_onesite_obs,
FT_twosite_obs, FT_correlation, FT_correlation_length) at every measured
inverse temperature.  The reference's check is rtol 1e-3 / atol 1e-4
(test/fulltest.py.in:141-142).

Observed deviations: FT_Kitaev 1e-12 (observables) and 1.3e-5 (the
transfer-matrix spectra, whose sub-leading eigenvalues are near-degenerate);
FT_TFI_square 2e-10 at beta = 1 and up to 1.2e-5 at beta = 2, where the ten
CTMRG iterations end before the environment has converged."""
import numpy as np
import pytest

from oracle import tenes_density as D
from oracle import tenes_oracle as O
from tests import _ft

TOL = {"ft_tfi_square": (5e-5, 5e-4), "ft_kitaev": (1e-10, 1e-4)}


def _tm(inp):
    t = inp.tm_params
    return O.TMParams(t.num_eigvals, t.maxdim_dense_eigensolver, t.arnoldi_maxdim, t.arnoldi_restartdim,
                      t.arnoldi_maxiter, t.arnoldi_rtol)


@pytest.mark.parametrize("stem", sorted(TOL))
def test_finite_temperature_golden(stem):
    exp = _ft.expected(stem)
    tol, tol_xi = TOL[stem]
    seen = []

    def close(v, re, im=None):
        assert abs(v.real - re) <= tol * max(1.0, abs(re)), (v, re)
        if im is not None:
            assert abs(v.imag - im) <= tol * max(1.0, abs(im)), (v, im)

    def on_measure(beta, inp, lat, p, one, two, multi, Tn):
        env, v1, norm, v2, norms2, _ = _ft.measure(inp, lat, p, one, two, multi, Tn)
        at = lambda key: [r for r in exp[key] if abs(r[0] - beta) < 1e-9]  # noqa: E731
        rows = at("onesite")
        assert rows
        for r in rows:
            close(norm[int(r[2])] if int(r[1]) == -1 else v1[int(r[1])][int(r[2])], r[3], r[4])
        for r in at("twosite"):
            if int(r[1]) >= 0:
                close(v2[int(r[1])][(int(r[2]), int(r[3]), int(r[4]))], r[5], r[6])
        bond_groups = {o.group for o in two if o.name == "bond_hamiltonian"}
        E = sum(sum(v2[g].values()).real for g in bond_groups) / lat.N_UNIT
        dens = [r for r in at("density") if int(r[1]) == 0]
        assert abs(E - dens[0][2]) <= tol * max(1.0, abs(dens[0][2]))
        cor = _ft.correlations(inp, lat, env, Tn, one)
        for r in at("correlation"):
            close(cor[(int(r[1]), int(r[2]), int(r[3]), int(r[4]), int(r[5]))], r[6], r[7])
        if beta > 0.0:  # measure.cpp:134-138 skips beta = 0
            for r in at("correlation_length"):
                ev = D.tm_eigenvalues(env, lat, int(r[1]), int(r[2]), _tm(inp))
                L = lat.LX_noskew if int(r[1]) == 0 else lat.LY_noskew
                xi, es = O.correlation_length(ev, L)
                assert xi == pytest.approx(r[3], rel=tol_xi)
                np.testing.assert_allclose(es, r[4:], rtol=tol_xi)
        seen.append(beta)

    _ft.run(stem, on_measure)
    betas = sorted({r[0] for r in exp["onesite"]})
    np.testing.assert_allclose(seen, betas, atol=1e-9)


def test_density_simple_update_equals_the_superoperator():
    """A bond step of the density simple update is Simple_update_bond on the
    d*d physical leg with kron(op, conj(op)) (simple_update.cpp:148-176); for
    a product of identities with one-site operators the one-site step is
    op^T rho op^dagger per site (simple_update.cpp:143-147)."""
    rng = np.random.default_rng(3)
    d = 2
    T = rng.standard_normal((1, 1, 1, 1, d, d)) + 1j * rng.standard_normal((1, 1, 1, 1, d, d))
    op = rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))

    class Up:
        source_site = 0
        source_leg = -1
        op = None

        def is_onesite(self):
            return True
    up = Up()
    up.op = op
    Tn = [T.copy()]
    D.su_density(Tn, None, None, up, O.Params())
    rho = T[0, 0, 0, 0]
    np.testing.assert_allclose(Tn[0][0, 0, 0, 0], op.T @ rho @ op.conj().T, atol=1e-13)
    a = rng.standard_normal((2, 3, 2, 3))
    b = rng.standard_normal((3, 2, 3, 2))
    k = D.kron4(a, b)
    assert k.shape == (6, 6, 6, 6)
    assert k[1 * 3 + 2, 0 * 2 + 1, 1 * 3 + 0, 2 * 2 + 1] == pytest.approx(a[1, 0, 1, 2] * b[2, 1, 0, 1])
