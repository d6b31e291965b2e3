"""The Kitaev workload's structure as a parity case: a 4x4 unit cell of
complex tensors on the brick-wall mapping of the honeycomb lattice (every
site has one vertical leg of dimension 1, so the left / right moves take the
identity projector of ctm.cpp:303-317), the other bond dimensions drawn from
{2, 3} by the seed (so neighbouring sites differ), CTMRG with the reference's
full-SVD corner projectors, GPU against the oracle: corner spectra and the
Kitaev bond energies with a [111] field."""
import numpy as np
import pytest

from oracle import tenes_oracle as O
from tests._helpers import SX, SY, SZ, gpu_env, oracle_params, random_tensors

pytestmark = pytest.mark.gpu


def brick_wall_lattice(LX=4, LY=4, seed=5, dims=(2, 3)):
    rng = np.random.default_rng(seed)
    lat = O.Lattice(LX, LY)
    N = LX * LY
    lat.physical_dims = [2] * N
    vd = [[0] * 4 for _ in range(N)]
    for y in range(LY):
        for x in range(LX):
            i = x + y * LX
            r = lat.right(i)
            vd[i][2] = vd[r][0] = int(rng.choice(dims))  # horizontal bond
    for y in range(LY):
        for x in range(LX):
            i = x + y * LX
            t = lat.top(i)
            # vertical bond present between a parity-1 site and the site above it
            D = int(rng.choice(dims)) if (x + y) % 2 == 1 else 1
            vd[i][1] = vd[t][3] = D
    lat.virtual_dims = vd
    return lat


def kitaev_bonds(lat):
    """(site, dx, dy, op): x / y bonds alternate along rows, z bonds on the
    present vertical legs; K = 1, op = -K S^a S^a."""
    out = []
    for i in range(lat.N_UNIT):
        x, y = i % lat.LX, i // lat.LX
        S = SX if (x + y) % 2 == 0 else SY
        out.append((i, 1, 0, -np.einsum("ac,bd->abcd", S, S)))
        if lat.virtual_dims[i][1] > 1:
            out.append((i, 0, 1, -np.einsum("ac,bd->abcd", SZ, SZ)))
    return out


def oracle_bond(oe, Tn, lat, s, dx, dy, op):
    e = oe
    if dy == 0:
        l, r = s, lat.other(s, 1, 0)
        return O.contract_two_sites_horizontal_op12(e.C1[l], e.C2[r], e.C3[r], e.C4[l], e.eTt[l], e.eTt[r],
                                                    e.eTr[r], e.eTb[r], e.eTb[l], e.eTl[l], Tn[l], Tn[r], op)
    t, b = lat.other(s, 0, 1), s
    return O.contract_two_sites_vertical_op12(e.C1[t], e.C2[t], e.C3[b], e.C4[b], e.eTt[t], e.eTr[t],
                                              e.eTr[b], e.eTb[b], e.eTl[b], e.eTl[t], Tn[t], Tn[b],
                                              op.transpose(1, 0, 3, 2))


def test_kitaev_brick_wall_complex_4x4():
    lat = brick_wall_lattice()
    assert any(v[1] == 1 for v in lat.virtual_dims) and len({v[2] for v in lat.virtual_dims}) > 1
    Tn = random_tensors(lat, 17, is_complex=True)
    chi, iters = 8, 3
    oe, ocnt, _, _ = O.calc_ctm_environment(Tn, oracle_params(chi, Max_CTM_Iteration=iters), lat)
    ge = gpu_env(lat, Tn, chi, True, max_ctm_iteration=iters)
    gcnt, _, _ = ge.calc_ctm_environment(True)
    assert gcnt == ocnt
    for w, name in enumerate(("C1", "C2", "C3", "C4")):
        for i in range(lat.N_UNIT):
            np.testing.assert_allclose(ge.corner_spectrum(w, i), O.corner_spectrum(getattr(oe, name)[i]),
                                       rtol=1e-9, atol=1e-12, err_msg=f"{name}[{i}]")
    ident = np.einsum("ac,bd->abcd", np.eye(2), np.eye(2))
    h = (SX + SY + SZ) * 0.05
    for (s, dx, dy, op) in kitaev_bonds(lat):
        g = ge.contract_bond_op12(s, dx, dy, op) / ge.contract_bond_op12(s, dx, dy, ident)
        o = oracle_bond(oe, Tn, lat, s, dx, dy, op) / oracle_bond(oe, Tn, lat, s, dx, dy, ident)
        assert abs(g - o) <= 1e-9 * max(abs(o), 1e-3), (s, dx, dy, g, o)
    for i in range(lat.N_UNIT):
        g = ge.contract_one_site(i, h) / ge.contract_one_site(i, np.eye(2))
        e = oe
        o = (O.contract_one_site(e.C1[i], e.C2[i], e.C3[i], e.C4[i], e.eTt[i], e.eTr[i], e.eTb[i], e.eTl[i],
                                 Tn[i], h)
             / O.contract_one_site(e.C1[i], e.C2[i], e.C3[i], e.C4[i], e.eTt[i], e.eTr[i], e.eTb[i], e.eTl[i],
                                   Tn[i], np.eye(2)))
        assert abs(g - o) <= 1e-9 * max(abs(o), 1e-3)


def test_kitaev_c5_shapes_ctm_energy_and_flux():
    """The Kitaev workload at its own shapes: 4x4 brick wall, per-bond D drawn
    from {3, 4, 5} by the seed, chi = 48, complex site tensors with i.i.d.
    uniform[-1, 1] parts; three CTMRG iterations with the reference's full-SVD
    corner projectors on both sides, then the corner spectra, every Kitaev bond
    term and the plaquette flux W_p = <prod sigma> of the cell's eight
    hexagons (2 x 3 windows), GPU against the oracle."""
    import bench
    vd = bench.brick_wall_dims(dims=(3, 4, 5))
    lat = O.Lattice(4, 4)
    lat.physical_dims = [2] * 16
    lat.virtual_dims = vd
    Tn = bench.random_complex_tensors(vd, 11)
    chi, iters = 48, 3
    oe, ocnt, _, _ = O.calc_ctm_environment(Tn, oracle_params(chi, Max_CTM_Iteration=iters), lat)
    ge = gpu_env(lat, Tn, chi, True, max_ctm_iteration=iters)
    gcnt, _, _ = ge.calc_ctm_environment(True)
    assert gcnt == ocnt
    for w, name in enumerate(("C1", "C2", "C3", "C4")):
        for i in range(lat.N_UNIT):
            g, o = ge.corner_spectrum(w, i), O.corner_spectrum(getattr(oe, name)[i])
            g = g[:len(o)] if len(g) > len(o) else g
            err = np.linalg.norm(g - o[:len(g)]) / np.linalg.norm(o)
            assert err <= 1e-9, (name, i, err)
    ident = np.einsum("ac,bd->abcd", np.eye(2), np.eye(2))
    for (s, dx, dy, op) in kitaev_bonds(lat):
        g = ge.contract_bond_op12(s, dx, dy, op) / ge.contract_bond_op12(s, dx, dy, ident)
        o = oracle_bond(oe, Tn, lat, s, dx, dy, op) / oracle_bond(oe, Tn, lat, s, dx, dy, ident)
        assert abs(g - o) <= 1e-9 * max(abs(o), 1e-3), (s, dx, dy, g, o)
    starts, ops = bench.hexagons()
    for s in starts:
        _, Cs, eTt, eTr, eTb, eTl, T = O._window(oe, Tn, lat, s, 0, 1, 2, 3)
        grid = [[ops.get((r, c), np.eye(2)) for c in range(3)] for r in range(2)]
        o = (O.contract_window(Cs, eTt, eTr, eTb, eTl, T, grid)
             / O.contract_window(Cs, eTt, eTr, eTb, eTl, T, [[np.eye(2)] * 3 for _ in range(2)]))
        g = ge.contract_window(s, 2, 3, 1, 0, ops) / ge.contract_window(s, 2, 3, 1, 0)
        assert abs(g - o) <= 1e-9 * max(abs(o), 1e-3), (s, g, o)
    ge.close()
