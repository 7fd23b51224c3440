"""Pins the CPU oracle (a restatement of mgpcg.py / pressure_project.py)
without the reference, which cannot run here (Taichi is not installable):

* the assembled system against an independent numpy assembly written from the
  formulas of pressure_project.py:15-64;
* the solution against scipy's sparse direct solver (FP64);
* the V-cycle preconditioner (mgpcg.py:125-148) against its defining
  properties: linear, symmetric, positive definite on FLUID cells;
* coarse labels against init_gridtype's rule (mgpcg.py:46-60);
* the committed golden fixtures.
"""
import os

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import mg_scenes
from oracle import OracleSolver

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def build(sc, real=np.float64, levels=None, clamp=None):
    o = OracleSolver(sc.dim, sc.res, levels or sc.levels, 2, 50, real=real)
    o.reinitialize_pressure(sc.cell_type, sc.velocity, sc.phi, sc.p0, sc.scale_A, sc.scale_b, True,
                            sc.gfm_clamp if clamp is None else clamp)
    return o


def numpy_assembly(sc, clamp):
    """pressure_project.py:15-64 at level 0, vectorised, float64."""
    ct = sc.cell_type
    dim = sc.dim
    fl = ct == mg_scenes.FLUID
    pad = np.pad(ct, 1, constant_values=mg_scenes.SOLID)
    phip = np.pad(sc.phi.astype(np.float64), 1, constant_values=1.0)
    sA, sB, p0 = sc.scale_A, sc.scale_b, sc.p0
    b = np.zeros(sc.res)
    Ad = np.zeros(sc.res)
    Ax = np.zeros((dim,) + sc.res)
    vel = [v.astype(np.float64) for v in sc.velocity]
    div = np.zeros(sc.res)
    for k in range(dim):
        lo = [slice(None)] * dim
        hi = [slice(None)] * dim
        lo[k] = slice(0, -1)
        hi[k] = slice(1, None)
        div += vel[k][tuple(lo)] - vel[k][tuple(hi)]
    b = np.where(fl, div * sB, 0.0)
    centre = tuple(slice(1, -1) for _ in range(dim))
    phi = sc.phi.astype(np.float64)
    for k in range(dim):
        for s in (-1, 1):
            sl = [slice(1, -1)] * dim
            sl[k] = slice(1 + s, pad.shape[k] - 1 + s)
            nt = pad[tuple(sl)]
            nphi = phip[tuple(sl)]
            solid = fl & (nt == mg_scenes.SOLID)
            air = fl & (nt == mg_scenes.AIR)
            flu = fl & (nt == mg_scenes.FLUID)
            if s < 0:
                lo = [slice(None)] * dim
                lo[k] = slice(0, -1)
                b = b - np.where(solid, sB * vel[k][tuple(lo)], 0.0)
            else:
                hi = [slice(None)] * dim
                hi[k] = slice(1, None)
                b = b + np.where(solid, sB * vel[k][tuple(hi)], 0.0)
            c = np.minimum((phi - nphi) / np.where(phi == 0, 1, phi), clamp)
            b = b + np.where(air, sA * c * p0, 0.0)
            Ad += np.where(flu, sA, 0.0) + np.where(air, sA * c, 0.0)
            if s > 0:
                Ax[k] = np.where(flu, -sA, Ax[k])
    _ = centre
    return b, Ad, Ax


def sparse_matrix(grid_type, Adiag, Ax):
    fl = grid_type == 0
    idx = -np.ones(fl.shape, np.int64)
    idx[fl] = np.arange(fl.sum())
    rows = [idx[fl]]
    cols = [idx[fl]]
    vals = [Adiag[fl]]
    dim = fl.ndim
    for k in range(dim):
        lo = [slice(None)] * dim
        hi = [slice(None)] * dim
        lo[k] = slice(0, -1)
        hi[k] = slice(1, None)
        a = Ax[k][tuple(lo)]
        m = (a != 0) & fl[tuple(lo)] & fl[tuple(hi)]
        i0 = idx[tuple(lo)][m]
        i1 = idx[tuple(hi)][m]
        rows += [i0, i1]
        cols += [i1, i0]
        vals += [a[m], a[m]]
    n = int(fl.sum())
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))


SCENES = {
    "dam2d_64": lambda: mg_scenes.dam_break_2d(n=64, levels=3),
    "dam2d_128": lambda: mg_scenes.dam_break_2d(n=128),
    "dam2d_64_le": lambda: mg_scenes.dam_break_2d(n=64, fluid_rule="le", gfm_clamp=1e3, levels=3),
    "drop3d_32": lambda: mg_scenes.ferro_drop_3d(n=32, levels=3),
}


@pytest.mark.parametrize("name", list(SCENES))
def test_assembly_matches_numpy(name):
    sc = SCENES[name]()
    o = build(sc)
    b, Ad, Ax = numpy_assembly(sc, sc.gfm_clamp)
    np.testing.assert_allclose(o.get("b"), b, rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(o.get("Adiag"), Ad, rtol=1e-12, atol=0)
    np.testing.assert_allclose(o.get("Ax"), Ax, rtol=1e-12, atol=0)


@pytest.mark.parametrize("name", list(SCENES))
def test_fp64_solution_matches_scipy(name):
    sc = SCENES[name]()
    o = build(sc)
    it = o.solve(1000, rel_tol=1e-24)
    assert o.last_rTr < 1e-24 * o.last_rTr0 or o.last_rTr < 1e-14
    A = sparse_matrix(o.get("grid_type"), o.get("Adiag"), o.get("Ax"))
    fl = o.get("grid_type") == 0
    xs = spla.spsolve(A.tocsc(), o.get("b")[fl])
    x = o.get("x")[fl]
    assert np.linalg.norm(x - xs) / np.linalg.norm(xs) < 1e-8
    assert it < 60


def _vcycle(o, r):
    o.set("r", r, 0)
    o.v_cycle()
    return o.get("z", 0)


@pytest.mark.parametrize("name", ["dam2d_64", "drop3d_32", "dam2d_64_le"])
def test_vcycle_linear_symmetric_positive(name):
    sc = SCENES[name]()
    o = build(sc)
    fl = o.get("grid_type") == 0
    rng = np.random.default_rng(11)
    u = np.where(fl, rng.standard_normal(sc.res), 0.0)
    v = np.where(fl, rng.standard_normal(sc.res), 0.0)
    Mu, Mv = _vcycle(o, u), _vcycle(o, v)
    Muv = _vcycle(o, 2.0 * u - 3.0 * v)
    np.testing.assert_allclose(Muv[fl], (2.0 * Mu - 3.0 * Mv)[fl], rtol=1e-9, atol=1e-9 * np.abs(Mu).max())
    a, b = float(np.sum(v[fl] * Mu[fl])), float(np.sum(u[fl] * Mv[fl]))
    assert abs(a - b) <= 1e-10 * max(abs(a), abs(b))
    assert float(np.sum(u[fl] * Mu[fl])) > 0 and float(np.sum(v[fl] * Mv[fl])) > 0


@pytest.mark.parametrize("name", list(SCENES))
def test_coarse_labels_follow_init_gridtype(name):
    sc = SCENES[name]()
    o = build(sc)
    for l in range(1, sc.levels):
        f = o.get("grid_type", l - 1)
        shp = tuple(n // 2 for n in f.shape)
        blocks = f.reshape(sum(((n, 2) for n in shp), ())).transpose(
            tuple(range(0, 2 * sc.dim, 2)) + tuple(range(1, 2 * sc.dim, 2))).reshape(shp + (-1,))
        exp = np.where((blocks == mg_scenes.AIR).any(-1), mg_scenes.AIR,
                       np.where((blocks == mg_scenes.FLUID).any(-1), mg_scenes.FLUID, mg_scenes.SOLID))
        np.testing.assert_array_equal(o.get("grid_type", l), exp)


def test_f32_solve_within_tolerance_of_f64():
    sc = SCENES["dam2d_128"]()
    o32 = build(sc, real=np.float32)
    it32 = o32.solve(500)
    o64 = build(sc)
    o64.solve(1000, rel_tol=1e-24)
    x32, x64 = o32.get("x"), o64.get("x")
    assert np.linalg.norm(x32 - x64) / np.linalg.norm(x64) < 1e-4
    o32b = build(sc, real=np.float32)
    assert abs(o32b.solve(500, acc_mode=0) - it32) <= 1


@pytest.mark.parametrize("fname", sorted(f for f in os.listdir(GOLDEN) if f.endswith(".npz")))
def test_golden_fixture_reproduced(fname):
    g = np.load(os.path.join(GOLDEN, fname))
    dim, res, L = int(g["dim"]), tuple(int(v) for v in g["res"]), int(g["levels"])
    vel = [g[f"vel{k}"] for k in range(dim)]
    sA = float(g["dt"]) / (float(g["rho"]) * float(g["dx"]) ** 2)
    o = OracleSolver(dim, res, L, 2, 50, real=np.float32)
    o.reinitialize_pressure(g["cell_type"], vel, g["phi"], float(g["p0"]), sA, 1.0 / float(g["dx"]), True,
                            float(g["gfm_clamp"]))
    for l in range(L):
        np.testing.assert_array_equal(o.get("grid_type", l), g[f"grid_type{l}"])
        np.testing.assert_array_equal(o.get("Adiag", l), g[f"Adiag{l}"])
        np.testing.assert_array_equal(o.get("Ax", l), g[f"Ax{l}"])
    np.testing.assert_array_equal(o.get("b"), g["b"])
    assert o.solve(500) == int(g["iters_f32"])
    np.testing.assert_array_equal(o.get("x"), g["x_f32"])


def test_oracle_rejects_uneven_levels():
    with pytest.raises(ValueError):
        OracleSolver(2, (100, 64), 4)


def _psi_numpy(chi, dx, pin):
    """Independent numpy assembly of the magnetic potential operator of one
    level: harmonic-mean mu faces over dx^2, Neumann boundary, the pinned row
    the identity over dx^2 and the couplings into the pinned cell removed.
    Returns (Adiag, Ax[k] as the + side coupling)."""
    mu = 1.0 + chi.astype(np.float64)
    dim = chi.ndim
    ad = np.zeros(chi.shape)
    ax = np.zeros((dim,) + chi.shape)
    for k in range(dim):
        lo = [slice(None)] * dim
        hi = [slice(None)] * dim
        lo[k] = slice(0, -1)
        hi[k] = slice(1, None)
        lo, hi = tuple(lo), tuple(hi)
        f = 2.0 * mu[lo] * mu[hi] / (mu[lo] + mu[hi]) / (dx * dx)
        ad[lo] += f
        ad[hi] += f
        ax[k][lo] = -f
        # couplings into the pinned cell are removed (its row is the identity)
        pk = list(pin)
        pk[k] -= 1
        if pk[k] >= 0:
            ax[k][tuple(pk)] = 0.0
    ad[tuple(pin)] = 1.0 / (dx * dx)
    for k in range(dim):
        ax[k][tuple(pin)] = 0.0
    return ad, ax


@pytest.mark.parametrize("coarse", ["galerkin", "rediscretise"])
def test_psi_operator_matches_numpy(coarse):
    """The magnetic potential operator of the 3D substep benchmark in the
    FP64 oracle against an independent numpy assembly: level 0, then level 1
    either as half the Galerkin operator (P piecewise constant, R its
    transpose) or rediscretised (chi the mean of the children, dx * 2, the
    pin's coarse cell), as potential_function.py:39-55 rebuilds its levels."""
    n, L, dx, pin = 16, 3, 1.0 / 16, (1, 1, 1)
    rng = np.random.default_rng(9)
    chi = (rng.random((n, n, n)) < 0.4).astype(np.float64)
    o = OracleSolver(3, (n, n, n), L, 2, 50, real=np.float64)
    o.full_reinitialize_psi(chi, (0.0, 1.0, 0.0), dx, pin, coarse_scale=0.5 if coarse == "galerkin" else 0.0)
    ad0, ax0 = _psi_numpy(chi, dx, pin)
    np.testing.assert_allclose(o.get("Adiag", 0), ad0, rtol=1e-12)
    np.testing.assert_allclose(o.get("Ax", 0), ax0, rtol=1e-12, atol=0)
    if coarse == "rediscretise":
        chi1 = chi.reshape(n // 2, 2, n // 2, 2, n // 2, 2).mean(axis=(1, 3, 5))
        ad1, ax1 = _psi_numpy(chi1, 2 * dx, tuple(p >> 1 for p in pin))
    else:
        # 1/2 P^T A P: the coarse diagonal sums the children's diagonals and
        # twice the couplings between children; the coarse + coupling sums the
        # children's couplings across the coarse face
        m = n // 2
        ad1 = np.zeros((m, m, m))
        ax1 = np.zeros((3, m, m, m))
        for off in np.ndindex(2, 2, 2):
            ch = tuple(slice(off[a], None, 2) for a in range(3))
            ad1 += ad0[ch]
            for k in range(3):
                if off[k] == 0:
                    ad1 += 2.0 * ax0[k][ch]
                else:
                    ax1[k] += ax0[k][ch]
        for k in range(3):
            sl = [slice(None)] * 3
            sl[k] = m - 1
            ax1[k][tuple(sl)] = 0.0
        ad1 *= 0.5
        ax1 *= 0.5
    np.testing.assert_allclose(o.get("Adiag", 1), ad1, rtol=1e-12)
    np.testing.assert_allclose(o.get("Ax", 1), ax1, rtol=1e-12, atol=1e-9)
