"""A second, independent restatement of the reference's MGPCG in numpy, checked
against the C++ oracle.

The C++ oracle is the checker of every GPU parity test, and the reference
itself cannot run here (Taichi is not installable).  This file restates
mgpcg.py:96-238 once more in vectorised float32 numpy, written from the
reference's statements and not from the oracle's code, and requires:

* the V-cycle (smooth, restrict, prolongate, bottom sweeps; mgpcg.py:104-148)
  bit-identical to the oracle's float32 V-cycle, given the same levels'
  labels, diagonals and couplings;
* the preconditioned CG loop (mgpcg.py:150-238) to reach the oracle's float32
  solution within 1e-5 relative L2 and +-1 iteration, the bar the GPU solves
  are held to.

Vectorising a half sweep is exact: a red-black update reads only cells of the
other colour.  The restriction's child sum follows a serial execution of the
reference kernel (fine cells in row-major order, so each coarse cell adds its
children in lexicographic offset order).  The reference's own order is an
unspecified parallel atomic sum.  The inner products multiply in float32 and
sum in float64, and alpha and beta are rounded to float32 as the reference's
0-d `real` fields hold them.
"""
import numpy as np
import pytest

import mg_scenes
from oracle import OracleSolver

F32 = np.float32
FLUID = mg_scenes.FLUID


def _shift(a, k, s):
    """a[I + s e_k], zero outside the grid (the scenes keep FLUID cells off the
    edge, so no FLUID update reads outside)."""
    out = np.zeros_like(a)
    src = [slice(None)] * a.ndim
    dst = [slice(None)] * a.ndim
    if s > 0:
        src[k], dst[k] = slice(1, None), slice(0, -1)
    else:
        src[k], dst[k] = slice(0, -1), slice(1, None)
    out[tuple(dst)] = a[tuple(src)]
    return out


class NumpyMGPCG:
    """mgpcg.py's MGPCGPoissonSolver state and kernels over numpy float32 arrays."""

    def __init__(self, dim, levels, pre_post, bottom, grid_type, Adiag, Ax):
        self.dim, self.L, self.pre_post, self.bottom = dim, levels, pre_post, bottom
        self.grid_type = [np.asarray(g) for g in grid_type]
        self.Adiag = [np.asarray(a, F32) for a in Adiag]
        self.Ax = [np.asarray(a, F32) for a in Ax]
        self.r = [np.zeros(g.shape, F32) for g in self.grid_type]
        self.z = [np.zeros(g.shape, F32) for g in self.grid_type]
        self.parity = [np.indices(g.shape).sum(axis=0) & 1 for g in self.grid_type]

    def neighbor_sum(self, Ax, x):  # mgpcg.py:96-101
        ret = np.zeros_like(x)
        for i in range(self.dim):
            ret = ret + (_shift(Ax[i], i, -1) * _shift(x, i, -1) + Ax[i] * _shift(x, i, +1))
        return ret

    def smooth(self, l, phase):  # mgpcg.py:103-109
        m = (self.parity[l] == phase) & (self.grid_type[l] == FLUID)
        with np.errstate(divide="ignore", invalid="ignore"):
            new = (self.r[l] - self.neighbor_sum(self.Ax[l], self.z[l])) / self.Adiag[l]
        self.z[l] = np.where(m, new, self.z[l])

    def restrict(self, l):  # mgpcg.py:111-118
        fl = self.grid_type[l] == FLUID
        Az = self.Adiag[l] * self.z[l]
        Az = Az + self.neighbor_sum(self.Ax[l], self.z[l])
        res = self.r[l] - Az
        rc = self.r[l + 1]
        for off in np.ndindex(*((2,) * self.dim)):
            sl = tuple(slice(o, None, 2) for o in off)
            rc = np.where(fl[sl], rc + res[sl], rc)
        self.r[l + 1] = rc

    def prolongate(self, l):  # mgpcg.py:120-123
        zc = self.z[l + 1]
        for k in range(self.dim):
            zc = np.repeat(zc, 2, axis=k)
        self.z[l] = self.z[l] + zc

    def v_cycle(self):  # mgpcg.py:125-148
        self.z[0][...] = 0
        for l in range(self.L - 1):
            for _ in range(self.pre_post):
                self.smooth(l, 0)
                self.smooth(l, 1)
            self.r[l + 1][...] = 0
            self.z[l + 1][...] = 0
            self.restrict(l)
        for _ in range(self.bottom // 2):
            self.smooth(self.L - 1, 0)
            self.smooth(self.L - 1, 1)
        for _ in range(self.bottom // 2):
            self.smooth(self.L - 1, 1)
            self.smooth(self.L - 1, 0)
        for l in reversed(range(self.L - 1)):
            self.prolongate(l)
            for _ in range(self.pre_post):
                self.smooth(l, 1)
                self.smooth(l, 0)

    def reduce(self, p, q):  # mgpcg.py:211-216: float32 products, summed in float64
        fl = self.grid_type[0] == FLUID
        return float(np.sum((p * q)[fl], dtype=np.float64))

    def solve(self, b, max_iters=500, rel_tol=1e-12, abs_tol=1e-14, eps=1e-12):  # mgpcg.py:150-209
        fl = self.grid_type[0] == FLUID
        x = np.zeros_like(b)
        p = np.zeros_like(b)
        beta = F32(0.0)
        self.r[0] = b.copy()
        initial_rTr = self.reduce(self.r[0], self.r[0])
        tol = max(abs_tol, initial_rTr * rel_tol)

        def update_p():  # mgpcg.py:234-238
            return np.where(fl, self.z[0] + beta * p, p)

        self.v_cycle()
        p = update_p()
        old_zTr = self.reduce(self.z[0], self.r[0])
        it = 0
        while max_iters == -1 or it < max_iters:
            Ap = np.where(fl, self.Adiag[0] * p + self.neighbor_sum(self.Ax[0], p), 0).astype(F32)  # :218-223
            pAp = self.reduce(p, Ap)
            alpha = F32(old_zTr / (pAp + eps))
            x = np.where(fl, x + alpha * p, x)                     # :225-231
            self.r[0] = np.where(fl, self.r[0] - alpha * Ap, self.r[0])
            rTr = self.reduce(self.r[0], self.r[0])
            if rTr < tol:
                break
            self.v_cycle()
            new_zTr = self.reduce(self.z[0], self.r[0])
            beta = F32(new_zTr / (old_zTr + eps))
            p = update_p()
            old_zTr = new_zTr
            it += 1
        return x, it


SCENES = {
    "dam2d_64": lambda: mg_scenes.dam_break_2d(n=64, levels=3),
    "dam2d_64_le": lambda: mg_scenes.dam_break_2d(n=64, fluid_rule="le", gfm_clamp=1e3, levels=3),
    "dam2d_128": lambda: mg_scenes.dam_break_2d(n=128),
    "drop3d_32": lambda: mg_scenes.ferro_drop_3d(n=32, levels=3),
}


def _oracle(sc):
    o = OracleSolver(sc.dim, sc.res, sc.levels, 2, 50, real=np.float32)
    o.reinitialize_pressure(sc.cell_type, sc.velocity, sc.phi, sc.p0, sc.scale_A, sc.scale_b, True, sc.gfm_clamp)
    return o


def _numpy_from(o, sc):
    L = sc.levels
    return NumpyMGPCG(sc.dim, L, 2, 50, [o.get("grid_type", l) for l in range(L)],
                      [o.get("Adiag", l) for l in range(L)], [o.get("Ax", l) for l in range(L)])


@pytest.mark.parametrize("name", list(SCENES))
def test_vcycle_bit_identical_to_oracle(name):
    sc = SCENES[name]()
    o = _oracle(sc)
    npm = _numpy_from(o, sc)
    fl = npm.grid_type[0] == FLUID
    rng = np.random.default_rng(5)
    for _ in range(2):
        r = np.where(fl, rng.standard_normal(sc.res), 0.0).astype(F32)
        o.set("r", r, 0)
        o.v_cycle()
        z_o = o.get("z", 0)
        npm.r[0] = r.copy()
        npm.v_cycle()
        assert np.array_equal(npm.z[0].view(np.uint32), z_o.view(np.uint32)), \
            f"{int(np.sum(npm.z[0] != z_o))} cells differ"
        for l in range(1, sc.levels):  # the coarse residuals the restriction built
            assert np.array_equal(npm.r[l], o.get("r", l)), l


@pytest.mark.parametrize("name", list(SCENES))
def test_solve_matches_oracle(name):
    sc = SCENES[name]()
    o = _oracle(sc)
    b = o.get("b", 0)
    npm = _numpy_from(o, sc)
    x_np, it_np = npm.solve(b.astype(F32))
    it_o = o.solve(500)
    x_o = o.get("x", 0)
    assert abs(it_np - it_o) <= 1, (it_np, it_o)
    err = float(np.linalg.norm(x_np.astype(np.float64) - x_o) / np.linalg.norm(x_o))
    assert err <= 1e-5, err


class _PostOrderSwapped(NumpyMGPCG):
    """The restatement with one planted change: post-smoothing colours in the
    pre-smoothing order (0 then 1, where mgpcg.py:146-147 smooths 1 then 0)."""

    def smooth(self, l, phase):
        if getattr(self, "_post", False):
            phase = 1 - phase
        super().smooth(l, phase)

    def prolongate(self, l):
        self._post = True
        super().prolongate(l)

    def v_cycle(self):
        self._post = False
        super().v_cycle()


def test_bit_identity_detects_a_changed_colour_order():
    """The bit-identity check is sharp enough to see a swapped colour order."""
    sc = SCENES["drop3d_32"]()
    o = _oracle(sc)
    L = sc.levels
    bad = _PostOrderSwapped(sc.dim, L, 2, 50, [o.get("grid_type", l) for l in range(L)],
                            [o.get("Adiag", l) for l in range(L)], [o.get("Ax", l) for l in range(L)])
    fl = bad.grid_type[0] == FLUID
    r = np.where(fl, np.random.default_rng(5).standard_normal(sc.res), 0.0).astype(F32)
    o.set("r", r, 0)
    o.v_cycle()
    bad.r[0] = r.copy()
    bad.v_cycle()
    assert not np.array_equal(bad.z[0], o.get("z", 0))


# ---- the pressure Strategy's system (pressure_project.py:15-64) and the coarse
# labels (mgpcg.py:46-60), restated in float32 numpy --------------------------------

AIR, SOLID = mg_scenes.AIR, mg_scenes.SOLID


def _nb(a, k, s, fill):
    """a[I + s e_k] with `fill` outside the grid (labels: SOLID)."""
    p = np.pad(a, 1, constant_values=fill)
    sl = [slice(1, -1)] * a.ndim
    sl[k] = slice(1 + s, p.shape[k] - 1 + s)
    return p[tuple(sl)]


def _vel_at(v, k, s):
    """velocity[k][I] (s = 0) or velocity[k][I + e_k] (s = 1) on the cell grid."""
    sl = [slice(None)] * v.ndim
    sl[k] = slice(s, v.shape[k] - 1 + s)
    return v[tuple(sl)]


def numpy_build_b(sc, clamp):  # pressure_project.py:15-38 (ghost fluid method on)
    ct = sc.cell_type
    fl = ct == FLUID
    sA, sB, p0 = F32(sc.scale_A), F32(sc.scale_b), F32(sc.p0)
    phi = sc.phi.astype(F32)
    vel = [v.astype(F32) for v in sc.velocity]
    b = np.zeros(sc.res, F32)
    for k in range(sc.dim):
        b = np.where(fl, b + (_vel_at(vel[k], k, 0) - _vel_at(vel[k], k, 1)), b)
    b = np.where(fl, b * sB, b)
    with np.errstate(divide="ignore", invalid="ignore"):
        for k in range(sc.dim):
            for s in (-1, 1):
                nt = _nb(ct, k, s, SOLID)
                if s < 0:
                    b = np.where(fl & (nt == SOLID), b - sB * (_vel_at(vel[k], k, 0) - F32(0)), b)
                else:
                    b = np.where(fl & (nt == SOLID), b + sB * (_vel_at(vel[k], k, 1) - F32(0)), b)
                c = (phi - _nb(phi, k, s, F32(1))) / phi
                b = np.where(fl & (nt == AIR), b + sA * np.minimum(c, F32(clamp)) * p0, b)
    return b


def numpy_build_A(sc, grid_type, level, clamp):  # pressure_project.py:43-64
    fl = grid_type == FLUID
    sA = F32(sc.scale_A)
    phi = sc.phi.astype(F32)
    Ad = np.zeros(grid_type.shape, F32)
    Ax = np.zeros((sc.dim,) + grid_type.shape, F32)
    with np.errstate(divide="ignore", invalid="ignore"):
        for k in range(sc.dim):
            for s in (-1, 1):
                nt = _nb(grid_type, k, s, SOLID)
                Ad = np.where(fl & (nt == FLUID), Ad + sA, Ad)
                if s > 0:
                    Ax[k] = np.where(fl & (nt == FLUID), -sA, Ax[k])
                if level == 0:
                    c = (phi - _nb(phi, k, s, F32(1))) / phi
                    Ad = np.where(fl & (nt == AIR), Ad + sA * np.minimum(c, F32(clamp)), Ad)
                else:
                    Ad = np.where(fl & (nt == AIR), Ad + sA, Ad)
    return Ad, Ax


def numpy_init_gridtype(fine):  # mgpcg.py:46-60
    kids = [fine[tuple(slice(o, None, 2) for o in off)] for off in np.ndindex(*((2,) * fine.ndim))]
    any_air = np.any([k == AIR for k in kids], axis=0)
    any_fluid = np.any([k == FLUID for k in kids], axis=0)
    return np.where(any_air, AIR, np.where(any_fluid, FLUID, SOLID)).astype(np.int8)


@pytest.mark.parametrize("name", list(SCENES))
def test_pressure_system_bit_identical_to_oracle(name):
    """b, and every level's labels, Adiag and Ax, restated in float32 numpy,
    equal the float32 oracle's bit for bit."""
    sc = SCENES[name]()
    o = _oracle(sc)
    b = numpy_build_b(sc, sc.gfm_clamp)
    assert np.array_equal(b.view(np.uint32), o.get("b", 0).view(np.uint32)), int(np.sum(b != o.get("b", 0)))
    gt = sc.cell_type.astype(np.int8)
    for l in range(sc.levels):
        if l > 0:
            gt = numpy_init_gridtype(gt)
        assert np.array_equal(gt, o.get("grid_type", l)), l
        Ad, Ax = numpy_build_A(sc, gt, l, sc.gfm_clamp)
        assert np.array_equal(Ad.view(np.uint32), o.get("Adiag", l).view(np.uint32)), (l, int(np.sum(Ad != o.get("Adiag", l))))
        assert np.array_equal(Ax.view(np.uint32), o.get("Ax", l).view(np.uint32)), l


@pytest.mark.parametrize("coarse_scale", [0.5, 0.0])
def test_psi_vcycle_bit_identical_to_oracle(coarse_scale):
    """The stored-coefficient V-cycle of the magnetic potential system (every
    cell FLUID, harmonic-mean couplings, Neumann edges, a pinned cell; coarse
    levels half-Galerkin or rediscretised), float32: the numpy restatement's
    V-cycle equals the oracle's bit for bit, on the levels the oracle built."""
    n, L, dx, pin = 32, 3, 1.0 / 32, (1, 1, 1)
    rng = np.random.default_rng(13)
    chi = (rng.random((n, n, n)) < 0.4).astype(np.float32)
    o = OracleSolver(3, (n, n, n), L, 2, 50, real=np.float32)
    o.full_reinitialize_psi(chi, (0.0, 1.0, 0.0), dx, pin, coarse_scale=coarse_scale)
    npm = NumpyMGPCG(3, L, 2, 50, [o.get("grid_type", l) for l in range(L)],
                     [o.get("Adiag", l) for l in range(L)], [o.get("Ax", l) for l in range(L)])
    assert all(np.all(g == FLUID) for g in npm.grid_type)
    r = rng.standard_normal((n, n, n)).astype(F32)
    o.set("r", r, 0)
    o.v_cycle()
    npm.r[0] = r.copy()
    npm.v_cycle()
    z_o = o.get("z", 0)
    assert np.array_equal(npm.z[0].view(np.uint32), z_o.view(np.uint32)), int(np.sum(npm.z[0] != z_o))
