"""Pins the oracle of the reference's other Strategies and of the pressure
update (oracle/simulator_oracle.cpp) without the reference, which cannot run
here (Taichi is not installable):

* apply_pressure against an independent vectorised numpy restatement of
  fluid_simulator.py:193-214 (f32, bit for bit);
* the magnetic Strategy and update with H = 0 against the plain pressure
  Strategy / update (magnetic_force.py reduces to pressure_project.py);
* utils.sample against a numpy restatement through the potential operator's
  coarse-level coefficients (potential_function.py:54-55);
* structural properties: the potential and surface tension operators are
  symmetric and definite; the smoothed volume of known shapes; normals and
  curvature of planes and circles; H = H_ext - grad psi of a linear psi.
"""
import numpy as np
import pytest

from oracle import OracleSolver
from oracle import simulator as S

FLUID, AIR, SOLID = 0, 1, 2


def scene_2d(n=24, seed=0):
    rng = np.random.default_rng(seed)
    ct = np.full((n, n), AIR, np.int32)
    x, y = np.meshgrid((np.arange(n) + 0.5) / n, (np.arange(n) + 0.5) / n, indexing="ij")
    phi = (np.hypot(x - 0.5, y - 0.4) - 0.25).astype(np.float32)
    phi[np.abs(phi) < 1e-4] = 1e-4
    ct[phi <= 0] = FLUID
    ct[0, :] = ct[-1, :] = ct[:, 0] = ct[:, -1] = SOLID
    vel = [rng.uniform(-1, 1, (n + (k == 0), n + (k == 1))).astype(np.float32) for k in range(2)]
    p = rng.uniform(-1, 1, (n, n)).astype(np.float32)
    return ct, phi, vel, p


def scene_3d(n=12, seed=1):
    rng = np.random.default_rng(seed)
    g = (np.arange(n) + 0.5) / n
    x, y, z = np.meshgrid(g, g, g, indexing="ij")
    phi = np.minimum(np.sqrt((x - 0.5) ** 2 + (y - 0.6) ** 2 + (z - 0.5) ** 2) - 0.2, y - 0.3).astype(np.float32)
    phi[np.abs(phi) < 1e-4] = 1e-4
    ct = np.where(phi <= 0, FLUID, AIR).astype(np.int32)
    for k in range(3):
        sl = [slice(None)] * 3
        sl[k] = 0
        ct[tuple(sl)] = SOLID
        sl[k] = -1
        ct[tuple(sl)] = SOLID
    vel = [rng.uniform(-1, 1, tuple(n + (a == k) for a in range(3))).astype(np.float32) for k in range(3)]
    p = rng.uniform(-1, 1, (n,) * 3).astype(np.float32)
    return ct, phi, vel, p


def numpy_apply_pressure(vel, p, ct, phi, scale, p0, clamp):
    """fluid_simulator.py:193-214, vectorised in f32 (ghost fluid on)."""
    f = np.float32
    dim = ct.ndim
    out = []
    for k in range(dim):
        u = vel[k].copy()
        n = ct.shape
        pad_ct = np.concatenate([np.full(tuple(1 if a == k else n[a] for a in range(dim)), SOLID, np.int32), ct],
                                axis=k)
        pad_p = np.concatenate([np.zeros(tuple(1 if a == k else n[a] for a in range(dim)), f), p], axis=k)
        pad_phi = np.concatenate([np.ones(tuple(1 if a == k else n[a] for a in range(dim)), f), phi], axis=k)
        sl0 = tuple(slice(0, n[a]) for a in range(dim))
        t1, t = pad_ct[sl0], ct
        p1, ph1 = pad_p[sl0], pad_phi[sl0]
        uu = u[sl0]
        active = (t1 == FLUID) | (t == FLUID)
        solid = (t1 == SOLID) | (t == SOLID)
        with np.errstate(divide="ignore", invalid="ignore"):
            c_fa = (ph1 - phi) / ph1
            c_af = (phi - ph1) / phi
        fa = f(scale) * (f(p0) - p1) * np.minimum(c_fa, f(clamp))
        af = f(scale) * (p - f(p0)) * np.minimum(c_af, f(clamp))
        ff = f(scale) * (p - p1)
        new = np.where(solid, f(0), np.where(t == AIR, uu - fa, np.where(t1 == AIR, uu - af, uu - ff)))
        uu[...] = np.where(active, new, uu)
        out.append(u)
    return out


@pytest.mark.parametrize("make", [scene_2d, scene_3d])
def test_apply_pressure_matches_numpy(make):
    ct, phi, vel, p = make()
    got = S.apply_pressure(vel, p, ct, phi, 0.37, 1e-3, True, 1e3)
    ref = numpy_apply_pressure(vel, p, ct, phi, 0.37, 1e-3, 1e3)
    for g, r in zip(got, ref):
        np.testing.assert_array_equal(g.view(np.uint32), r.view(np.uint32))


def test_apply_pressure_without_ghost_fluid_and_zero_H():
    ct, phi, vel, p = scene_2d()
    plain = S.apply_pressure(vel, p, ct, phi, 0.5, 2e-3, False)
    H0 = [np.zeros_like(v) for v in vel]
    mag = S.apply_magnetic_force(vel, p, ct, H0, 0.5, 2e-3, 123.0)
    for a, b in zip(plain, mag):
        np.testing.assert_array_equal(a, b)
    # edge faces between the SOLID ring and the outside have no FLUID side: untouched
    np.testing.assert_array_equal(plain[0][0, :], vel[0][0, :])
    # faces between the SOLID ring and a FLUID cell are zeroed
    assert np.all(plain[0][1, 1:-1][ct[1, 1:-1] == FLUID] == 0.0)
    # faces with no FLUID side keep their velocity
    air_air = (ct[1:, :] != FLUID) & (ct[:-1, :] != FLUID)
    np.testing.assert_array_equal(plain[0][1:-1][air_air], vel[0][1:-1][air_air])


def test_magnetic_b_with_zero_H_is_the_pressure_b():
    ct, phi, vel, _ = scene_2d()
    o = OracleSolver(2, ct.shape, 3, 2, 50, real=np.float32)
    o.reinitialize_pressure(ct, vel, phi, 1e-3, 0.7, 3.0, False, 1e3)
    b_ref = o.get("b")
    H0 = [np.zeros_like(v) for v in vel]
    b = S.build_magnetic_b(o.get("grid_type"), vel, H0, 1e-3, 0.7, 3.0, 99.0)
    np.testing.assert_array_equal(b, b_ref)


def test_magnetic_b_air_term():
    """A uniform field H adds scale_A * coef * |H|^2 per AIR face."""
    ct, phi, vel, _ = scene_2d()
    o = OracleSolver(2, ct.shape, 3, 2, 50, real=np.float32)
    o.reinitialize_pressure(ct, vel, phi, 0.0, 0.5, 3.0, False, 1e3)
    b0 = o.get("b").astype(np.float64)
    H = [np.full(v.shape, 2.0, np.float32) for v in vel]
    b = S.build_magnetic_b(o.get("grid_type"), vel, H, 0.0, 0.5, 3.0, 0.25).astype(np.float64)
    pad = np.pad(ct, 1, constant_values=SOLID)
    n_air = sum((np.roll(pad, s, axis=a) == AIR)[1:-1, 1:-1].astype(int) for a in range(2) for s in (-1, 1))
    fl = ct == FLUID
    np.testing.assert_allclose(b[fl] - b0[fl], (0.5 * 0.25 * 8.0 * n_air)[fl], rtol=1e-5, atol=1e-5)


def numpy_sample(d, pos):
    """utils.py:12-33 restated in float64 for a cell field d at positions pos (..., dim)."""
    dim = d.ndim
    i = [np.clip(np.trunc(pos[..., a]).astype(int), 0, d.shape[a] - 1) for a in range(dim)]
    ip = [np.clip(i[a] + 1, 0, d.shape[a] - 1) for a in range(dim)]
    w = [np.clip(pos[..., a] - i[a], 0.0, 1.0) for a in range(dim)]
    out = 0.0
    for corner in np.ndindex(*(2,) * dim):
        idx = tuple(ip[a] if corner[a] else i[a] for a in range(dim))
        wt = 1.0
        for a in range(dim):
            wt = wt * (w[a] if corner[a] else 1.0 - w[a])
        out = out + wt * d[idx]
    return out


@pytest.mark.parametrize("level", [0, 1, 2])
def test_potential_A_coefficients_sample_chi(level):
    rng = np.random.default_rng(5)
    n, dx = 16, 1.0 / 16
    chi = rng.uniform(0, 5, (n, n)).astype(np.float32)
    Ad, Ax = S.build_potential_A(chi, level, dx)
    nl = n >> level
    dxl = dx * 2 ** level
    for k in range(2):
        I = np.stack(np.meshgrid(np.arange(nl), np.arange(nl), indexing="ij"), -1).astype(np.float64)
        pos = I.copy()
        pos[..., k] += 0.5
        cf = (1.0 + numpy_sample(chi.astype(np.float64), pos * 2 ** level)) / dxl
        up = I[..., k] + 2 <= n  # in_domain(I + e_k) against the fine res
        origin = (I[..., 0] == 0) & (I[..., 1] == 0)
        exp = np.where(up & ~origin, cf, 0.0)
        np.testing.assert_allclose(Ax[k], exp, rtol=2e-6, atol=0)
    assert Ad[0, 0] == np.float32(1.0 / dxl)


def assemble(Ad, Ax):
    """Dense matrix of (Adiag, Ax) with the solver's neighbour rule (mgpcg.py:96-102)."""
    shp = Ad.shape
    N = Ad.size
    idx = np.arange(N).reshape(shp)
    A = np.diag(Ad.ravel().astype(np.float64))
    for k in range(len(shp)):
        lo = [slice(None)] * len(shp)
        hi = [slice(None)] * len(shp)
        lo[k] = slice(0, -1)
        hi[k] = slice(1, None)
        a, b = idx[tuple(lo)].ravel(), idx[tuple(hi)].ravel()
        c = Ax[k][tuple(lo)].ravel().astype(np.float64)
        A[a, b] += c
        A[b, a] += c
    return A


def test_potential_A_is_negative_definite_off_the_pin():
    rng = np.random.default_rng(6)
    chi = rng.uniform(0, 5, (12, 12)).astype(np.float32)
    Ad, Ax = S.build_potential_A(chi, 0, 1.0 / 12)
    A = assemble(Ad, Ax)
    assert np.all(A[0, 1:] == 0) and np.all(A[1:, 0] == 0) and A[0, 0] > 0
    ev = np.linalg.eigvalsh(A[1:, 1:])
    assert ev.max() < 0


def test_potential_b_uniform_field():
    n = 10
    chi = np.full((n, n), 2.0, np.float32)
    H = [np.zeros((n + 1, n), np.float32), np.full((n, n + 1), 3.0, np.float32)]
    b = S.build_potential_b(chi, H)
    j = np.arange(n)
    exp_col = 6.0 * ((j + 2 <= n).astype(np.float64) - (j - 1 >= 0).astype(np.float64))
    exp = np.broadcast_to(exp_col, (n, n)).copy()
    exp[0, 0] = 0.0
    np.testing.assert_array_equal(b, exp.astype(np.float32))


def test_volume_of_known_shapes():
    n, dx = 32, 1.0 / 32
    eps = 5 * dx
    assert S.volume(np.full((n, n), -1.0, np.float32), eps) == n * n
    assert S.volume(np.full((n, n), 1.0, np.float32), eps) == 0.0
    y = (np.arange(n) + 0.5) * dx
    phi = np.broadcast_to(y - 0.4, (n, n)).astype(np.float32)  # fluid below y = 0.4
    v = S.volume(phi, eps)
    # corners sit at (j + o - 0.5) in index units (clamped at the wall): half a cell below 0.4 / dx
    assert abs(v - n * (0.4 / dx)) < 0.6 * n


def test_volume_control_steps():
    n, dx, dt = 16, 1.0 / 16, 0.01
    eps = 5 * dx
    ct = np.zeros((n, n), np.int8)
    ct[:, n // 2:] = AIR
    y = (np.arange(n) + 0.5) * dx
    phi0 = np.broadcast_to(y - 0.5, (n, n)).astype(np.float32)
    phi1 = np.broadcast_to(y - 0.45, (n, n)).astype(np.float32)
    k_p = 2.3 / (25 * dt)
    k_i = (k_p / 4) ** 2
    st = np.array([0, 0, 0, 0, 0, k_p, k_i, dt], np.float64)
    b = np.arange(n * n, dtype=np.float32).reshape(n, n) / 7
    b1, st = S.volume_control(phi0, eps, ct, b, st)
    np.testing.assert_array_equal(b1, b)  # first step only records vol_0
    assert st[0] == 1 and st[1] == S.volume(phi0, eps)
    b2, st = S.volume_control(phi1, eps, ct, b, st)
    vol1 = S.volume(phi1, eps)
    x = (vol1 - st[1]) / st[1]
    c = (-k_p * x - k_i * (x * dt)) / (x + 1)
    assert st[3] == vol1 and np.isclose(st[4], c, rtol=1e-12)
    fl = ct == FLUID
    np.testing.assert_array_equal(b2[fl], b[fl] + np.float32(c))
    np.testing.assert_array_equal(b2[~fl], b[~fl])


def test_normals_and_curvature():
    n, dx = 48, 1.0 / 48
    g = (np.arange(n) + 0.5) * dx
    x, y = np.meshgrid(g, g, indexing="ij")
    plane = (0.6 * x + 0.8 * y).astype(np.float32)
    nn = S.calc_n(plane, 0, dx)
    inner = (slice(2, -2), slice(2, -2))
    np.testing.assert_allclose(nn[0][inner], 0.6, atol=1e-4)
    np.testing.assert_allclose(nn[1][inner], 0.8, atol=1e-4)
    kap = S.calc_kappa(nn, dx)
    np.testing.assert_allclose(kap[3:-3, 3:-3], 0.0, atol=5e-2)
    R = 0.3
    circle = (np.hypot(x - 0.5, y - 0.5) - R).astype(np.float32)
    kc = S.calc_kappa(S.calc_n(circle, 1, dx), dx)
    near = np.abs(circle) < 0.5 * dx
    assert near.sum() > 20
    assert abs(np.median(kc[near]) * R - 1.0) < 0.1


def test_surface_tension_operator_spd_and_b():
    n, dx, dt, sigma = 16, 1.0 / 16, 0.01, 7.28e-2
    eps = 5 * dx
    g = (np.arange(n) + 0.5) * dx
    x, y = np.meshgrid(g, g, indexing="ij")
    phi = (np.hypot(x - 0.5, y - 0.5) - 0.3).astype(np.float32)
    for level in (0, 1):
        Ad, Ax = S.build_st_A(phi, level, 0, sigma, dt, dx, eps)
        A = assemble(Ad, Ax)
        assert np.allclose(A, A.T)
        assert np.linalg.eigvalsh(A).min() > 0
        off = np.abs(A - np.diag(np.diag(A))).sum(1)
        assert np.all(np.diag(A) >= np.float32(1 / dt) + 0.999 * off - 1e-3)
    rng = np.random.default_rng(3)
    u = rng.uniform(-1, 1, (n + 1, n)).astype(np.float32)
    nn = S.calc_n(phi, 0, dx)
    kap = S.calc_kappa(nn, dx)
    b0 = S.build_st_b(0, u, phi, nn, kap, 0.0, dt, dx, eps)
    np.testing.assert_array_equal(b0, u[:n] / np.float32(dt))
    b = S.build_st_b(0, u, phi, nn, kap, sigma, dt, dx, eps)
    I = np.stack(np.meshgrid(np.arange(n), np.arange(n), indexing="ij"), -1).astype(np.float64)
    I[..., 1] += 0.5  # delta is sampled at I + 0.5 (1 - e_d), d = 0
    far = np.abs(numpy_sample(phi.astype(np.float64), I)) >= eps * (1 + 1e-6)
    np.testing.assert_array_equal(b[far], b0[far])
    assert np.any(b[~far] != b0[~far])


def test_update_H_and_chi():
    n, dx = 8, 0.5
    psi = np.broadcast_to(np.arange(n, dtype=np.float32) * 1.5, (n, n)).T.copy()  # psi = 1.5 i
    He = [np.full((n + 1, n), 2.0, np.float32), np.full((n, n + 1), -1.0, np.float32)]
    H = S.update_H(psi, He, dx)
    np.testing.assert_array_equal(H[0][1:n], np.float32(2.0 - 3.0))
    np.testing.assert_array_equal(H[0][[0, n]], 2.0)
    np.testing.assert_array_equal(H[1], -1.0)
    eps = 0.1
    phi = np.array([[-1.0, -0.1, 0.0, 0.1, 1.0]], np.float32)
    chi = S.update_chi(phi, 5.0, eps)
    np.testing.assert_allclose(chi, [[5.0, 5.0, 2.5, 0.0, 0.0]], atol=1e-6)


# ---------------------------------------------------------------- labels, phi
def test_level_set_shapes_match_float64_sdf():
    """LevelSet.initialize_with_aabb / _sphere (level_set.py:40-64) against the
    float64 signed distances of mg_scenes, and the union rule."""
    import mg_scenes
    for dim, n in ((2, 48), (3, 20)):
        dx = 1.0 / n
        g = (np.arange(n) + 0.5) * dx
        pts = np.meshgrid(*([g] * dim), indexing="ij")
        lo, hi = np.array([0.2, 0.1, 0.3][:dim]), np.array([0.6, 0.7, 0.55][:dim])
        box = S.level_set_shape((n,) * dim, dx, False, lo, hi)
        np.testing.assert_allclose(box, mg_scenes.box_sdf(pts, lo, hi), atol=1e-6)
        c = np.array([0.5, 0.45, 0.5][:dim])
        sph = S.level_set_shape((n,) * dim, dx, True, c, 0.23)
        np.testing.assert_allclose(sph, mg_scenes.sphere_sdf(pts, c, 0.23), atol=1e-6)
        both = S.level_set_shape((n,) * dim, dx, True, c, 0.23, phi=box)
        np.testing.assert_array_equal(both, np.minimum(box, sph))


def test_apply_markers_and_boundary():
    n = 10
    phi = np.linspace(-1, 1, n * n, dtype=np.float32).reshape(n, n)
    phi[3, 3] = 0.0
    ct = S.init_boundary(np.full((n, n), AIR, np.int32))
    assert (ct[0] == SOLID).all() and (ct[:, -1] == SOLID).all() and (ct[1:-1, 1:-1] == AIR).all()
    le = S.apply_markers(ct, phi)
    lt = S.apply_markers(ct, phi, strict=True)
    inner = ct != SOLID
    np.testing.assert_array_equal(le[inner], np.where(phi[inner] <= 0, FLUID, AIR))
    np.testing.assert_array_equal(lt[inner], np.where(phi[inner] < 0, FLUID, AIR))
    assert le[3, 3] == FLUID and lt[3, 3] == AIR
    np.testing.assert_array_equal(le[~inner], SOLID)
    again = S.apply_markers(np.where(inner, FLUID, ct).astype(np.int32), phi)  # stale labels are reset
    np.testing.assert_array_equal(again, le)


def _sphere_case(dim, n):
    import mg_scenes
    dx = 1.0 / n
    g = (np.arange(n) + 0.5) * dx
    pts = np.meshgrid(*([g] * dim), indexing="ij")
    exact = mg_scenes.sphere_sdf(pts, [0.5] * dim, 0.3)
    distorted = (exact * 3 * (1 + 0.5 * pts[0])).astype(np.float32)  # same zero set, not a distance
    return dx, exact, distorted


@pytest.mark.parametrize("dim,n", [(2, 64), (3, 32)])
def test_redistance_restores_distance(dim, n):
    """FastSweepingLevelSet.redistance (level_set.py:260-334): interface cells
    get the linear-crossing distance (target_surface, restated in numpy here),
    the rest the sweeps' upwind distance; within 5 dx of the interface the
    result is within 0.4 dx of the exact distance, and signs are kept."""
    dx, exact, phi = _sphere_case(dim, n)
    out, valid = S.redistance(phi, dx, 2)
    assert np.all(np.sign(out) == np.sign(phi))
    band = np.abs(exact) < 5 * dx
    assert np.abs(out - exact)[band].max() < 0.4 * dx
    # target_surface in numpy
    f = np.float32
    est = np.full(phi.shape, f(1e20))
    change = np.zeros(phi.shape, bool)
    for k in range(dim):
        for s in (-1, 1):
            q = np.roll(phi, -s, axis=k)
            inb = np.ones(phi.shape, bool)
            idx = [slice(None)] * dim
            idx[k] = -1 if s > 0 else 0
            inb[tuple(idx)] = False
            sc = inb & (np.sign(phi) != np.sign(q))
            with np.errstate(divide="ignore", invalid="ignore"):
                e0 = (np.sign(phi).astype(f) * (phi / (phi - q))).astype(f) * f(dx)
            take = sc & (np.abs(e0) < np.abs(est))
            est = np.where(take, e0, est)
            change |= sc
    np.testing.assert_array_equal(valid == 0, change)
    np.testing.assert_array_equal(out[change].view(np.uint32), est[change].astype(np.float32).view(np.uint32))


# ---------------------------------------------------- advection, extrapolation
def _markers_serial(shape, mk, dx, repeat=2):
    """distance_to_markers + markers_propagate (level_set.py:114-122, 336-379)
    restated with float32 scalars, markers in index order, lines in order."""
    dim = len(shape)
    dx = np.float32(dx)
    phi = np.full(shape, np.float32(1e20), np.float32)
    valid = np.full(shape, -1, np.int32)

    def dist(m, c):
        s = np.float32(0)
        for a in range(dim):
            diff = np.float32(np.float32(m[a]) - (np.float32(c[a]) + np.float32(0.5)) * dx)
            s = np.float32(diff * diff) if a == 0 else np.float32(s + diff * diff)
        return np.float32(np.sqrt(s))

    for p, m in enumerate(mk):
        c = [int(np.float32(m[a]) / dx) for a in range(dim)]  # truncation toward zero
        if all(0 <= c[a] < shape[a] for a in range(dim)):
            d = dist(m, c)
            if d < phi[tuple(c)]:
                phi[tuple(c)] = d
                valid[tuple(c)] = p
    for _ in range(repeat):
        for axis in reversed(range(dim)):
            for dr in (1, -1):
                for idx in np.ndindex(*[shape[a] if a != axis else 1 for a in range(dim)]):
                    for step in range(shape[axis]):
                        c = list(idx)
                        c[axis] = step if dr > 0 else shape[axis] - 1 - step
                        nc = list(c)
                        nc[axis] += dr
                        if not 0 <= nc[axis] < shape[axis]:
                            continue
                        v = valid[tuple(nc)]
                        if v < 0:
                            continue
                        d = dist(mk[v], c)
                        if d < phi[tuple(c)]:
                            phi[tuple(c)] = d
                            valid[tuple(c)] = v
    return phi, valid


def _marker_cloud(shape, dx, n, seed):
    rng = np.random.default_rng(seed)
    ext = np.array(shape, np.float64) * dx
    mk = rng.uniform(0.2, 0.7, (n, len(shape))) * ext
    extra = np.array([mk[0] + 1e-4 * dx, -0.3 * np.ones(len(shape)) * dx, ext + dx], np.float64)  # same cell; truncation; outside
    return np.concatenate([mk, extra]).astype(np.float32)


@pytest.mark.parametrize("shape", [(7, 6, 5), (9, 8)])
def test_markers_distance_matches_serial_restatement(shape):
    """FastSweepingLevelSet.build_from_markers' first part: the oracle against an
    independent float32-scalar restatement, bit for bit (a marker just outside
    the lower faces lands in cell 0 by truncation; one far outside is ignored;
    two markers share a cell)."""
    dx = 0.1
    mk = _marker_cloud(shape, dx, 9, 5)
    phi, valid = S.markers_distance(shape, mk, dx, 2)
    rphi, rvalid = _markers_serial(shape, mk, dx, 2)
    np.testing.assert_array_equal(phi, rphi)
    np.testing.assert_array_equal(valid, rvalid)
    assert valid[(0,) * len(shape)] == len(mk) - 2  # the truncated marker
    assert (phi < 1e20).sum() > len(mk) - 2


def test_target_minus_and_smoothing_match_numpy():
    rng = np.random.default_rng(7)
    shape = (6, 7, 8)
    dx = 0.05
    phi0 = rng.uniform(-2, 2, shape).astype(np.float32) * np.float32(dx)
    phi, temp, valid = S.target_minus(phi0, dx)
    ref = (phi0 - np.float32(0.99 * dx)).astype(np.float32)
    np.testing.assert_array_equal(phi, ref)
    sg = np.sign(ref)
    change = np.zeros(shape, bool)
    for k in range(3):
        for s in (-1, 1):
            sh = np.roll(sg, -s, axis=k)
            m = np.ones(shape, bool)
            idx = [slice(None)] * 3
            idx[k] = slice(-1, None) if s > 0 else slice(0, 1)
            m[tuple(idx)] = False
            change |= m & (sh != sg)
    exp_temp = np.where(ref > 0, ref, np.where(change, ref, np.float32(-1))).astype(np.float32)
    exp_valid = np.where((ref > 0) | change, 0, -1)
    np.testing.assert_array_equal(temp, exp_temp)
    np.testing.assert_array_equal(valid, exp_valid)
    # smoothing: min(mean of the in-range axis neighbours, self), summed axis by axis
    src = rng.uniform(-1, 1, shape).astype(np.float32)
    tot = np.zeros(shape, np.float32)
    cnt = np.zeros(shape, np.int32)
    for k in range(3):
        for s in (-1, 1):
            nb = np.roll(src, -s, axis=k)
            m = np.ones(shape, bool)
            idx = [slice(None)] * 3
            idx[k] = slice(-1, None) if s > 0 else slice(0, 1)
            m[tuple(idx)] = False
            tot = np.where(m, (tot + nb).astype(np.float32), tot)
            cnt += m
    avg = (tot / cnt.astype(np.float32)).astype(np.float32)
    np.testing.assert_array_equal(S.ls_smooth(src), np.minimum(avg, src))


def test_build_from_markers_fills_a_ball():
    """A ball filled with markers (4 a cell): negative inside, about the
    distance to the ball minus the marker radius just outside."""
    n = 24
    dx = 1.0 / n
    g = (np.arange(n) + 0.5) * dx
    X = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    rng = np.random.default_rng(3)
    pts = np.concatenate([X + rng.uniform(-0.45, 0.45, X.shape) * dx for _ in range(4)])
    inside = np.linalg.norm(pts - 0.5, axis=1) < 0.25
    phi = S.build_from_markers((n, n, n), pts[inside].astype(np.float32), dx)
    r = np.linalg.norm(X.reshape(n, n, n, 3) - 0.5, axis=-1)
    assert (phi[r < 0.2] < 0).all()
    band = (r > 0.3) & (r < 0.33)
    assert (phi[band] > 0).all() and (phi[band] < 3 * dx).all()


def test_advect_identity_and_translation():
    """advect (fluid_simulator.py:216-221): zero velocity leaves a field
    unchanged (up to the f32 round trip (I + 0.5) dx / dx - 0.5, an ulp off I,
    which mixes in neighbours with weights ~1e-7); a uniform velocity
    translates a linear field."""
    n, dx, dt = 24, 1.0 / 24, 0.01
    rng = np.random.default_rng(1)
    zero = [np.zeros((n + (k == 0), n + (k == 1)), np.float32) for k in range(2)]
    f = rng.standard_normal((n, n)).astype(np.float32)
    np.testing.assert_allclose(S.advect(zero, f, -1, dx, dt), f, rtol=0, atol=1e-5)
    u0 = rng.standard_normal((n + 1, n)).astype(np.float32)
    np.testing.assert_allclose(S.advect(zero, u0, 0, dx, dt), u0, rtol=0, atol=1e-5)
    c = (0.7, -0.4)
    vel = [np.full((n + (k == 0), n + (k == 1)), c[k], np.float32) for k in range(2)]
    x, y = np.meshgrid((np.arange(n) + 0.5) * dx, (np.arange(n) + 0.5) * dx, indexing="ij")
    lin = (2 * x + 3 * y).astype(np.float32)
    out = S.advect(vel, lin, -1, dx, dt)
    exact = 2 * (x - c[0] * dt) + 3 * (y - c[1] * dt)
    np.testing.assert_allclose(out[2:-2, 2:-2], exact[2:-2, 2:-2], atol=1e-5)


def test_extrapolate_matches_numpy():
    """extrap_velocity (fluid_simulator.py:244-272) against a vectorised numpy
    restatement of mark_valid and diffuse_quantity."""
    rng = np.random.default_rng(3)
    for dim, n in ((2, 20), (3, 10)):
        ct = np.full((n,) * dim, AIR, np.int32)
        ct[tuple(slice(n // 4, n // 2) for _ in range(dim))] = FLUID
        for k in range(dim):
            shp = tuple(n + (a == k) for a in range(dim))
            u = rng.standard_normal(shp).astype(np.float32)
            got, gvalid = S.extrapolate(u, k, ct, 10)
            # numpy: faces beside FLUID are valid
            pad = np.full(tuple(s + 2 for s in shp), False)
            fl = ct == FLUID
            lo = [slice(1, -1)] * dim
            hi = [slice(1, -1)] * dim
            valid = np.zeros(shp, bool)
            sl_hi = tuple(slice(0, n) if a == k else slice(None) for a in range(dim))
            sl_lo = tuple(slice(1, n + 1) if a == k else slice(None) for a in range(dim))
            valid[sl_hi] |= fl
            valid[sl_lo] |= fl
            uu = u.copy()
            for _ in range(10):
                src, vs = uu.copy(), valid.copy()
                ps = np.pad(src, 1)
                pv = np.pad(vs, 1)
                tot = np.zeros(shp, np.float32)
                cnt = np.zeros(shp, np.int32)
                for off in np.ndindex(*(3,) * dim):
                    sl = tuple(slice(o, o + s) for o, s in zip(off, shp))
                    tot = (tot + np.where(pv[sl], ps[sl], np.float32(0))).astype(np.float32)
                    cnt += pv[sl]
                fill = (~vs) & (cnt > 0)
                with np.errstate(divide="ignore", invalid="ignore"):
                    uu = np.where(fill, (tot / cnt.astype(np.float32)).astype(np.float32), uu)
                valid = vs | fill
            np.testing.assert_array_equal(gvalid.astype(bool), valid)
            np.testing.assert_array_equal(got.view(np.uint32), uu.view(np.uint32))


def test_boundary_and_gravity():
    n = 8
    rng = np.random.default_rng(4)
    ct = S.init_boundary(np.full((n, n), AIR, np.int32))
    vel = [rng.standard_normal((n + (k == 0), n + (k == 1))).astype(np.float32) for k in range(2)]
    out = S.enforce_boundary(vel, ct)
    solid = ct == SOLID
    for k in range(2):
        lo = tuple(slice(0, n) if a == k else slice(None) for a in range(2))
        hi = tuple(slice(1, n + 1) if a == k else slice(None) for a in range(2))
        touched = np.zeros(out[k].shape, bool)
        touched[lo] |= solid
        touched[hi] |= solid
        np.testing.assert_array_equal(out[k][touched], 0.0)
        np.testing.assert_array_equal(out[k][~touched], vel[k][~touched])
    g = S.add_gravity(vel, (0.0, -9.8), np.float32(1 / 60))
    np.testing.assert_array_equal(g[0], vel[0])
    np.testing.assert_array_equal(g[1], vel[1] + np.float32(-9.8) * np.float32(1 / 60))
