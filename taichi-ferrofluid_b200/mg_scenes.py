"""Seeded synthetic Poisson scenes for the MGPCG pressure path.

The reference has no dataset or benchmark inputs; its simulators build
cell_type, phi and MAC velocities on the fly.  These generators produce the
same kinds of fields with numpy's ``default_rng`` so that every solve here is
reproducible:

* labels follow ``utils.py:4-6`` (FLUID=0, AIR=1, SOLID=2);
* a one-cell SOLID wall ring as ``FluidSimulator.init_boundary``
  (fluid_simulator.py:337-341);
* FLUID where phi < 0 (``fluid_rule="lt"``) or phi <= 0 as the reference's
  ``apply_markers`` (fluid_simulator.py:151-159, ``fluid_rule="le"``);
* phi sampled at cell centres (I + 0.5) * dx as ``LevelSet.initialize_with_*``
  (level_set.py:40-64);
* face velocity k has shape res + e_k (fluid_simulator.py:75-76).

Axis 0 is x, axis 1 is y (gravity axis), axis 2 is z; arrays are row-major
with the last axis fastest, as Taichi's dense fields.
"""
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

FLUID, AIR, SOLID = 0, 1, 2


@dataclass
class Scene:
    """One pressure solve's inputs: what a simulator hands the solver."""
    dim: int
    res: tuple
    dx: float
    dt: float
    rho: float
    p0: float
    phi: np.ndarray                      # float32, shape res
    cell_type: np.ndarray                # int32, shape res
    velocity: List[np.ndarray]           # float32, shape res + e_k
    levels: int = 4
    gfm_clamp: float = 100.0             # theta >= 0.01
    extra_rhs: Optional[np.ndarray] = None   # added to b on FLUID cells (float32)
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def scale_A(self) -> float:
        """fluid_simulator.py:178, dt / (rho dx^2)."""
        return self.dt / (self.rho * self.dx * self.dx)

    @property
    def scale_b(self) -> float:
        """fluid_simulator.py:179, 1 / dx."""
        return 1.0 / self.dx

    @property
    def cells(self) -> int:
        return int(np.prod(self.res))


def cell_centres(res, dx):
    axes = [(np.arange(n, dtype=np.float64) + 0.5) * dx for n in res]
    return np.meshgrid(*axes, indexing="ij")


def box_sdf(pts, lo, hi):
    """Signed distance to an axis-aligned box, level_set.py:40-54 convention."""
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    inside = np.ones(pts[0].shape, bool)
    for k, x in enumerate(pts):
        inside &= (x > lo[k]) & (x < hi[k])
    # inside: max over axes of max(lo - x, x - hi) (negative)
    neg = np.full(pts[0].shape, -np.inf)
    for k, x in enumerate(pts):
        neg = np.maximum(neg, np.maximum(lo[k] - x, x - hi[k]))
    # outside: distance to the closest point of the box
    d2 = np.zeros(pts[0].shape)
    for k, x in enumerate(pts):
        q = np.clip(x, lo[k], hi[k])
        d2 += (x - q) ** 2
    return np.where(inside, neg, np.sqrt(d2))


def sphere_sdf(pts, centre, radius):
    """level_set.py:61-64 convention: |x - c| - r."""
    d2 = np.zeros(pts[0].shape)
    for k, x in enumerate(pts):
        d2 += (x - centre[k]) ** 2
    return np.sqrt(d2) - radius


def labels_from_phi(phi, fluid_rule="lt"):
    """SOLID ring, FLUID where phi < 0 (or <= 0), AIR elsewhere."""
    ct = np.full(phi.shape, AIR, np.int32)
    fl = (phi < 0) if fluid_rule == "lt" else (phi <= 0)
    ct[fl] = FLUID
    ring = np.zeros(phi.shape, bool)
    for k in range(phi.ndim):
        sl = [slice(None)] * phi.ndim
        sl[k] = 0
        ring[tuple(sl)] = True
        sl[k] = phi.shape[k] - 1
        ring[tuple(sl)] = True
    ct[ring] = SOLID
    return ct


def random_velocity(rng, res, gravity_dt=0.0):
    """MAC face velocities U[-1, 1] as float32; axis-1 faces get gravity*dt added."""
    vel = []
    for k in range(len(res)):
        shp = list(res)
        shp[k] += 1
        v = rng.uniform(-1.0, 1.0, size=shp).astype(np.float32)
        if k == 1 and gravity_dt != 0.0:
            v += np.float32(gravity_dt)
        vel.append(v)
    return vel


# --------------------------------------------------------------------------
# 2D dam break at 128^2 (the reference's CPU-runnable size)
# --------------------------------------------------------------------------
def dam_break_2d(n=128, seed=0, fluid_rule="lt", gfm_clamp=100.0, levels=4):
    dx = 1.0 / n
    pts = cell_centres((n, n), dx)
    phi = box_sdf(pts, (0.0, 0.0), (0.4, 0.6)).astype(np.float32)
    rng = np.random.default_rng(seed)
    vel = random_velocity(rng, (n, n))
    return Scene(dim=2, res=(n, n), dx=dx, dt=1.25e-2, rho=1000.0, p0=1e-3, phi=phi,
                 cell_type=labels_from_phi(phi, fluid_rule), velocity=vel, levels=levels,
                 gfm_clamp=gfm_clamp, name=f"dam_break_2d_{n}")


# --------------------------------------------------------------------------
# 3D ferrofluid substep: a drop above a pool
# --------------------------------------------------------------------------
def drop_pool_phi(res, dx):
    pts = cell_centres(res, dx)
    sph = sphere_sdf(pts, (0.5, 0.7, 0.5), 0.15)
    pool = pts[1] - 0.3
    return np.minimum(sph, pool).astype(np.float32)


def ferro_drop_3d(n=128, seed=1, fluid_rule="lt", gfm_clamp=100.0, levels=5):
    dx = 1.0 / n
    dt = 1.0 / 60.0
    phi = drop_pool_phi((n, n, n), dx)
    rng = np.random.default_rng(seed)
    vel = random_velocity(rng, (n, n, n), gravity_dt=-9.8 * dt)
    return Scene(dim=3, res=(n, n, n), dx=dx, dt=dt, rho=1000.0, p0=1e-3, phi=phi,
                 cell_type=labels_from_phi(phi, fluid_rule), velocity=vel, levels=levels,
                 gfm_clamp=gfm_clamp, name=f"ferro_drop_3d_{n}")


def smooth_field(res, dx, seed, n_modes=8):
    """Sum of n_modes sinusoids with integer wavenumbers 1-4 and seeded phases."""
    rng = np.random.default_rng(seed)
    pts = cell_centres(res, dx)
    f = np.zeros(res, np.float64)
    for _ in range(n_modes):
        kv = rng.integers(1, 5, size=len(res))
        ph = rng.uniform(0.0, 2.0 * np.pi)
        arg = np.zeros(res, np.float64)
        for k, x in enumerate(pts):
            arg += kv[k] * x
        f += np.sin(2.0 * np.pi * arg + ph)
    return f


def precision_3d(n=256, seed=2, levels=6, amp=0.1, fluid_rule="lt", gfm_clamp=100.0):
    """The drop/pool scene with rhs += amp * (smooth field) on FLUID cells."""
    sc = ferro_drop_3d(n=n, seed=seed, fluid_rule=fluid_rule, gfm_clamp=gfm_clamp, levels=levels)
    sc.extra_rhs = (amp * smooth_field(sc.res, sc.dx, seed + 1000)).astype(np.float32)
    sc.name = f"precision_3d_{n}"
    return sc


# --------------------------------------------------------------------------
# Batches of uneven independent solves
# --------------------------------------------------------------------------
SIDES_2D = tuple(range(64, 513, 32))
SIDES_3D = tuple(range(32, 161, 16))


def domain_shapes(rng, dim):
    """1-3 boxes or spheres: ("box", centre, half sizes) or ("sphere", centre, radius),
    size/radius U[0.1, 0.3], centre U[0.2, 0.8]."""
    shapes = []
    for _ in range(int(rng.integers(1, 4))):
        centre = rng.uniform(0.2, 0.8, size=dim)
        if rng.random() < 0.5:
            shapes.append(("box", centre, rng.uniform(0.1, 0.3, size=dim)))
        else:
            shapes.append(("sphere", centre, rng.uniform(0.1, 0.3)))
    return shapes


def shapes_phi(shapes, pts):
    """Signed distance to the union of `shapes` at the points `pts`."""
    phi = None
    for kind, centre, size in shapes:
        d = box_sdf(pts, centre - size, centre + size) if kind == "box" else sphere_sdf(pts, centre, size)
        phi = d if phi is None else np.minimum(phi, d)
    return phi


def random_domain_phi(rng, res, dx):
    """Union of 1-3 boxes or spheres, size/radius U[0.1, 0.3], centre U[0.2, 0.8]."""
    return shapes_phi(domain_shapes(rng, len(res)), cell_centres(res, dx))


def batch_scene_params(seed=3, n2d=64, n3d=32):
    """Draws (dim, side, scene_seed) for each instance of a batch."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n2d):
        out.append((2, int(rng.choice(SIDES_2D)), int(rng.integers(0, 2**31 - 1))))
    for i in range(n3d):
        out.append((3, int(rng.choice(SIDES_3D)), int(rng.integers(0, 2**31 - 1))))
    return out


def instance_scene(dim, side, scene_seed, levels=4, shift=None, fluid_rule="lt", gfm_clamp=100.0):
    """One batch instance; ``shift`` (in cells, per axis) translates phi."""
    rng = np.random.default_rng(scene_seed)
    res = (side,) * dim
    dx = 1.0 / side
    dt = 1.0 / 60.0
    # geometry draws first, velocity after, so a shift does not change them
    geo_rng = np.random.default_rng(rng.integers(0, 2**31 - 1))
    vel_rng = np.random.default_rng(rng.integers(0, 2**31 - 1))
    if shift is None:
        phi = random_domain_phi(geo_rng, res, dx)
    else:
        # phi_t(x) = phi_0(x - shift*dx): evaluate the shapes at shifted points
        pts = cell_centres(res, dx)
        pts = [p - s * dx for p, s in zip(pts, shift)]
        phi = _random_domain_phi_at(geo_rng, pts, dim)
    phi = phi.astype(np.float32)
    vel = random_velocity(vel_rng, res, gravity_dt=-9.8 * dt)
    return Scene(dim=dim, res=res, dx=dx, dt=dt, rho=1000.0, p0=1e-3, phi=phi,
                 cell_type=labels_from_phi(phi, fluid_rule), velocity=vel, levels=levels,
                 gfm_clamp=gfm_clamp, name=f"inst{dim}d_{side}_{scene_seed}")


def _random_domain_phi_at(rng, pts, dim):
    return shapes_phi(domain_shapes(rng, dim), pts)


def instance_shapes(dim, scene_seed):
    """The shapes and the velocity seed instance_scene draws for a scene seed."""
    rng = np.random.default_rng(scene_seed)
    geo_rng = np.random.default_rng(rng.integers(0, 2**31 - 1))
    vel_seed = int(rng.integers(0, 2**31 - 1))
    return domain_shapes(geo_rng, dim), vel_seed


def batch_scenes(seed=3, n2d=64, n3d=32, levels=4):
    return [instance_scene(d, s, ss, levels=levels) for d, s, ss in batch_scene_params(seed, n2d, n3d)]


# --------------------------------------------------------------------------
# Serving stream: scenes that move by 0.5 cell per substep
# --------------------------------------------------------------------------
def serving_sessions(seed=4, n_sessions=32, substeps=20, rate_hz=100.0, n2d_frac=2 / 3):
    """Poisson arrivals of scene sessions; each session is ``substeps`` chained solves.

    Returns a list of dicts {t_arrive, dim, side, scene_seed, direction}.  The
    scene's level set shifts by 0.5 cell per substep along ``direction``.
    """
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n_sessions):
        t += rng.exponential(1.0 / rate_hz)
        if rng.random() < n2d_frac:
            dim, side = 2, int(rng.choice(SIDES_2D))
        else:
            dim, side = 3, int(rng.choice(SIDES_3D))
        d = rng.normal(size=dim)
        d /= np.linalg.norm(d)
        out.append(dict(t_arrive=t, dim=dim, side=side, scene_seed=int(rng.integers(0, 2**31 - 1)),
                        direction=d, substeps=substeps))
    return out


def session_scene(sess, step, levels=4):
    shift = tuple(0.5 * step * c for c in sess["direction"])
    return instance_scene(sess["dim"], sess["side"], sess["scene_seed"], levels=levels, shift=shift)
