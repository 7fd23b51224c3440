"""Shared set-up for the parity tests: one scene fed to the CUDA solver and to
the CPU oracle with identical inputs."""
import numpy as np

import mg_scenes


def small_3d(n=32, seed=1, levels=3):
    """The 3D drop/pool scene at a size the oracle finishes in well under a second."""
    return mg_scenes.ferro_drop_3d(n=n, seed=seed, levels=levels)


def box_3d(res, levels, seed=5):
    """A drop above a pool on a non-cubic grid (res = planes, rows, columns)."""
    n = max(res)
    dx = 1.0 / n
    phi = mg_scenes.drop_pool_phi(res, dx)
    rng = np.random.default_rng(seed)
    vel = mg_scenes.random_velocity(rng, res, gravity_dt=-9.8 / 60.0)
    return mg_scenes.Scene(dim=3, res=res, dx=dx, dt=1.0 / 60.0, rho=1000.0, p0=1e-3, phi=phi,
                           cell_type=mg_scenes.labels_from_phi(phi), velocity=vel, levels=levels,
                           gfm_clamp=100.0, name="box_" + "x".join(map(str, res)))


def oracle_for(scene, real=np.float32, bottom=50, pre_post=2, levels=None, clamp=None):
    from oracle import OracleSolver
    L = levels or scene.levels
    o = OracleSolver(scene.dim, scene.res, L, pre_post, bottom, real=real)
    o.reinitialize_pressure(scene.cell_type, scene.velocity, scene.phi, scene.p0, scene.scale_A, scene.scale_b,
                            True, scene.gfm_clamp if clamp is None else clamp)
    if scene.extra_rhs is not None:
        b = o.get("b")
        fl = o.get("grid_type") == 0
        b[fl] = (b[fl].astype(real) + scene.extra_rhs[fl].astype(real)).astype(real)
        o.set("b", b)
    return o


def true_rel_resid(solver):
    """||b - A x|| / ||b|| over FLUID cells, in float64 from the solver's own
    float32 A, b and x (independent of the solver's residual bookkeeping)."""
    x = solver.x.double().cpu().numpy()
    b = solver.b.double().cpu().numpy()
    ad = solver.Adiag[0].double().cpu().numpy()
    ax = np.moveaxis(solver.Ax[0].double().cpu().numpy(), -1, 0)
    fl = solver.grid_type[0].cpu().numpy() == 0
    Axv = ad * x
    for k in range(solver.dim):
        lo = [slice(None)] * solver.dim
        hi = [slice(None)] * solver.dim
        lo[k] = slice(0, -1)
        hi[k] = slice(1, None)
        lo, hi = tuple(lo), tuple(hi)
        Axv[hi] += ax[k][lo] * x[lo]
        Axv[lo] += ax[k][lo] * x[hi]
    r = np.where(fl, b - Axv, 0.0)
    nb = np.linalg.norm(np.where(fl, b, 0.0))
    return float(np.linalg.norm(r) / nb)


def gpu_for(scene, storage=None, bottom=50, pre_post=2, levels=None, clamp=None, refresh_every=None,
            stored_kernels=False):
    import torch
    from mgpcg import MGPCGPoissonSolver
    from pressure_project import PressureProjectStrategy
    dev = torch.device("cuda", 0)
    L = levels or scene.levels
    s = MGPCGPoissonSolver(scene.dim, scene.res, L, pre_post, bottom, storage=storage, device=dev,
                           refresh_every=refresh_every, stored_kernels=stored_kernels)
    vel = [torch.from_numpy(v).to(dev) for v in scene.velocity]
    phi = torch.from_numpy(scene.phi).to(dev)
    st = PressureProjectStrategy(scene.dim, vel, True, phi, scene.p0,
                                 gfm_clamp=scene.gfm_clamp if clamp is None else clamp)
    st.scale_A = scene.scale_A
    st.scale_b = scene.scale_b
    s.reinitialize(torch.from_numpy(scene.cell_type).to(dev), st)
    if scene.extra_rhs is not None:
        src = torch.from_numpy(scene.extra_rhs).to(dev)
        from mg_lib import check
        check(s.lib.mg_add_rhs(s.plan, src.data_ptr(), 1.0, s._s()), "mg_add_rhs")
        torch.cuda.synchronize()
    return s, st


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    d = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (d if d > 0 else 1.0))
