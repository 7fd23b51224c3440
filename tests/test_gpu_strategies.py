"""The reference's other Strategies and the pressure update on the CUDA path,
against the oracle (oracle/simulator_oracle.cpp), through the drop-in classes
and the C ABI.

Bit-exact (f32, same operation order): apply_pressure, apply_magnetic_force,
MagneticForceStrategy b, PotentialFunctionStrategy b and A on every level,
calc_n, calc_kappa, update_magnetic_field.  Within float tolerance where the
reference calls sin / cos (the library's and the C library's differ in the
last bits): the smoothed volume (1e-6 relative), chi (1e-6), the surface
tension system (1e-5 relative).  Solves: +-1 iteration and 1e-5 relative L2,
as for the pressure solve.
"""
import numpy as np
import pytest

from helpers import rel_l2
from test_oracle_strategies import FLUID, AIR, SOLID, scene_2d, scene_3d

pytestmark = pytest.mark.gpu


def _dev():
    import torch
    return torch.device("cuda", 0)


def _t(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(_dev())


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _pressure_pair(make, levels=3):
    from mgpcg import MGPCGPoissonSolver
    from pressure_project import PressureProjectStrategy
    from oracle import OracleSolver
    ct, phi, vel, _ = make()
    dim = ct.ndim
    g = MGPCGPoissonSolver(dim, ct.shape, levels, 2, 50, device=_dev())
    st = PressureProjectStrategy(dim, [_t(v) for v in vel], True, _t(phi), 1e-3)
    st.scale_A, st.scale_b = 0.8, 4.0
    g.reinitialize(_t(ct), st)
    o = OracleSolver(dim, ct.shape, levels, 2, 50, real=np.float32)
    o.reinitialize_pressure(ct, vel, phi, 1e-3, 0.8, 4.0, True, 1e3)
    return ct, phi, vel, g, o


# ---------------------------------------------------------------- apply_pressure
@pytest.mark.parametrize("make", [scene_2d, scene_3d])
@pytest.mark.parametrize("ghost", [True, False])
def test_apply_pressure_bit_exact(make, ghost):
    import fluid_ops
    from oracle import simulator as S
    ct, phi, vel, g, o = _pressure_pair(make)
    g.solve(200)
    x = g.x.cpu().numpy()
    dt, rho, dx, p0 = 0.0125, 1000.0, 1.0 / ct.shape[0], 1e-3
    u = [_t(v) for v in vel]
    fluid_ops.apply_pressure(g, u, dt, rho, dx, p0, phi=_t(phi), ghost_fluid_method=ghost)  # x and labels of g
    ref = S.apply_pressure(vel, x, ct, phi, fluid_ops.pressure_scale(dt, rho, dx), p0, ghost, 1e3)
    for a, b in zip(u, ref):
        np.testing.assert_array_equal(_bits(a.cpu().numpy()), _bits(b))
    # explicit pressure and int32 labels give the same result
    u2 = [_t(v) for v in vel]
    fluid_ops.apply_pressure(g, u2, dt, rho, dx, p0, phi=_t(phi), ghost_fluid_method=ghost, cell_type=_t(ct),
                             pressure=_t(x))
    for a, b in zip(u2, ref):
        np.testing.assert_array_equal(_bits(a.cpu().numpy()), _bits(b))


@pytest.mark.parametrize("make", [scene_2d, scene_3d])
def test_apply_magnetic_force_bit_exact(make):
    import fluid_ops
    from oracle import simulator as S
    ct, phi, vel, p = make()
    from mgpcg import MGPCGPoissonSolver
    g = MGPCGPoissonSolver(ct.ndim, ct.shape, 2, 2, 50, device=_dev())
    rng = np.random.default_rng(11)
    H = [rng.uniform(-2e4, 2e4, v.shape).astype(np.float32) for v in vel]
    u = [_t(v) for v in vel]
    k, mu0 = 5.0, 4 * np.pi * 1e-7
    fluid_ops.apply_magnetic_force(g, u, [_t(h) for h in H], 0.0125, 1000.0, 0.05, 1e-3, k, mu0,
                                   cell_type=_t(ct), pressure=_t(p))
    ref = S.apply_magnetic_force(vel, p, ct, H, fluid_ops.pressure_scale(0.0125, 1000.0, 0.05), 1e-3,
                                 0.5 * k * mu0)
    for a, b in zip(u, ref):
        np.testing.assert_array_equal(_bits(a.cpu().numpy()), _bits(b))


# ------------------------------------------------------------ magnetic force b
@pytest.mark.parametrize("make", [scene_2d, scene_3d])
def test_magnetic_force_strategy_bit_exact(make):
    from mgpcg import MGPCGPoissonSolver
    from magnetic_force import MagneticForceStrategy
    from oracle import OracleSolver
    from oracle import simulator as S
    ct, phi, vel, _ = make()
    dim = ct.ndim
    rng = np.random.default_rng(12)
    H = [rng.uniform(0, 1.2e4, v.shape).astype(np.float32) for v in vel]
    k, mu0 = 5.0, 4 * np.pi * 1e-7
    g = MGPCGPoissonSolver(dim, ct.shape, 3, 2, 50, device=_dev())
    st = MagneticForceStrategy(dim, [_t(v) for v in vel], True, _t(phi), 1e-3, mu0, k, [_t(h) for h in H])
    st.scale_A, st.scale_b = 0.8, 4.0
    g.reinitialize(_t(ct), st)
    o = OracleSolver(dim, ct.shape, 3, 2, 50, real=np.float32)
    o.reinitialize_pressure(ct, vel, phi, 1e-3, 0.8, 4.0, True, 1e3)  # build_A is inherited
    b = S.build_magnetic_b(o.get("grid_type"), vel, H, 1e-3, 0.8, 4.0, np.float32(0.5 * k * mu0))
    np.testing.assert_array_equal(_bits(g.b.cpu().numpy()), _bits(b))
    for l in range(3):
        np.testing.assert_array_equal(g.Adiag[l].cpu().numpy(), o.get("Adiag", l))
    o.set("b", b)
    it = g.solve(300)
    it_o = o.solve(300)
    assert g.last_status == "converged" and abs(it - it_o) <= 1
    assert rel_l2(g.x.cpu().numpy(), o.get("x")) < 1e-5


# ------------------------------------------------------- potential function
def _potential_inputs(dim, n):
    from oracle import simulator as S
    dx = 1.0 / n
    g = (np.arange(n) + 0.5) * dx
    X = np.meshgrid(*([g] * dim), indexing="ij")
    phi = (np.sqrt(sum((x - 0.5) ** 2 for x in X)) - 0.25).astype(np.float32)
    chi = S.update_chi(phi, 5.0, 5 * dx)
    He = [np.full(tuple(n + (a == k) for a in range(dim)), 1.2e4 if k == 1 else 0.0, np.float32)
          for k in range(dim)]
    return dx, phi, chi, He


@pytest.mark.parametrize("dim,n,levels", [(2, 64, 4), (3, 32, 3)])
def test_potential_function_system_and_solve(dim, n, levels):
    from mgpcg import MGPCGPoissonSolver
    from potential_function import PotentialFunctionStrategy
    from oracle import OracleSolver
    from oracle import simulator as S
    dx, phi, chi, He = _potential_inputs(dim, n)
    g = MGPCGPoissonSolver(dim, (n,) * dim, levels, 2, 50, device=_dev())
    st = PotentialFunctionStrategy(dim, (n,) * dim, dx, [_t(h) for h in He], _t(chi))
    g.full_reinitialize(st)
    b = S.build_potential_b(chi, He)
    np.testing.assert_array_equal(_bits(g.b.cpu().numpy()), _bits(b))
    AD, AX = [], []
    for l in range(levels):
        Ad, Ax = S.build_potential_A(chi, l, dx)
        np.testing.assert_array_equal(_bits(g.Adiag[l].cpu().numpy()), _bits(Ad))
        np.testing.assert_array_equal(_bits(np.moveaxis(g.Ax[l].cpu().numpy(), -1, 0)), _bits(Ax))
        AD.append(Ad)
        AX.append(Ax)
    o = OracleSolver(dim, (n,) * dim, levels, 2, 50, real=np.float32)
    o.set_system([np.zeros((n >> l,) * dim, np.int8) for l in range(levels)], AD, AX, b)
    it = g.solve(500)
    it_o = o.solve(500)
    assert g.last_status == "converged", g.last_status
    assert abs(it - it_o) <= 1, (it, it_o)
    assert rel_l2(g.x.cpu().numpy(), o.get("x")) < 1e-5


def test_magnetic_field_and_susceptibility():
    import torch
    import fluid_ops
    from mgpcg import MGPCGPoissonSolver
    from oracle import simulator as S
    dim, n = 3, 24
    dx, phi, chi_ref, He = _potential_inputs(dim, n)
    g = MGPCGPoissonSolver(dim, (n,) * dim, 2, 2, 50, device=_dev())
    chi = torch.zeros((n,) * dim, dtype=torch.float32, device=_dev())
    fluid_ops.update_magnetic_susceptibility(g, _t(phi), 5.0, 5 * dx, chi)
    np.testing.assert_allclose(chi.cpu().numpy(), chi_ref, rtol=1e-6, atol=1e-6)
    psi = np.random.default_rng(4).standard_normal((n,) * dim).astype(np.float32)
    H = [torch.zeros(h.shape, dtype=torch.float32, device=_dev()) for h in He]
    fluid_ops.update_magnetic_field(g, [_t(h) for h in He], dx, H, psi=_t(psi))
    ref = S.update_H(psi, He, dx)
    for a, b in zip(H, ref):
        np.testing.assert_array_equal(_bits(a.cpu().numpy()), _bits(b))


# ------------------------------------------------------------ volume control
def test_volume_and_volume_control():
    from mgpcg import MGPCGPoissonSolver
    from volume_control import PressureProjectWithVolumeControlStrategy
    from oracle import OracleSolver
    from oracle import simulator as S
    ct, phi, vel, _ = scene_2d(n=32)
    n = ct.shape[0]
    dx, dt = 1.0 / n, 0.0125
    eps = 5 * dx
    g = MGPCGPoissonSolver(2, ct.shape, 3, 2, 50, device=_dev())

    class LS:
        pass

    ls = LS()
    ls.eps = eps
    st = PressureProjectWithVolumeControlStrategy(2, [_t(v) for v in vel], True, _t(phi), 1e-3, ls, dt)
    st.scale_A, st.scale_b = 0.8, 4.0
    vol_g = st.calc_volume(g)
    vol_o = S.volume(phi, eps)
    assert abs(vol_g - vol_o) <= 1e-6 * vol_o
    o = OracleSolver(2, ct.shape, 3, 2, 50, real=np.float32)
    state = np.array([0, 0, 0, 0, 0, st.k_p, st.k_i, dt], np.float64)
    for step, ph in enumerate([phi, phi + np.float32(0.02)]):  # the fluid shrinks
        ct = np.where(ph <= 0, FLUID, AIR).astype(np.int32)  # labels follow phi (fluid_simulator.py:151-159)
        ct[0, :] = ct[-1, :] = ct[:, 0] = ct[:, -1] = SOLID
        st.phi = _t(ph)
        g.reinitialize(_t(ct), st)
        o.reinitialize_pressure(ct, vel, ph, 1e-3, 0.8, 4.0, True, 1e3)
        b_o, state = S.volume_control(ph, eps, o.get("grid_type"), o.get("b"), state)
        assert st.step == step + 1
        np.testing.assert_allclose(st.last_volume, state[3], rtol=1e-6)
        np.testing.assert_allclose(st.vol_0, state[1], rtol=1e-6)
        if step:
            np.testing.assert_allclose(st.last_c, state[4], rtol=1e-4)
        np.testing.assert_allclose(g.b.cpu().numpy(), b_o, rtol=1e-5, atol=1e-4 * np.abs(b_o).max())
    assert st.last_c > 0  # the volume shrank: the controller adds divergence
    g.solve(300)
    assert g.last_status == "converged"


# ------------------------------------------------------------ surface tension
class _LevelSet:
    def __init__(self, phi, dx):
        self.phi = phi
        self.eps = 5 * dx


class _Sim:
    def __init__(self, dim, n, phi, vel, solver):
        self.dim, self.res, self.dt, self.dx, self.real = dim, (n,) * dim, 0.0125, 1.0 / n, float
        self.verbose = False
        self.velocity = vel
        self.level_set = _LevelSet(phi, self.dx)
        self.poisson_solver = solver


@pytest.mark.parametrize("dim,n,levels", [(2, 64, 4), (3, 32, 3)])
def test_surface_tension_parity(dim, n, levels):
    from mgpcg import MGPCGPoissonSolver
    from surface_tension import SurfaceTension
    from oracle import OracleSolver
    from oracle import simulator as S
    dx = 1.0 / n
    g = (np.arange(n) + 0.5) * dx
    X = np.meshgrid(*([g] * dim), indexing="ij")
    phi = (np.sqrt(sum((x - 0.5) ** 2 for x in X)) - 0.3).astype(np.float32)
    rng = np.random.default_rng(9)
    vel = [rng.uniform(-1, 1, tuple(n + (a == k) for a in range(dim))).astype(np.float32) for k in range(dim)]
    solver = MGPCGPoissonSolver(dim, (n,) * dim, levels, 2, 50, device=_dev())
    sim = _Sim(dim, n, _t(phi), [_t(v) for v in vel], solver)
    st = SurfaceTension(sim)
    # one axis by hand: the intermediate fields against the oracle
    st.calc_n(0, sim.level_set.phi)
    st.calc_kappa(0, sim.level_set.phi)
    n_o = S.calc_n(phi, 0, dx)
    k_o = S.calc_kappa(n_o, dx)
    np.testing.assert_array_equal(_bits(st.n.cpu().numpy()), _bits(n_o))
    np.testing.assert_array_equal(_bits(st.kappa.cpu().numpy()), _bits(k_o))
    # the full step: one solve per axis, x copied into u_d
    st.solve_surface_tension()
    eps = 5 * dx
    for k in range(dim):
        nk = S.calc_n(phi, k, dx)
        kk = S.calc_kappa(nk, dx)
        b = S.build_st_b(k, vel[k], phi, nk, kk, st.sigma, sim.dt, dx, eps)
        AD, AX = zip(*[S.build_st_A(phi, l, k, st.sigma, sim.dt, dx, eps) for l in range(levels)])
        o = OracleSolver(dim, (n,) * dim, levels, 2, 50, real=np.float32)
        o.set_system([np.zeros((n >> l,) * dim, np.int8) for l in range(levels)], AD, AX, b)
        o.solve(500)
        u = sim.velocity[k].cpu().numpy()
        inner = tuple(slice(0, n) for _ in range(dim))
        assert rel_l2(u[inner], o.get("x")) < 1e-5, k
        last = tuple(slice(n, n + 1) if a == k else slice(None) for a in range(dim))
        np.testing.assert_array_equal(u[last], vel[k][last])  # the face beyond x is untouched
