"""The velocity steps around the projection on the CUDA path - semi-Lagrangian
advection of the velocity and the level set, velocity extrapolation, the solid
boundary and gravity (fluid_simulator.py:160-272) - against the oracle, bit
for bit (f32, the reference's operation order, no reductions)."""
import numpy as np
import pytest

from test_oracle_strategies import FLUID, AIR, SOLID

pytestmark = pytest.mark.gpu


def _t(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _bits(t):
    return t.detach().cpu().numpy().view(np.uint32)


def _scene(dim, n, seed=5):
    rng = np.random.default_rng(seed)
    vel = [rng.uniform(-2, 2, tuple(n + (a == k) for a in range(dim))).astype(np.float32) for k in range(dim)]
    g = (np.arange(n) + 0.5) / n
    X = np.meshgrid(*([g] * dim), indexing="ij")
    phi = (np.sqrt(sum((x - 0.5) ** 2 for x in X)) - 0.3).astype(np.float32)
    ct = np.where(phi < 0, FLUID, AIR).astype(np.int32)
    for k in range(dim):
        for e in (0, -1):
            idx = [slice(None)] * dim
            idx[k] = e
            ct[tuple(idx)] = SOLID
    return vel, phi, ct


@pytest.mark.parametrize("dim,n", [(2, 64), (3, 24)])
def test_advect_quantity_bit_exact(dim, n):
    import torch
    import fluid_ops
    from oracle import simulator as S
    vel, phi, _ = _scene(dim, n)
    dx, dt = 1.0 / n, 0.0125
    u = [_t(v) for v in vel]
    backup = [torch.empty_like(v) for v in u]
    ph, ph_t = _t(phi), torch.empty_like(_t(phi))
    fluid_ops.advect_quantity(u, backup, dx, dt, phi=ph, phi_temp=ph_t)
    np.testing.assert_array_equal(_bits(ph_t), S.advect(vel, phi, -1, dx, dt).view(np.uint32))
    for k in range(dim):
        np.testing.assert_array_equal(_bits(backup[k]), S.advect(vel, vel[k], k, dx, dt).view(np.uint32))
    fluid_ops.update_quantity(u, backup, ph, ph_t)
    assert torch.equal(u[0], backup[0]) and torch.equal(ph, ph_t)


@pytest.mark.parametrize("iterations", [10, 3])
@pytest.mark.parametrize("dim,n", [(2, 48), (3, 20)])
def test_extrap_velocity_bit_exact(dim, n, iterations):
    import fluid_ops
    from oracle import simulator as S
    vel, _, ct = _scene(dim, n)
    u = [_t(v) for v in vel]
    fluid_ops.extrap_velocity(u, _t(ct), iterations)
    for k in range(dim):
        ref, _ = S.extrapolate(vel[k], k, ct, iterations)
        np.testing.assert_array_equal(_bits(u[k]), ref.view(np.uint32))


def test_boundary_and_gravity_bit_exact():
    import fluid_ops
    from oracle import simulator as S
    vel, _, ct = _scene(3, 20)
    u = [_t(v) for v in vel]
    fluid_ops.enforce_boundary(u, _t(ct))
    ref = S.enforce_boundary(vel, ct)
    fluid_ops.add_gravity(u, (0.0, -9.8, 0.0), np.float32(1 / 60))
    ref = S.add_gravity(ref, (0.0, -9.8, 0.0), np.float32(1 / 60))
    for a, b in zip(u, ref):
        np.testing.assert_array_equal(_bits(a), b.view(np.uint32))
