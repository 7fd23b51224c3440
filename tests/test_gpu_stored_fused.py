"""The fused V-cycle on whole-domain stored-coefficient operators (every cell
FLUID, arbitrary couplings): the magnetic potential of the 3D substep, the
reference-form PotentialFunctionStrategy (whose coarse levels couple to a
cell beyond the level's edge, rule H1) and the surface tension operator.

The system is assembled by the oracle and written into both solvers, so only
the V-cycle and the solve are compared: the fused V-cycle against the oracle's
v_cycle (mgpcg.py:125-148) BIT-EXACT, and the fused solve against the
one-launch-per-reference-kernel solve BIT-EXACT (x and iteration count).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _psi(n, levels):
    import mg_scenes
    from oracle import OracleSolver
    sc = mg_scenes.ferro_drop_3d(n=n, levels=levels)
    chi = (sc.phi < 0).astype(np.float32)
    o = OracleSolver(3, sc.res, levels, 2, 50, real=np.float32)
    o.full_reinitialize_psi(chi, (0.0, 1.0, 0.0), sc.dx, (1, 1, 1))
    return [o.get("Adiag", l) for l in range(levels)], [o.get("Ax", l) for l in range(levels)], o.get("b")


def _field(n):
    dx = 1.0 / n
    g = (np.arange(n) + 0.5) * dx
    X = np.meshgrid(g, g, g, indexing="ij")
    return dx, (np.sqrt((X[0] - 0.5) ** 2 + (X[1] - 0.55) ** 2 + (X[2] - 0.5) ** 2) - 0.27).astype(np.float32)


def _potential(n, levels):
    from oracle import simulator as S
    dx, phi = _field(n)
    chi = S.update_chi(phi, 5.0, 5 * dx)
    He = [np.full(tuple(n + (a == k) for a in range(3)), 1.2e4 if k == 1 else 0.0, np.float32) for k in range(3)]
    AD, AX = zip(*[S.build_potential_A(chi, l, dx) for l in range(levels)])
    return list(AD), list(AX), S.build_potential_b(chi, He)


def _surface_tension(n, levels, d=1):
    from oracle import simulator as S
    dx, phi = _field(n)
    rng = np.random.default_rng(2)
    u = rng.uniform(-1, 1, tuple(n + (a == d) for a in range(3))).astype(np.float32)
    nn = S.calc_n(phi, d, dx)
    kap = S.calc_kappa(nn, dx)
    args = (7.28e-2, 0.0125, dx, 5 * dx)
    AD, AX = zip(*[S.build_st_A(phi, l, d, *args) for l in range(levels)])
    return list(AD), list(AX), S.build_st_b(d, u, phi, nn, kap, *args)


SYSTEMS = {
    "psi_32": lambda: (3, 32, _psi(32, 3)),
    "psi_64": lambda: (4, 64, _psi(64, 4)),
    "potential_32": lambda: (3, 32, _potential(32, 3)),
    "potential_64": lambda: (4, 64, _potential(64, 4)),
    "surface_tension_48": lambda: (4, 48, _surface_tension(48, 4)),
}


def _pair(name, pre_post=2, stored_kernels=False):
    import torch
    from mgpcg import MGPCGPoissonSolver
    from oracle import OracleSolver
    levels, n, (AD, AX, b) = SYSTEMS[name]()
    res = (n, n, n)
    g = MGPCGPoissonSolver(3, res, levels, pre_post, 50, device="cuda", stored_kernels=stored_kernels)
    g.initialize()
    for l in range(levels):
        g.grid_type[l].zero_()  # every cell FLUID
        g.Adiag[l].copy_(torch.from_numpy(AD[l]))
        g.Ax[l].copy_(torch.from_numpy(np.ascontiguousarray(np.moveaxis(AX[l], 0, -1))))
    g.b.copy_(torch.from_numpy(b))
    g.prepare()
    o = OracleSolver(3, res, levels, pre_post, 50, real=np.float32)
    o.set_system([np.zeros(tuple(v >> l for v in res), np.int8) for l in range(levels)], AD, AX, b)
    return g, o


def _bits(t):
    return t.detach().float().cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("split", ["tuned", "streamed", "alternate"])
@pytest.mark.parametrize("pre_post", [1, 2])
@pytest.mark.parametrize("name", list(SYSTEMS))
def test_stored_fused_v_cycle_bit_exact(name, pre_post, split):
    """Streamed levels, per-kernel (split) levels and their mixtures."""
    import torch
    g, o = _pair(name, pre_post)
    assert g.operator_form(0) == 2  # whole-domain stored form, fused V-cycle
    _, lc = g.split_levels()
    assert lc >= 1
    if split == "streamed":
        assert g.split_levels(0) == (0, lc)
    elif split == "alternate":  # levels 0, 2, ... per-kernel; 1, 3, ... streamed
        want = 0b0101 & ((1 << lc) - 1)
        assert g.split_levels(want) == (want, lc)
    o.set("r", o.get("b"), 0)
    g.r[0].copy_(g.b)
    g.v_cycle()
    o.v_cycle()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(_bits(g.z[0]), o.get("z", 0).view(np.uint32))


@pytest.mark.parametrize("name", list(SYSTEMS))
def test_stored_fused_solve_equals_per_kernel_solve(name):
    g1, o = _pair(name)
    g2, _ = _pair(name, stored_kernels=True)
    assert g2.operator_form(0) == 0
    it1 = g1.solve(500)
    it2 = g2.solve(500)
    assert g1.last_status == "converged", g1.last_status
    assert it1 == it2
    np.testing.assert_array_equal(_bits(g1.x), _bits(g2.x))
    assert g1.launch_counts()[1] < g2.launch_counts()[1]
    it_o = o.solve(500)
    assert abs(it1 - it_o) <= 1
