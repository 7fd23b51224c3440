"""Parity at the benchmark sizes themselves, not only at smaller grids.

* The 3D ferrofluid substep at 128^3 (5 levels): (a) the ghost-fluid pressure
  solve and (b) the magnetic potential solve, each against the float32 oracle
  (iterations +-1, pressure within 1e-5 relative L2) and against the FP64
  oracle solved to a 1e-12 relative residual (the error is printed and
  asserted).  The V-cycle of the pressure operator is compared bit for bit.
* The 256^3 precision scene (6 levels) in float32, FP16 and BF16 V-cycle
  storage: the mixed form's true relative residual (FP64, from its FP64 x)
  reaches 1e-6 and the error against the FP64 oracle is printed and asserted;
  the float32 solve also matches the float32 oracle within 1e-5 and +-1
  iteration.

Error bounds are the float32 floors measured with FP64 solves of the
float32-rounded systems: no float32 solve can come closer to the FP64
system's solution than that system's own solution does.

The solver follows mgpcg.py:150-209 (rel_tol compares squared norms, so
1e-12 is a 1e-6 relative residual).
"""
import numpy as np
import pytest

import mg_scenes
from helpers import gpu_for, oracle_for, rel_l2, true_rel_resid

pytestmark = pytest.mark.gpu

PSI_H = (0.0, 1.0, 0.0)
PSI_PIN = (1, 1, 1)


@pytest.fixture(scope="module")
def drop128():
    return mg_scenes.ferro_drop_3d(n=128, seed=1, levels=5)


def test_substep128_pressure_vcycle_bit_exact(drop128):
    """One V-cycle of the 128^3 pressure operator on r = b (mgpcg.py:125-148)."""
    import torch
    sc = drop128
    g, _ = gpu_for(sc)
    o = oracle_for(sc)
    o.set("r", o.get("b"), 0)
    g.r[0].copy_(g.b)
    g.v_cycle()
    o.v_cycle()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(g.z[0].cpu().numpy(), o.get("z", 0))


def test_substep128_pressure_solve(drop128):
    sc = drop128
    g, _ = gpu_for(sc)
    it = g.solve(500)
    assert g.last_status == "converged"
    x = g.x.cpu().numpy()
    o = oracle_for(sc)
    it_o = o.solve(500)
    assert abs(it - it_o) <= 1, (it, it_o)
    e32 = rel_l2(x, o.get("x"))
    assert e32 < 1e-5, e32
    o64 = oracle_for(sc, real=np.float64)
    it64 = o64.solve(1000, rel_tol=1e-24)
    err = rel_l2(x, o64.get("x"))
    res = true_rel_resid(g)
    print(f"pressure 128^3: iters {it} (oracle {it_o}, FP64 {it64}), rel L2 vs f32 oracle {e32:.2e}, "
          f"error vs FP64 {err:.2e}, true rel resid {res:.2e}")
    # the float32 form stops on the recursive residual (mgpcg.py:175-190);
    # the true one drifts above it (measured 2.7e-6, the oracle's too)
    assert res < 5e-6, res
    # the float32 system itself (A, b rounded to float32) has a solution
    # 1.17e-4 from the FP64 system's (measured with an FP64 solve of it):
    # no float32 solve can be closer
    assert err < 1.5e-4, err


def test_substep128_psi_solve(drop128):
    import torch
    from magnetic_potential import MagneticPotentialStrategy
    from mgpcg import MGPCGPoissonSolver
    from oracle import OracleSolver
    sc = drop128
    chi = (sc.phi < 0).astype(np.float32)
    g = MGPCGPoissonSolver(3, sc.res, 5, 2, 50, device="cuda")
    g.full_reinitialize(MagneticPotentialStrategy(3, torch.from_numpy(chi).cuda(), PSI_H, sc.dx, PSI_PIN))
    it = g.solve(500)
    assert g.last_status == "converged"
    x = g.x.cpu().numpy()
    o = OracleSolver(3, sc.res, 5, 2, 50, real=np.float32)
    o.full_reinitialize_psi(chi, PSI_H, sc.dx, PSI_PIN)
    it_o = o.solve(500)
    assert abs(it - it_o) <= 1, (it, it_o)
    e32 = rel_l2(x, o.get("x"))
    assert e32 < 1e-5, e32
    o64 = OracleSolver(3, sc.res, 5, 2, 50, real=np.float64)
    o64.full_reinitialize_psi(chi, PSI_H, sc.dx, PSI_PIN)
    it64 = o64.solve(2000, rel_tol=1e-24, abs_tol=0.0, eps=0.0)
    err = rel_l2(x, o64.get("x"))
    res = true_rel_resid(g)
    print(f"psi 128^3: iters {it} (oracle {it_o}, FP64 {it64}), rel L2 vs f32 oracle {e32:.2e}, "
          f"error vs FP64 {err:.2e}, true rel resid {res:.2e}")
    # psi grows across the whole domain while b lives at the interface: the
    # float32 rounding of the exact solution alone leaves a 5e-5 true
    # residual, and the float32 system's solution is 1.5e-3 from the FP64
    # system's (both measured with FP64 solves); the oracle's float32 solve
    # is bit-identical to this one
    assert res < 5e-4, res
    assert err < 2e-3, err


@pytest.fixture(scope="module")
def precision256():
    """The 256^3 scene and its FP64 oracle solution at a 1e-12 relative residual."""
    sc = mg_scenes.precision_3d(n=256, seed=2, levels=6)
    o64 = oracle_for(sc, real=np.float64)
    it64 = o64.solve(1000, rel_tol=1e-24)
    return sc, o64.get("x"), it64


@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
def test_precision256(storage, precision256):
    sc, x64, it64 = precision256
    g, _ = gpu_for(sc, storage=None if storage == "f32" else storage)
    it = g.solve(500)
    assert g.last_status == "converged", (g.last_status, it)
    x = g.x.cpu().numpy()
    res = true_rel_resid(g)
    err = rel_l2(x, x64)
    msg = f"precision256 {storage}: iters {it} (FP64 oracle {it64}), true rel resid {res:.2e}, error vs FP64 {err:.2e}"
    if storage == "f32":
        o = oracle_for(sc)
        it_o = o.solve(500)
        e32 = rel_l2(x, o.get("x"))
        msg += f", oracle f32 iters {it_o}, rel L2 vs f32 oracle {e32:.2e}"
        assert abs(it - it_o) <= 1, (it, it_o)
        assert e32 < 1e-5, e32
    msg += f", solver's residual {g.last_rel_resid:.2e}"
    print(msg)
    # the float32 system's own solution is 4.9e-4 from the FP64 system's
    # (measured with an FP64 solve of it): no float32 solve can be closer
    assert err < 6e-4, err
    if storage == "f32":
        # stopped on the recursive residual: the true one drifts above it
        assert res < 1e-5, res
    else:
        # the mixed form accumulates x in FP64 and stops on its true residual,
        # recomputed in FP64 (iterative refinement)
        assert g.last_rel_resid <= 1e-6, g.last_rel_resid
        # the float32 rounding of the solution alone leaves 0.84e-6 at 256^3
        assert res < 2e-6, res


def test_substep128_psi_coarse_forms(drop128):
    """The psi solve of the 3D substep with its coarse levels as half the
    Galerkin operator (the default) and rediscretised as the reference's
    potential Strategy does: both converge and match the float32 oracle run
    the same way; the iteration counts are printed side by side."""
    import torch
    from magnetic_potential import MagneticPotentialStrategy
    from mgpcg import MGPCGPoissonSolver
    from oracle import OracleSolver
    sc = drop128
    chi = (sc.phi < 0).astype(np.float32)
    out = {}
    for coarse, scale in (("galerkin", 0.5), ("rediscretise", 0.0)):
        g = MGPCGPoissonSolver(3, sc.res, 5, 2, 50, device="cuda")
        g.full_reinitialize(MagneticPotentialStrategy(3, torch.from_numpy(chi).cuda(), PSI_H, sc.dx, PSI_PIN,
                                                      coarse=coarse))
        it = g.solve(500)
        assert g.last_status == "converged"
        o = OracleSolver(3, sc.res, 5, 2, 50, real=np.float32)
        o.full_reinitialize_psi(chi, PSI_H, sc.dx, PSI_PIN, coarse_scale=scale)
        it_o = o.solve(500)
        assert abs(it - it_o) <= 1, (coarse, it, it_o)
        assert rel_l2(g.x.cpu().numpy(), o.get("x")) < 1e-5
        out[coarse] = it
    print(f"psi 128^3 iterations: half Galerkin {out['galerkin']}, rediscretised {out['rediscretise']}")
