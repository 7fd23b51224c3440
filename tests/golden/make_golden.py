"""Generates the golden fixtures of the MGPCG path (run from the repo root).

The reference (Taichi DSL Python) cannot run here, so these vectors come from
the CPU oracle (oracle/), whose restatement is itself pinned by
tests/test_oracle.py (scipy direct solves, independent assembly, V-cycle
symmetry).  They freeze the oracle's outputs so that the GPU path and any
later change of the oracle are checked against the same numbers.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "taichi-ferrofluid_b200"))
sys.path.insert(0, ROOT)

import mg_scenes  # noqa: E402
from oracle import OracleSolver  # noqa: E402

CASES = {
    "dam2d_32": lambda: mg_scenes.dam_break_2d(n=32, seed=0, levels=3),
    "drop3d_16": lambda: mg_scenes.ferro_drop_3d(n=16, seed=1, levels=3),
    "dam2d_32_ref_rules": lambda: mg_scenes.dam_break_2d(n=32, seed=7, fluid_rule="le", gfm_clamp=1e3, levels=3),
}


def make(name):
    sc = CASES[name]()
    out = dict(dim=sc.dim, res=np.array(sc.res), levels=sc.levels, dt=sc.dt, rho=sc.rho, p0=sc.p0, dx=sc.dx,
               gfm_clamp=sc.gfm_clamp, phi=sc.phi, cell_type=sc.cell_type)
    for k, v in enumerate(sc.velocity):
        out[f"vel{k}"] = v
    o = OracleSolver(sc.dim, sc.res, sc.levels, 2, 50, real=np.float32)
    o.reinitialize_pressure(sc.cell_type, sc.velocity, sc.phi, sc.p0, sc.scale_A, sc.scale_b, True, sc.gfm_clamp)
    for l in range(sc.levels):
        out[f"grid_type{l}"] = o.get("grid_type", l)
        out[f"Adiag{l}"] = o.get("Adiag", l)
        out[f"Ax{l}"] = o.get("Ax", l)
    out["b"] = o.get("b")
    o.set("r", out["b"], 0)
    o.v_cycle()
    out["z_vcycle"] = o.get("z", 0)
    o2 = OracleSolver(sc.dim, sc.res, sc.levels, 2, 50, real=np.float32)
    o2.reinitialize_pressure(sc.cell_type, sc.velocity, sc.phi, sc.p0, sc.scale_A, sc.scale_b, True, sc.gfm_clamp)
    out["iters_f32"] = o2.solve(500, acc_mode=1)
    out["x_f32"] = o2.get("x")
    o3 = OracleSolver(sc.dim, sc.res, sc.levels, 2, 50, real=np.float64)
    o3.reinitialize_pressure(sc.cell_type, sc.velocity, sc.phi, sc.p0, sc.scale_A, sc.scale_b, True, sc.gfm_clamp)
    o3.solve(1000, rel_tol=1e-24)
    out["x_f64"] = o3.get("x")
    return out


if __name__ == "__main__":
    here = os.path.dirname(os.path.abspath(__file__))
    for name in CASES:
        np.savez_compressed(os.path.join(here, f"{name}.npz"), **make(name))
        print("wrote", name)
