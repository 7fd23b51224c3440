"""Autotuner of the multigrid parameters a caller may leave open.

The reference fixes them per call (``MGPCGPoissonSolver(dim, res,
n_mg_levels=4, pre_and_post_smoothing=2, bottom_smoothing=50)``, mgpcg.py:6;
the simulators pass their own, fluid_simulator.py:92-96).  Where a caller
lets the library choose - the batched and served solves - this module picks,
per grid shape and storage type, the smoothing sweeps per level, the bottom
sweeps and the level count by MEASURING the time to a 1e-6 relative residual
of a sample solve on the device:

* ``pre_post`` in (1, 2, 3): more sweeps per level make each V-cycle slower
  and the preconditioner stronger (fewer PCG iterations);
* ``bottom`` in (10, 25, 50) sweeps on the coarsest grid;
* the level count: the rule's choice (coarsest grid 8..16 cells a side) and
  one level fewer or more where the shape halves evenly.

The kernel-level launch shapes (tile shape, grid, planes per step, where the
cluster-resident V-cycle starts) are tuned separately by the library each
time a plan shape is first prepared (mg_plan_prepare); every candidate here
runs with its own tuned launch shapes.  Every candidate solve converges to the
same tolerance; a candidate that does not is discarded.  Results are cached
per (dim, shape, storage) for the process.
"""
import torch

from mgpcg import MGPCGPoissonSolver

SWEEPS = (1, 2, 3)
BOTTOMS = (10, 25, 50)

_cache = {}


def rule_levels(dim, side):
    """Level count that brings the coarsest grid to 8..16 cells per side."""
    L = 1
    while side % (1 << L) == 0 and (side >> L) >= 8 and L < 8:
        L += 1
    return L


def level_choices(res):
    """The rule's level count and its neighbours that halve every axis evenly
    down to a coarsest grid of at least 4 cells a side."""
    side = min(res)
    L0 = rule_levels(len(res), side)
    out = []
    for L in (L0 - 1, L0, L0 + 1):
        if L >= 2 and all(n % (1 << (L - 1)) == 0 and (n >> (L - 1)) >= 4 for n in res):
            out.append(L)
    return out or [L0]


def _solve_ms(solver, sc, device, reps):
    """Device ms of a one-call pressure solve (set-up + PCG loop), min of reps."""
    stream = torch.cuda.current_stream(device)
    solver.pressure_solve_async(sc.ct, sc.vel, sc.phi, sc.p0, sc.scale_A, sc.scale_b, True, sc.gfm_clamp)
    st = solver.stats()  # warm-up: workspace, kernel launch shapes, graph
    best = None
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        solver.pressure_solve_async(sc.ct, sc.vel, sc.phi, sc.p0, sc.scale_A, sc.scale_b, True, sc.gfm_clamp)
        e1.record(stream)
        st = solver.stats()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    return best, st


class _DeviceInputs:
    """A scene's labels, velocities and level set on the device."""

    def __init__(self, scene, device):
        self.ct = torch.from_numpy(scene.cell_type).to(device)
        self.vel = [torch.from_numpy(v).to(device) for v in scene.velocity]
        self.phi = torch.from_numpy(scene.phi).to(device)
        self.p0, self.scale_A, self.scale_b, self.gfm_clamp = scene.p0, scene.scale_A, scene.scale_b, scene.gfm_clamp


def tune(scene, storage="f32", device=None, sweeps=SWEEPS, bottoms=BOTTOMS, levels=None, reps=2):
    """Times every (pre_post, bottom, levels) candidate on the scene's
    pressure solve and returns the fastest that converges, with the table:
    {"pre_post", "bottom", "levels", "ms", "iters", "candidates": [...]}."""
    device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    key = (scene.dim, tuple(scene.res), storage, tuple(sweeps), tuple(bottoms), tuple(levels or ()))
    if key in _cache:
        return _cache[key]
    sc = _DeviceInputs(scene, device)
    table = []
    for L in (levels or level_choices(scene.res)):
        for pp in sweeps:
            for bot in bottoms:
                solver = MGPCGPoissonSolver(scene.dim, scene.res, L, pp, bot, storage=storage, device=device)
                ms, st = _solve_ms(solver, sc, device, reps)
                table.append({"levels": L, "pre_post": pp, "bottom": bot, "ms": round(ms, 4), "iters": st.iters,
                              "converged": st.status == 0})
                solver.close()
                del solver
    ok = [c for c in table if c["converged"]]
    if not ok:
        raise RuntimeError(f"no candidate converged for a {scene.dim}D {scene.res} scene")
    best = min(ok, key=lambda c: c["ms"])
    out = {"pre_post": best["pre_post"], "bottom": best["bottom"], "levels": best["levels"], "ms": best["ms"],
           "iters": best["iters"], "candidates": table}
    _cache[key] = out
    return out


def size_class(dim, side):
    """Buckets of the batch's size range that share one tuned choice."""
    if dim == 2:
        return (2, 0 if side <= 128 else (1 if side <= 288 else 2))
    return (3, 0 if side <= 64 else (1 if side <= 112 else 2))


def tune_classes(scenes, storage="f32", device=None, **kw):
    """Tunes on the largest scene of each size class and returns, per scene,
    (levels, pre_post, bottom), plus the per-class results.  A class's choice
    applies to all of its scenes (the level count re-derived per shape: the
    class winner's offset from the rule)."""
    classes = {}
    for sc in scenes:
        k = size_class(sc.dim, min(sc.res))
        if k not in classes or sc.cells > classes[k].cells:
            classes[k] = sc
    results = {}
    for k, sc in sorted(classes.items()):
        r = tune(sc, storage, device, **kw)
        results[k] = dict(r, scene=sc.name, offset=r["levels"] - rule_levels(sc.dim, min(sc.res)))
    per_scene = []
    for sc in scenes:
        r = results[size_class(sc.dim, min(sc.res))]
        L = rule_levels(sc.dim, min(sc.res)) + r["offset"]
        choices = level_choices(sc.res)
        if L not in choices:
            L = min(choices, key=lambda c: abs(c - L))
        per_scene.append((L, r["pre_post"], r["bottom"]))
    return per_scene, results


def class_params(results):
    """(dim, side) -> (levels, pre_post, bottom) from tune_classes' per-class
    results, for sessions of the same size distribution (the rule's levels,
    2 and 50 for a class that was not tuned)."""
    def params(dim, side):
        r = results.get(size_class(dim, side))
        if r is None:
            return rule_levels(dim, side), 2, 50
        L = rule_levels(dim, side) + r["offset"]
        choices = level_choices((side,) * dim)
        if L not in choices:
            L = min(choices, key=lambda c: abs(c - L))
        return L, r["pre_post"], r["bottom"]
    return params
