"""Benchmark of the MGPCG Poisson path: solves/s and p50/p99 latency.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload substep128|precision256|dam2d] [--storage f32|f16|bf16]

A step is one substep's worth of Poisson solves of the workload, each solve
= reinitialize(cell_type, strategy) + solve(500) at 1e-6 relative residual:

* substep128 (default): the 3D ferrofluid substep at 128^3, 5 levels, pre/post
  2, bottom 50: (a) the ghost-fluid pressure solve, (b) the magnetic potential
  solve when available.
* precision256: the 256^3 drop/pool scene with the smooth extra source, 6 levels.
* dam2d: the 2D dam break at 128^2, 4 levels (the reference's CPU-runnable case).

Inputs are seeded synthetic fields (mg_scenes); there is no dataset.
`value` = solves/s with the inputs resident in HBM; `e2e` = the same through
the public API with every step's inputs copied from pinned host memory and its
result copied back, pipelined as a serving loop would (a copy stream uploads
step k+1's inputs and reads back step k's result while step k solves), timed
from the first upload to the last read-back.  L2 (126 MB) is flushed before
every timed solve.  Multi-GPU runs are independent replicas (the path shards by solve).
`--impl reference` times the CPU oracle (C++/OpenMP restatement of the
reference; the Taichi reference cannot be installed here) on the same workload.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "taichi-ferrofluid_b200")
for _p in (PKG, ROOT):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

import mg_scenes  # noqa: E402

def _substep128():
    sc = mg_scenes.ferro_drop_3d(n=128, seed=1, levels=5)
    return [("pressure", sc), ("psi", sc)]


# each workload: a list of (kind, scene) solves per step; kind "pressure" is the
# ghost-fluid pressure solve, "psi" the magnetic potential solve (chi = 1 in the fluid)
WORKLOADS = {
    "substep128": dict(desc="3D ferrofluid substep 128^3, 5 levels: (a) ghost-fluid pressure solve + "
                            "(b) magnetic potential solve", cases=_substep128, solves=2),
    "pressure128": dict(desc="3D ghost-fluid pressure solve 128^3, 5 levels",
                        cases=lambda: [("pressure", mg_scenes.ferro_drop_3d(n=128, seed=1, levels=5))], solves=1),
    "precision256": dict(desc="3D drop/pool 256^3 with smooth source, 6 levels",
                         cases=lambda: [("pressure", mg_scenes.precision_3d(n=256, seed=2, levels=6))], solves=1),
    "dam2d": dict(desc="2D dam break 128^2, 4 levels",
                  cases=lambda: [("pressure", mg_scenes.dam_break_2d())], solves=1),
}

PSI_H = (0.0, 1.0, 0.0)
PSI_PIN = (1, 1, 1)


def psi_chi(scene):
    """Susceptibility of the potential solve: 1 inside the fluid, 0 outside."""
    return (scene.phi < 0).astype(np.float32)

MAX_ITERS = 500
REL_TOL = 1e-12  # squared: 1e-6 relative residual
DIRECT_LAUNCH = False  # set by --direct

# DRAM bytes (read + write) per launch of the dominant kernels, from one ncu
# capture each of the column-register sweep the autotuner picks for level 0
# (profiles/k_colsweep_l0_precision256.md, profiles/dram_traffic_substep128.md);
# the bench line's roofline.traffic.  At 128^3 the sweeps' writes stay in L2.
NCU_DRAM_BYTES = {
    ("substep128", "pre_l0"): 16.83e6, ("substep128", "post_l0"): 26.29e6,
    ("pressure128", "pre_l0"): 16.83e6, ("pressure128", "post_l0"): 26.29e6,
    ("substep128", "Ap_alpha"): 11.70e6, ("pressure128", "Ap_alpha"): 11.70e6,
    ("substep128", "xr"): 24.33e6, ("pressure128", "xr"): 24.33e6,
    ("precision256", "pre_l0"): 191.3e6, ("precision256", "post_l0"): 268.9e6,
}


def workload_config(args, world):
    """The workload both arms run (the same dict in the GPU and reference lines)."""
    wl = WORKLOADS[args.workload]
    return {"workload": args.workload, "desc": wl["desc"], "storage": args.storage,
            "solves_per_step": wl["solves"],
            "max_iters": MAX_ITERS, "rel_resid": 1e-6, "parallelism": f"replicas x{world}",
            "l2": "flushed between timed solves (a 256 MB buffer written before each; L2 is 126 MB)"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="substep128", choices=list(WORKLOADS))
    ap.add_argument("--storage", default="f32", choices=["f32", "f16", "bf16"])
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU baseline sample length")
    ap.add_argument("--no-variants", action="store_true", help="skip the batched / served comparison")
    ap.add_argument("--direct", action="store_true",
                    help="launch the PCG iterations from a host loop instead of the CUDA graph (the same "
                         "kernels; for profilers that do not follow conditional graph nodes; slower)")
    return ap.parse_args()


# ---------------------------------------------------------------- distributed
def dist_init(n, group=True):
    """Rank, world size and local rank from torchrun's environment.  With
    `group` and more than one rank, joins the process group: NCCL with the
    local GPU selected where CUDA is present, else gloo (the host-logic tests).
    The reference arm passes group=False: rank 0 alone works, so its ranks
    take no collective step."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and group:
        import torch
        import torch.distributed as dist
        import datetime
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def max_over_ranks(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(v)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------- clocks
class Clocks:
    """nvidia-smi sampled every 100 ms while the timed region runs."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                        rows.append(parts)
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = sorted(float(r[1]) for r in rows)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": float(rows[0][2]), "reasons": reasons,
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())
                if any(r[3].replace(".", "").isdigit() for r in rows) else None}


# ---------------------------------------------------------------- GPU arm
class PsiCase:
    """The magnetic potential solve: full_reinitialize + solve (ferrofluid_simulator.py:77-87)."""

    kind = "psi"

    def __init__(self, scene, storage, dev):
        import torch
        from mgpcg import MGPCGPoissonSolver
        from magnetic_potential import MagneticPotentialStrategy
        self.scene = scene
        self.dev = dev
        # the potential operator has stored coefficients: always float32 grids
        self.solver = MGPCGPoissonSolver(scene.dim, scene.res, scene.levels, 2, 50, device=dev,
                                         direct_launch=DIRECT_LAUNCH)
        self.chi = torch.from_numpy(psi_chi(scene)).to(dev)
        self.strategy = MagneticPotentialStrategy(scene.dim, self.chi, PSI_H, scene.dx, PSI_PIN)
        self.h_chi = torch.from_numpy(psi_chi(scene)).pin_memory()
        self.h_x = torch.empty(scene.res, dtype=torch.float32).pin_memory()
        self.x_stage = torch.empty(scene.res, dtype=torch.float32, device=dev)
        self.h2d_bytes = self.h_chi.numel() * 4
        self.d2h_bytes = self.h_x.numel() * 4

    def upload(self):
        """H2D of a step's inputs (on the current stream)."""
        self.chi.copy_(self.h_chi, non_blocking=True)

    def setup(self):
        self.solver.full_reinitialize(self.strategy)

    def run(self):
        self.setup()
        self.solver.solve_async(MAX_ITERS, REL_TOL)


def make_case(kind, scene, storage, dev):
    return PsiCase(scene, storage, dev) if kind == "psi" else GpuCase(scene, storage, dev)


class GpuCase:
    """One pressure solve of a scene through the drop-in API with device-resident inputs."""

    kind = "pressure"

    def __init__(self, scene, storage, dev):
        import torch
        from mgpcg import MGPCGPoissonSolver
        from pressure_project import PressureProjectStrategy
        self.scene = scene
        self.dev = dev
        self.solver = MGPCGPoissonSolver(scene.dim, scene.res, scene.levels, 2, 50, storage=storage, device=dev,
                                         direct_launch=DIRECT_LAUNCH)
        self.vel = [torch.from_numpy(v).to(dev) for v in scene.velocity]
        self.phi = torch.from_numpy(scene.phi).to(dev)
        self.ct = torch.from_numpy(scene.cell_type).to(dev)
        self.extra = torch.from_numpy(scene.extra_rhs).to(dev) if scene.extra_rhs is not None else None
        self.strategy = PressureProjectStrategy(scene.dim, self.vel, True, self.phi, scene.p0,
                                                gfm_clamp=scene.gfm_clamp)
        self.strategy.scale_A = scene.scale_A
        self.strategy.scale_b = scene.scale_b
        # pinned host copies for the end-to-end path
        self.h_vel = [torch.from_numpy(v).pin_memory() for v in scene.velocity]
        self.h_phi = torch.from_numpy(scene.phi).pin_memory()
        self.h_ct = torch.from_numpy(scene.cell_type).pin_memory()
        self.h_x = torch.empty(scene.res, dtype=torch.float32).pin_memory()
        self.x_stage = torch.empty(scene.res, dtype=torch.float32, device=dev)
        self.h2d_bytes = sum(t.numel() * t.element_size() for t in self.h_vel) + \
            self.h_phi.numel() * 4 + self.h_ct.numel() * 4
        self.d2h_bytes = self.h_x.numel() * 4

    def setup(self):
        s = self.solver
        s.reinitialize(self.ct, self.strategy)
        if self.extra is not None:
            from mg_lib import check
            check(s.lib.mg_add_rhs(s.plan, self.extra.data_ptr(), 1.0, s._s()), "mg_add_rhs")

    def run(self):
        """reinitialize + solve, enqueued; returns nothing (stats read later)."""
        self.setup()
        self.solver.solve_async(MAX_ITERS, REL_TOL)

    def upload(self):
        """H2D of a step's inputs (on the current stream): velocities, phi, labels."""
        for d, h in zip(self.vel, self.h_vel):
            d.copy_(h, non_blocking=True)
        self.phi.copy_(self.h_phi, non_blocking=True)
        self.ct.copy_(self.h_ct, non_blocking=True)


def stage_bytes(solver, storage):
    """Algorithmic bytes per level-0 cell of each pipeline stage: every array a
    stage must read or write once (labels and couplings only where the stage
    needs them; the coarse arrays per fine cell), without re-reads."""
    sv = 4 if storage == "f32" else 2
    d = solver.dim
    coarse = 2 ** d
    cg = {
        "Ap_alpha": 4 + 4 + 4 * d + 1 + 4,                     # p, Adiag, Ax, label, Ap out
        "xr": 4 * 4 + 1 + 2 * 4,                               # x, p, r, Ap, label; x, r out
    }
    if solver.operator_form(0) == 1:  # fused V-cycle kernels of the label-uniform form
        return dict(cg, **{
            "Ap_alpha": 4 + 4 + 4,                              # Adiag, p; Ap out (no Ax, no labels)
            "pre_l0": 4 + sv + sv + 2 * sv / coarse,           # r, Ad; z out, r_c + z_c out
            "post_l0": sv + sv / coarse + 4 + sv + sv,          # zt, z_c, r, Ad; z out
        })
    return {
        "pre_l0": 4 + sv + 1 + sv + 2 * sv / coarse,          # r, Ad, label, z out, r_c + z_c out
        "post_l0": sv + sv / coarse + 4 + sv + 1 + sv,         # z, z_c, r, Ad, label, z out
        "Ap_alpha": 4 + 4 + 4 * d + 1 + 4,                     # p, Adiag, Ax, label, Ap out
        "xr": 4 * 4 + 1 + 2 * 4,                               # x, p, r, Ap, label; x, r out
    }


def time_stages(case, storage, reps=20):
    """CUDA-event time of each pipeline stage on the solver's stream."""
    import torch
    s = case.solver
    stream = torch.cuda.current_stream(case.dev)
    out = {}
    stages = {"pre_l0": (0, 0), "post_l0": (1, 0), "coarse": (2, 0), "Ap_alpha": (3, 0), "xr": (4, 0),
              "vcycle": (5, 0)}
    on, first = s.resident()
    if on:  # the cluster launch (levels `first` down) replaces the coarse block
        stages.pop("coarse")
        stages["cluster"] = (6, 0)
        if first == 0:
            stages.pop("pre_l0")
            stages.pop("post_l0")
    for name, (st, lv) in stages.items():
        try:
            s.launch_stage(st, lv)
        except Exception:
            continue
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            s.launch_stage(st, lv)
        e1.record(stream)
        torch.cuda.synchronize()
        out[name] = e0.elapsed_time(e1) / reps
    return out


def gpu_arm(args, rank, world, local):
    import torch
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    wl = WORKLOADS[args.workload]
    cases = [make_case(kind, sc, args.storage, dev) for kind, sc in wl["cases"]()]
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        times = []
        for c in cases:
            flush.fill_(1)  # L2 flush, outside the timed region
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            c.run()
            e1.record(stream)
            times.append((e0, e1))
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in times]

    def e2e_run(k_steps):
        """k_steps steps through host buffers, pipelined over two streams: a
        step's inputs are uploaded (pinned H2D, copy stream) once the step
        before has built its system from the previous ones, and each result
        is staged on the device and read back (D2H, copy stream) while the
        next solve runs.  Every step moves all of its inputs and its result;
        the device time from the first upload to the last read-back is
        returned, with the per-step intervals on the compute stream."""
        copy = torch.cuda.Stream(dev)
        ev = lambda: torch.cuda.Event(enable_timing=True)
        e0 = ev()
        e0.record(stream)
        copy.wait_event(e0)
        up = {}
        back = {}
        with torch.cuda.stream(copy):
            for c in cases:
                c.upload()
                up[c.kind] = torch.cuda.Event()
                up[c.kind].record(copy)
        marks = []
        for k in range(k_steps):
            m = ev()
            m.record(stream)
            marks.append(m)
            for c in cases:
                flush.fill_(1)  # L2 flush between solves, as for the resident-input timing
                stream.wait_event(up[c.kind])
                c.setup()
                free = torch.cuda.Event()
                free.record(stream)
                c.solver.solve_async(MAX_ITERS, REL_TOL)
                if c.kind in back:
                    stream.wait_event(back[c.kind])  # the previous read-back of x_stage is done
                c.x_stage.copy_(c.solver.x)
                done = torch.cuda.Event()
                done.record(stream)
                copy.wait_event(free)
                with torch.cuda.stream(copy):
                    if k + 1 < k_steps:
                        c.upload()
                        up[c.kind] = torch.cuda.Event()
                        up[c.kind].record(copy)
                    copy.wait_event(done)
                    c.h_x.copy_(c.x_stage, non_blocking=True)
                    back[c.kind] = torch.cuda.Event()
                    back[c.kind].record(copy)
        for c in cases:
            stream.wait_event(back[c.kind])
        e1 = ev()
        e1.record(stream)
        torch.cuda.synchronize()
        marks.append(e1)
        per_step = [a.elapsed_time(b) for a, b in zip(marks[:-1], marks[1:])]
        return e0.elapsed_time(e1), per_step

    for _ in range(args.warmup):
        step()
    e2e_run(max(1, args.warmup))
    torch.cuda.synchronize()
    barrier(world)
    with Clocks(local) as clk:
        solve_ms = []
        iters = []
        per_case_iters = {c.kind: [] for c in cases}
        for _ in range(args.steps):
            solve_ms += step()
            for c in cases:
                st = c.solver.stats()
                iters.append((c, st.iters))
                per_case_iters[c.kind].append(st.iters)
        torch.cuda.synchronize()
    barrier(world)
    e2e_total, e2e_steps = e2e_run(args.steps)
    torch.cuda.synchronize()
    for c in cases:  # the pipeline delivered the last step's result to the host
        if not torch.equal(c.h_x, c.solver.x.cpu()):
            raise RuntimeError(f"e2e read-back of the {c.kind} solve differs from the device result")
    total_ms = max_over_ranks(sum(solve_ms), world)
    total_e2e = max_over_ranks(e2e_total, world)
    n_solves = len(solve_ms) * world
    # outcome of the last solve of each case, checked against the target
    rel = [c.solver.last_rel_resid for c in cases]
    status = [c.solver.last_status for c in cases]
    # launches: setup + prologue + iterations * body
    launches = 0
    for c, it in iters:
        pro, body = c.solver.launch_counts()
        L = c.solver.n_mg_levels
        if c.kind == "psi":   # build_b, build_A, L-1 Galerkin, prepare (L + 2), set_params
            setup = 2 + (L - 1) + (L + 2) + 1
        else:                 # cell_type, build_b, L build_A, L-1 coarsen, prepare, set_params
            setup = 2 + L + (L - 1) + (L + 2) + (L if c.solver.storage != 0 else 0) + 1
        launches += setup + pro + it * body
    stage_ms = time_stages(cases[0], args.storage)
    sb = stage_bytes(cases[0].solver, args.storage)
    cells = cases[0].scene.cells
    kernels = {}
    for k, ms in stage_ms.items():
        kernels[k] = {"ms": round(ms, 5)}
        if k in sb:
            gbs = sb[k] * cells / (ms * 1e-3) / 1e9
            kernels[k].update({"bytes_per_cell": sb[k], "GB_s": round(gbs, 1)})
    dom = max((k for k in kernels if k in sb), key=lambda k: kernels[k]["ms"])
    peak, peak_source = _hbm_peak()
    lat = sorted(solve_ms)
    res = {
        "metric": "Poisson solves/s at 1e-6 relative residual (p50/p99 ms per solve)",
        "value": round(n_solves / (total_ms * 1e-3), 3),
        "unit": "solves/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(total_ms / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if args.storage == "f32" else f"{args.storage}-storage/f32-arith/f64-dots",
        "data": "synthetic (seeded mg_scenes)",
        "config": workload_config(args, world),
        "timing": {"l2": "flushed before every timed solve",
                   "launch": "direct host loop (profiling)" if DIRECT_LAUNCH else "CUDA graph, device-side while"},
        "p50_ms": round(lat[len(lat) // 2], 4), "p99_ms": round(lat[min(len(lat) - 1, int(0.99 * len(lat)))], 4),
        "pcg_iters": {k: {"min": min(v), "max": max(v)} for k, v in per_case_iters.items()},
        "vcycle": {c.kind: {"operator_form": c.solver.operator_form(0),
                            "split_levels_bits": c.solver.split_levels()[0],
                            "streamed_levels": c.solver.split_levels()[1],
                            "one_plane_step_bits": c.solver.step_planes(),
                            "grid_extra_bits": c.solver.grid_extra(),
                            "sweep_kernel_bits": c.solver.sweep_kernel(),
                            "levels": c.solver.n_mg_levels, "pre_post": 2, "bottom": 50,
                            "cluster_from_level": c.solver.resident()[1] if c.solver.resident()[0] else None}
                   for c in cases},
        "last_rel_resid": rel, "last_status": status,
        "cell_iters_per_s": round(sum(c.scene.cells * (i + 1) for c, i in iters) * world / (total_ms * 1e-3), 1),
        "e2e": {"value": round(n_solves / (total_e2e * 1e-3), 3), "unit": "solves/s",
                "h2d_bytes_per_step": sum(c.h2d_bytes for c in cases),
                "d2h_bytes_per_step": sum(c.d2h_bytes for c in cases),
                "p50_step_ms": round(sorted(e2e_steps)[len(e2e_steps) // 2], 4),
                "pipeline": "two streams: step k+1's uploads and step k's read-back overlap the solves"},
        "gpu_launches": launches * world,
        "roofline": {"bound": "hbm", "kernel": dom,
                     "achieved": kernels[dom]["GB_s"], "peak": peak, "unit": "GB/s",
                     "frac": round(kernels[dom]["GB_s"] / peak, 4), "peak_source": peak_source,
                     "traffic": NCU_DRAM_BYTES.get((args.workload, dom)) if args.storage == "f32" else None,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per launch, profiles/"},
        "kernels": kernels,
        "clocks": clk.summary(),
    }
    return res, cases


# ---------------------------------------------------------------- batched / served forms
def variants(dev, reps=3):
    """The 96-instance uneven batch, the served session stream at swept
    arrival rates, and the 256^3 precision scene in f32 / f16 / bf16 storage,
    each against the plain FP32 one-at-a-time form on the same GPU
    (device-resident inputs; the batch and the precision solves are timed
    with CUDA events, serving by wall clock per request)."""
    batched, classes = batched_variant(dev, reps)
    import mg_tune
    out = {"batched": batched, "served": served_variant(dev, tuned=mg_tune.class_params(classes))}
    out["psi_coarse_forms"] = psi_coarse_variant(dev)
    out["precision256"], xs = precision_variant(dev)
    return out, xs


def psi_coarse_variant(dev, reps=3):
    """The substep's magnetic potential solve at 128^3 with its coarse levels
    as half the Galerkin operator (the default) and rediscretised as the
    reference's potential Strategy builds them (chi re-sampled per level, dx
    2^l): iterations and device ms of full_reinitialize + solve."""
    import torch
    from magnetic_potential import MagneticPotentialStrategy
    from mgpcg import MGPCGPoissonSolver
    sc = mg_scenes.ferro_drop_3d(n=128, seed=1, levels=5)
    chi = torch.from_numpy(psi_chi(sc)).to(dev)
    stream = torch.cuda.current_stream(dev)
    out = {}
    for coarse in ("galerkin", "rediscretise"):
        g = MGPCGPoissonSolver(3, sc.res, 5, 2, 50, device=dev)
        st = MagneticPotentialStrategy(3, chi, PSI_H, sc.dx, PSI_PIN, coarse=coarse)
        g.full_reinitialize(st)
        g.solve(MAX_ITERS)
        ms = []
        for _ in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            g.full_reinitialize(st)
            g.solve_async(MAX_ITERS, REL_TOL)
            e1.record(stream)
            stt = g.stats()
            ms.append(e0.elapsed_time(e1))
        out["half_galerkin" if coarse == "galerkin" else "rediscretised"] = {
            "iters": stt.iters, "status": g.last_status, "ms_per_solve": round(min(ms), 3)}
        g.close()
    return out


def batched_variant(dev, reps=3):
    import torch
    import mg_batch
    import mg_serve
    params = mg_scenes.batch_scene_params(seed=3)
    scenes = [mg_scenes.instance_scene(d, s, ss, levels=mg_serve.levels_for(d, s)) for d, s, ss in params]
    bt = {"instances": len(scenes), "cells": int(sum(s.cells for s in scenes))}
    for storage in ("f32", "f16"):
        b = mg_batch.BatchSolver(scenes, storage=storage, streams=32, device=dev)
        b.solve()
        ms = min(b.solve()[0] for _ in range(reps))
        _, st = b.solve()
        bt[f"batched_{storage}"] = {"solves_per_s": round(len(scenes) / (ms * 1e-3), 1), "batch_ms": round(ms, 3),
                                    "form": "each instance's own CUDA graph on a pool of 32 streams",
                                    "converged": sum(s.status == 0 for s in st),
                                    "iters_max": max(s.iters for s in st)}
        b.solve_batched()
        msb = min(b.solve_batched()[0] for _ in range(reps))
        _, st = b.solve_batched()
        pro, body = b.batch_launch_counts()
        bt[f"batched_kernels_{storage}"] = {"solves_per_s": round(len(scenes) / (msb * 1e-3), 1),
                                            "batch_ms": round(msb, 3),
                                            "converged": sum(s.status == 0 for s in st),
                                            "iters_max": max(s.iters for s in st),
                                            "launches_per_pass": body,
                                            "form": "one launch per V-cycle stage / CG step for all instances "
                                                    "of a sub-batch (tables of blocks), one CUDA graph each, "
                                                    f"{b.batch_groups} sub-batches on their own streams"}
        if storage == "f32":
            b.solve_one_at_a_time()
            ms1 = min(b.solve_one_at_a_time()[0] for _ in range(2))
            bt["plain_f32_one_at_a_time"] = {"solves_per_s": round(len(scenes) / (ms1 * 1e-3), 1),
                                             "batch_ms": round(ms1, 3)}
        del b
        torch.cuda.empty_cache()
    # the sweeps per level, bottom sweeps and level count chosen by measurement
    # (mg_tune) per size class, instead of the fixed rule (2, 50, levels_for)
    import mg_tune
    per_scene, classes = mg_tune.tune_classes(scenes, "f32", dev, bottoms=(10, 50), reps=1)
    b = mg_batch.BatchSolver(scenes, storage="f32", streams=32, device=dev, params=per_scene)
    b.solve()
    ms = min(b.solve()[0] for _ in range(reps))
    _, st = b.solve()
    bt["batched_tuned_f32"] = {"solves_per_s": round(len(scenes) / (ms * 1e-3), 1), "batch_ms": round(ms, 3),
                               "form": "streams, tuned (levels, pre_post, bottom) per size class",
                               "converged": sum(s.status == 0 for s in st), "iters_max": max(s.iters for s in st),
                               "classes": {f"{k[0]}D-{['small', 'medium', 'large'][k[1]]}":
                                           {"levels_offset": r["offset"], "pre_post": r["pre_post"],
                                            "bottom": r["bottom"], "ms": r["ms"], "iters": r["iters"],
                                            "tuned_on": r["scene"]} for k, r in classes.items()}}
    del b
    torch.cuda.empty_cache()
    if all(pp == 2 for _, pp, _ in per_scene):  # the batched kernels run pre_post 2
        for storage in ("f32", "f16"):
            b = mg_batch.BatchSolver(scenes, storage=storage, streams=32, device=dev, params=per_scene)
            try:
                b.solve_batched()
            except Exception as e:  # an instance outside the batched kernels' form
                bt[f"batched_kernels_tuned_{storage}"] = {"skipped": str(e)[:200]}
                del b
                continue
            ms = min(b.solve_batched()[0] for _ in range(reps))
            _, st = b.solve_batched()
            bt[f"batched_kernels_tuned_{storage}"] = {
                "solves_per_s": round(len(scenes) / (ms * 1e-3), 1), "batch_ms": round(ms, 3),
                "form": "batched kernels, tuned (levels, pre_post, bottom) per size class",
                "converged": sum(s.status == 0 for s in st), "iters_max": max(s.iters for s in st)}
            del b
            torch.cuda.empty_cache()
    base = bt["plain_f32_one_at_a_time"]["solves_per_s"]
    bt["speedup_vs_plain"] = {k: round(bt[k]["solves_per_s"] / base, 2) for k in bt
                              if k.startswith("batched_") and isinstance(bt[k], dict) and "solves_per_s" in bt[k]}
    bt["tuned_params"] = per_scene_summary(scenes, per_scene)
    return bt, classes


def per_scene_summary(scenes, params):
    """Distinct (dim, side) -> (levels, pre_post, bottom) of a tuned batch."""
    out = {}
    for sc, (L, pp, bot) in zip(scenes, params):
        out[f"{sc.dim}D-{sc.res[0]}"] = [L, pp, bot]
    return out


SERVE_RATES_HZ = (100, 400, 1600, 6400)


def served_variant(dev, n_sessions=32, substeps=20, tuned=None):
    """Open-loop Poisson arrivals of scene sessions drawn from the batch's size
    and domain distribution, at each rate of SERVE_RATES_HZ: served (warm
    starts, continuous batching on 32 streams) in f32 and f16 against the same
    stream solved one request at a time in plain f32 from a cold start; then
    the highest rate again with an HBM budget of a quarter of the sessions'
    total workspace, so that admission queues."""
    import torch
    import mg_serve
    sweep = {}
    for rate in SERVE_RATES_HZ:
        specs = mg_scenes.serving_sessions(seed=4, n_sessions=n_sessions, substeps=substeps, rate_hz=rate)
        scenes = mg_serve.SolveServer(device=dev).scenes_for(specs)
        row = {}
        for storage in ("f32", "f16"):
            srv = mg_serve.SolveServer(storage=storage, streams=32, device=dev)
            srv.warm(specs)
            recs, wall = srv.run(specs, scenes=scenes)
            row[f"served_{storage}"] = dict(mg_serve.summarize(recs, wall), start="warm (previous substep)")
            del srv
            torch.cuda.empty_cache()
        srv = mg_serve.SolveServer(storage="f32", streams=1, device=dev)
        srv.run_one_at_a_time(specs, scenes=scenes)  # creates and warms one solver per shape
        recs, wall = srv.run_one_at_a_time(specs, scenes=scenes)
        row["plain_f32_one_at_a_time"] = dict(mg_serve.summarize(recs, wall), start="cold (x = 0, mgpcg.py:70)")
        base = row["plain_f32_one_at_a_time"]["solves_per_s"]
        if tuned is not None and rate == SERVE_RATES_HZ[-1]:
            # the batch's tuned (levels, pre_post, bottom) per size class
            for storage in ("f32", "f16"):
                tsrv = mg_serve.SolveServer(storage=storage, streams=32, device=dev, params=tuned)
                tsrv.warm(specs)
                recs, wall = tsrv.run(specs, scenes=scenes)
                row[f"served_tuned_{storage}"] = dict(mg_serve.summarize(recs, wall), start="warm (previous substep)")
                del tsrv
                torch.cuda.empty_cache()
        row["speedup_vs_plain"] = {k: round(row[k]["solves_per_s"] / base, 2) for k in row
                                   if k.startswith("served_")}
        sweep[str(rate)] = row
        del srv, scenes
        torch.cuda.empty_cache()
    # the highest rate with a budget that binds
    rate = SERVE_RATES_HZ[-1]
    specs = mg_scenes.serving_sessions(seed=4, n_sessions=n_sessions, substeps=substeps, rate_hz=rate)
    sizes = [mg_serve.plan_bytes(s["dim"], (s["side"],) * s["dim"], mg_serve.levels_for(s["dim"], s["side"]), "f16")
             for s in specs]
    need = sum(sizes)
    budget = max(0.25 * need, 1.05 * max(sizes))  # binds, yet every session fits alone
    scenes = mg_serve.SolveServer(device=dev).scenes_for(specs)
    srv = mg_serve.SolveServer(storage="f16", streams=32, device=dev, hbm_budget=budget)
    srv.warm(specs)
    recs, wall = srv.run(specs, scenes=scenes)
    bound = dict(mg_serve.summarize(recs, wall), rate_hz=rate, budget_bytes=int(budget), demand_bytes=int(need),
                 peak_in_use_bytes=int(srv.peak_in_use), peak_resident_bytes=int(srv.peak_resident),
                 admission_waits=srv.admission_waits, evictions=srv.evictions)
    del srv, scenes
    torch.cuda.empty_cache()
    return {"sessions": n_sessions, "substeps": substeps, "hbm_budget_gb": 120, "rates_hz": list(SERVE_RATES_HZ),
            "by_rate": sweep, "budget_bound_f16": bound}


def true_rel_resid(solver):
    """||b - A x|| / ||b|| over FLUID cells in float64 on the host, from the
    solver's own float32 A, b and x (a check of the reported residual, not a
    solve)."""
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
    return float(np.linalg.norm(r) / np.linalg.norm(np.where(fl, b, 0.0)))


def precision_variant(dev, reps=3):
    """The 256^3 precision scene (6 levels, smooth extra source) in float32
    and in FP16 / BF16 V-cycle storage: solves/s (inputs larger than L2),
    iterations, the true relative residual and the level-0 sweeps' roofline.
    Returns the row and each storage's solution (for the error against the
    FP64 oracle, computed in the CPU leg)."""
    import torch
    sc = mg_scenes.precision_3d(n=256, seed=2, levels=6)
    row = {"scene": sc.name, "cells": sc.cells, "levels": sc.levels}
    xs = {}
    peak = _hbm_peak()[0]
    stream = torch.cuda.current_stream(dev)
    for storage in ("f32", "f16", "bf16"):
        c = GpuCase(sc, storage, dev)
        c.run()
        torch.cuda.synchronize()
        ms = []
        for _ in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            c.run()
            e1.record(stream)
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        st = c.solver.stats()
        status = c.solver.last_status
        true_res = true_rel_resid(c.solver)
        xs[storage] = c.solver.x.cpu().numpy()  # before the stage timing below overwrites x
        stage_ms = time_stages(c, storage)
        sb = stage_bytes(c.solver, storage)
        kern = {}
        for k in ("pre_l0", "post_l0", "Ap_alpha", "xr"):
            if k in stage_ms and k in sb:
                gbs = sb[k] * sc.cells / (stage_ms[k] * 1e-3) / 1e9
                kern[k] = {"ms": round(stage_ms[k], 5), "bytes_per_cell": sb[k], "GB_s": round(gbs, 1),
                           "frac_of_measured_hbm": round(gbs / peak, 4)}
        row[storage] = {"solves_per_s": round(1e3 / min(ms), 3), "ms_per_solve": round(min(ms), 3),
                        "iters": st.iters, "status": status,
                        "solver_rel_resid": math.sqrt(st.rTr / st.bTb) if st.bTb > 0 else 0.0,
                        "true_rel_resid_of_f32_x": true_res, "kernels": kern}
        del c
        torch.cuda.empty_cache()
    row["speedup_vs_f32"] = {k: round(row[k]["solves_per_s"] / row["f32"]["solves_per_s"], 3) for k in ("f16", "bf16")}
    return row, (sc, xs)


def _hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
        return float(peaks["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs"
    except Exception:
        return 6650.0, "fallback 6650 GB/s"


# ---------------------------------------------------------------- CPU (oracle)
def cpu_solve_rate(cases, seconds, threads=None):
    """Solves/s of the CPU oracle (float32, all host threads) on the workload's
    (kind, scene) solves: setup + solve, like the GPU arm's step."""
    from oracle import OracleSolver
    from oracle import oracle as omod
    if threads:
        omod.set_threads(threads)
    n = 0
    t0 = time.perf_counter()
    iters = []
    while True:
        for kind, sc in cases:
            o = OracleSolver(sc.dim, sc.res, sc.levels, 2, 50, real=np.float32)
            if kind == "psi":
                o.full_reinitialize_psi(psi_chi(sc), PSI_H, sc.dx, PSI_PIN)
            else:
                o.reinitialize_pressure(sc.cell_type, sc.velocity, sc.phi, sc.p0, sc.scale_A, sc.scale_b, True,
                                        sc.gfm_clamp)
                if sc.extra_rhs is not None:
                    b = o.get("b")
                    fl = o.get("grid_type") == 0
                    b[fl] = b[fl] + sc.extra_rhs[fl]
                    o.set("b", b)
            iters.append(o.solve(MAX_ITERS, REL_TOL))
            n += 1
        if time.perf_counter() - t0 >= seconds:
            break
    dt = time.perf_counter() - t0
    return n / dt, n, dt, omod.max_threads(), iters


def fp64_errors(scene, xs):
    """Relative L2 error of each solution against the FP64 oracle solve
    converged to a 1e-12 relative residual (the CPU leg's check of the
    precision variant)."""
    from oracle import OracleSolver
    t0 = time.perf_counter()
    o = OracleSolver(scene.dim, scene.res, scene.levels, 2, 50, real=np.float64)
    o.reinitialize_pressure(scene.cell_type, scene.velocity, scene.phi, scene.p0, scene.scale_A, scene.scale_b, True,
                            scene.gfm_clamp)
    b = o.get("b")
    fl = o.get("grid_type") == 0
    b[fl] = b[fl] + scene.extra_rhs[fl].astype(np.float64)
    o.set("b", b)
    it = o.solve(1000, rel_tol=1e-24)
    x64 = o.get("x")
    d = np.linalg.norm(x64)
    out = {k: float(np.linalg.norm(x.astype(np.float64) - x64) / d) for k, x in xs.items()}
    out["fp64_iters"] = it
    out["fp64_solve_s"] = round(time.perf_counter() - t0, 2)
    return out


def reference_arm(args, rank, world):
    if rank != 0:
        return None
    wl = WORKLOADS[args.workload]
    cases = wl["cases"]()
    per_step = []   # seconds per step (all of the workload's solves)
    per_solve = []
    n_solves = 0
    for i in range(args.warmup + args.steps):
        rate, n, dt, cores, iters = cpu_solve_rate(cases, 0.0)
        if i >= args.warmup:
            per_step.append(dt)
            per_solve += [dt / n] * n
            n_solves += n
    tot = sum(per_step)
    v = n_solves / tot
    lat = sorted(x * 1e3 for x in per_solve)
    return {
        "impl": "reference",
        "metric": "Poisson solves/s at 1e-6 relative residual (p50/p99 ms per solve)",
        "value": round(v, 4), "unit": "solves/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(tot / args.steps * 1e3, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded mg_scenes)",
        "config": workload_config(args, world),
        "p50_ms": round(lat[len(lat) // 2], 3), "p99_ms": round(lat[-1], 3),
        "cpu_baseline": {"value": round(v, 4), "unit": "solves/s", "cores": cores, "kind": "port",
                         "sample": f"{args.steps} timed solves of the workload by the C++/OpenMP oracle "
                                   f"(the Taichi reference is not installable)"},
        "e2e": {"value": round(v, 4), "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    global DIRECT_LAUNCH
    args = parse()
    DIRECT_LAUNCH = args.direct
    rank, world, local = dist_init(args.gpus, group=args.impl != "reference")
    if args.impl == "reference":
        out = reference_arm(args, rank, world)
        if out is not None:
            print(json.dumps(out))
        return
    res, cases = gpu_arm(args, rank, world, local)
    if rank == 0:
        with_cpu = world == 1 and args.cpu_seconds > 0
        rate, n, dt, cores, iters = cpu_solve_rate([(c.kind, c.scene) for c in cases], args.cpu_seconds) \
            if with_cpu else (None, 0, 0, 0, [])
        if with_cpu:
            res["cpu_baseline"] = {"value": round(rate, 4), "unit": "solves/s", "cores": cores, "kind": "port",
                                   "sample": f"{n} solves of the workload in {dt:.1f} s by the C++/OpenMP oracle "
                                             f"(float32, {cores} threads); CPU iterations {min(iters)}-{max(iters)}"}
        if world == 1 and not args.no_variants:
            import torch
            res["variants"], (sc256, xs256) = variants(torch.device("cuda", local))
            if with_cpu:
                res["variants"]["precision256"]["error_vs_fp64"] = fp64_errors(sc256, xs256)
            # the same roofline on the 256^3 scene, whose working set does not
            # fit L2 (the honest HBM case for the level-0 sweeps)
            k256 = res["variants"]["precision256"]["f32"]["kernels"]
            dom = max((k for k in ("pre_l0", "post_l0") if k in k256), key=lambda k: k256[k]["ms"])
            res["roofline_hbm_256"] = {"bound": "hbm", "kernel": dom, "workload": "precision256 (256^3, f32)",
                                       "achieved": k256[dom]["GB_s"], "peak": res["roofline"]["peak"],
                                       "unit": "GB/s", "frac": k256[dom]["frac_of_measured_hbm"],
                                       "traffic": NCU_DRAM_BYTES.get(("precision256", dom))}
        print(json.dumps(res))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
