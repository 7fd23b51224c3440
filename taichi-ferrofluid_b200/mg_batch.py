"""Batched solves of many independent pressure problems of uneven sizes.

Two forms.  ``solve_batched``: one kernel launch per V-cycle stage and CG
step for all instances of a sub-batch, driven by per-instance tables of
blocks, the sub-batch's whole PCG loop in one CUDA graph that runs while any
of its instances is unconverged (mg_batch_* in the library); a few
sub-batches of nearly equal size run on their own streams, so that one's
latency-bound stages overlap another's.  ``solve``: each instance's own graph
on a pool of streams (below).

Every instance keeps its own solver plan and workspace resident on the device
(its multigrid hierarchy, its previous pressure) and is solved by ONE library
call, ``mg_pressure_solve_async``: reinitialize(cell_type, strategy) + the
device-resident PCG loop captured in a CUDA graph, with no host
synchronization.  A batch enqueues every instance's call across a pool of CUDA
streams, so the small, latency-bound kernels of many instances overlap on the
GPU's 148 SMs; the host waits once per batch.

``solve_one_at_a_time`` is the plain form the batch is compared with: the
reference's usage, reinitialize + a blocking solve per instance, on one stream.
"""
import time

import torch

import mg_lib
from mgpcg import MGPCGPoissonSolver
from pressure_project import PressureProjectStrategy


class Instance:
    """One scene's resident solver and device inputs."""

    def __init__(self, scene, storage, device, levels=None, pre_post=2, bottom=50):
        self.scene = scene
        L = levels if levels is not None else scene.levels
        self.solver = MGPCGPoissonSolver(scene.dim, scene.res, L, pre_post, bottom, storage=storage,
                                         device=device)
        self.ct = torch.from_numpy(scene.cell_type).to(device)
        self.vel = [torch.from_numpy(v).to(device) for v in scene.velocity]
        self.phi = torch.from_numpy(scene.phi).to(device)
        self.strategy = None

    @property
    def workspace_bytes(self):
        return self.solver.workspace.numel()

    def setup(self, stream, warm_start=False):
        sc = self.scene
        self.solver.pressure_setup_async(self.ct, self.vel, self.phi, sc.p0, sc.scale_A, sc.scale_b, True,
                                         sc.gfm_clamp, warm_start=warm_start, stream=stream)

    def launch(self, stream, max_iters, rel_tol, warm_start=False):
        sc = self.scene
        self.solver.pressure_solve_async(self.ct, self.vel, self.phi, sc.p0, sc.scale_A, sc.scale_b, True,
                                         sc.gfm_clamp, max_iters=max_iters, rel_tol=rel_tol,
                                         warm_start=warm_start, stream=stream)

    def solve_blocking(self, max_iters, rel_tol):
        """reinitialize + solve through the drop-in API (mgpcg.py:79-87, :150)."""
        if self.strategy is None:
            sc = self.scene
            self.strategy = PressureProjectStrategy(sc.dim, self.vel, True, self.phi, sc.p0,
                                                    gfm_clamp=sc.gfm_clamp)
            self.strategy.scale_A = sc.scale_A
            self.strategy.scale_b = sc.scale_b
        self.solver.reinitialize(self.ct, self.strategy)
        return self.solver.solve(max_iters, rel_tol=rel_tol)


class BatchSolver:
    def __init__(self, scenes, storage="f32", streams=16, device=None, levels=None, pre_post=2, bottom=50,
                 params=None):
        """``params``: per scene (levels, pre_and_post_smoothing, bottom_smoothing),
        e.g. mg_tune.tune_classes' choice; else ``levels`` (one value or one
        per scene), ``pre_post`` and ``bottom`` for all."""
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        if params is None:
            params = [(levels[i] if isinstance(levels, (list, tuple)) else levels, pre_post, bottom)
                      for i in range(len(scenes))]
        self.instances = [Instance(sc, storage, self.device, *params[i]) for i, sc in enumerate(scenes)]
        self.streams = [torch.cuda.Stream(self.device) for _ in range(streams)]
        # largest instances first: the long solves start early
        self.order = sorted(range(len(self.instances)), key=lambda i: -self.instances[i].scene.cells)
        self._batches = None
        # sub-batches of solve_batched, each its own graph and stream (measured on
        # the 96-instance batch: 1 / 2 / 4 / 8 / 24 groups give 1,836 / 2,082 /
        # 2,348 / 2,465 / 2,535 solves/s in f32)
        self.batch_groups = 8

    @property
    def workspace_bytes(self):
        return sum(i.workspace_bytes for i in self.instances)

    def solve(self, max_iters=500, rel_tol=1e-12, timed=True):
        """Solves every instance; returns (device ms of the whole batch, stats)."""
        main = torch.cuda.current_stream(self.device)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(main)
        for s in self.streams:
            s.wait_event(e0)
        for k, i in enumerate(self.order):
            self.instances[i].launch(self.streams[k % len(self.streams)], max_iters, rel_tol)
        for s in self.streams:
            ev = torch.cuda.Event()
            ev.record(s)
            main.wait_event(ev)
        e1.record(main)
        torch.cuda.synchronize(self.device)
        stats = [inst.solver.stats() for inst in self.instances]
        return e0.elapsed_time(e1), stats

    def solve_batched(self, max_iters=500, rel_tol=1e-12, warm_start=False, groups=None):
        """Every instance's system built (one library call each, no host
        synchronisation), then batched solves: one kernel launch per V-cycle
        stage and CG step for all instances of a group, driven by tables of
        (instance, block), each group's loop in one CUDA graph (mg_batch_*).
        The instances are split into ``groups`` sub-batches of nearly equal
        cell counts (default: ``self.batch_groups``), each on its own stream,
        so that one group's latency-bound coarse launch overlaps another's
        sweeps.  Returns (device ms from the first set-up to the end, stats)."""
        g = self.batch_groups if groups is None else int(groups)
        g = max(1, min(g, len(self.instances)))
        if self._batches is None or len(self._batches) != g:
            self._make_batches(g)
        main = torch.cuda.current_stream(self.device)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(main)
        prm = mg_lib.SolveParams()
        prm.max_iters = int(max_iters)
        prm.rel_tol = float(rel_tol)
        prm.abs_tol = 1e-14
        prm.eps = 1e-12
        prm.warm_start = 1 if warm_start else 0
        for idx, b, _, st in self._batches:
            st.wait_event(e0)
            for i in idx:
                self.instances[i].setup(st, warm_start)
            mg_lib.check(self._lib.mg_batch_solve_async(b, mg_lib.ctypes.byref(prm), st.cuda_stream),
                         "mg_batch_solve_async")
            ev = torch.cuda.Event()
            ev.record(st)
            main.wait_event(ev)
        e1.record(main)
        torch.cuda.synchronize(self.device)
        stats = [inst.solver.stats() for inst in self.instances]
        return e0.elapsed_time(e1), stats

    def _make_batches(self, groups):
        """Tables and graphs of the batched solves, from the instances' prepared
        plans (their launch shapes are fixed once a shape is prepared): the
        instances, largest first, each to the group with the fewest cells."""
        self._free_batches()
        self._lib = mg_lib.load()
        parts = [[] for _ in range(groups)]
        cells = [0] * groups
        for i in self.order:
            k = min(range(groups), key=lambda j: cells[j])
            parts[k].append(i)
            cells[k] += self.instances[i].scene.cells
        # every instance's plan prepared: its set-up has run once
        main = torch.cuda.current_stream(self.device)
        for i in self.order:
            self.instances[i].setup(main)
        torch.cuda.synchronize(self.device)
        self._batches = []
        for idx in parts:
            arr = (mg_lib.ctypes.c_void_p * len(idx))(*[self.instances[i].solver.plan.value for i in idx])
            b = mg_lib.ctypes.c_void_p()
            mg_lib.check(self._lib.mg_batch_create(arr, len(idx), mg_lib.ctypes.byref(b)), "mg_batch_create")
            n = int(self._lib.mg_batch_workspace_bytes(b))
            ws = torch.empty(max(n, 256), dtype=torch.uint8, device=self.device)
            st = torch.cuda.Stream(self.device)
            mg_lib.check(self._lib.mg_batch_bind(b, ws.data_ptr(), st.cuda_stream), "mg_batch_bind")
            self._batches.append((idx, b, ws, st))
        torch.cuda.synchronize(self.device)

    def batch_launch_counts(self):
        """(kernels before the loop, kernels per loop pass), summed over the groups."""
        pro = body = 0
        for _, b, _, _ in self._batches:
            a, c = mg_lib.ctypes.c_int32(), mg_lib.ctypes.c_int32()
            mg_lib.check(self._lib.mg_batch_launch_counts(b, mg_lib.ctypes.byref(a), mg_lib.ctypes.byref(c)),
                         "mg_batch_launch_counts")
            pro += int(a.value)
            body += int(c.value)
        return pro, body

    def _free_batches(self):
        for _, b, _, _ in (getattr(self, "_batches", None) or []):
            if b is not None and b.value:
                self._lib.mg_batch_destroy(b)
        self._batches = None

    def __del__(self):
        if getattr(self, "_batches", None):
            torch.cuda.synchronize(self.device)
            self._free_batches()

    def solve_one_at_a_time(self, max_iters=500, rel_tol=1e-12):
        """The plain form: each instance reinitialized and solved (blocking) in turn."""
        torch.cuda.synchronize(self.device)
        t0 = time.perf_counter()
        iters = [inst.solve_blocking(max_iters, rel_tol) for inst in self.instances]
        torch.cuda.synchronize(self.device)
        return (time.perf_counter() - t0) * 1e3, iters
