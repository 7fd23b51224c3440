"""A continuous-batching Poisson solve server.

Requests are substeps of scene sessions: each session is a fluid domain whose
level set moves by half a cell per substep; every substep needs one ghost-fluid
pressure solve (cell_type, coefficients and rhs rebuilt), and the next substep
can only be requested once the previous pressure exists, as in a simulator
(fluid_simulator.py:307-324).  Sessions arrive as an open-loop Poisson process.

The server
* admits a session when its resident workspace fits the HBM budget (sessions
  wait in arrival order otherwise) and keeps its multigrid hierarchy and its
  previous-substep pressure on the device: the pressure is the next solve's
  warm start (``mg_pressure_solve_async`` with warm_start);
* runs every admitted session's current request as soon as it is issued, on a
  pool of CUDA streams, so requests that arrive while others are on the GPU
  overlap with them (continuous batching, not a queue);
* reuses the workspaces of finished sessions for new sessions of the same shape;
* reports per-request latency (issue to completion) and solves/s.

``run_one_at_a_time`` serves the same stream with the plain form: one request
at a time, FP32 grids, cold start, blocking solve through the drop-in API.
"""
import heapq
import math
import time

import numpy as np
import torch

import mg_lib
import mg_scenes
from mgpcg import MGPCGPoissonSolver
from pressure_project import PressureProjectStrategy

FLUID, AIR, SOLID = mg_lib.FLUID, mg_lib.AIR, mg_lib.SOLID


def plan_bytes(dim, res, levels, storage):
    """Workspace bytes a solver of this shape needs (host-side computation),
    with the defaults MGPCGPoissonSolver takes (the mixed form's true-residual
    refresh and its FP64 x)."""
    lib = mg_lib.load()
    d = mg_lib.PlanDesc()
    d.dim = dim
    for k in range(3):
        d.res[k] = res[k] if k < dim else 1
    d.levels = levels
    d.pre_post = 2
    d.bottom = 50
    d.storage = mg_lib.STORE[storage]
    d.refresh_every = 10 if d.storage != 0 else 0
    p = mg_lib.ctypes.c_void_p()
    mg_lib.check(lib.mg_plan_create(mg_lib.ctypes.byref(d), mg_lib.ctypes.byref(p)), "mg_plan_create")
    n = int(lib.mg_plan_workspace_bytes(p))
    lib.mg_plan_destroy(p)
    return n


def levels_for(dim, side):
    """Level count that brings the coarsest grid to 8..16 cells per side."""
    L = 1
    while side % (1 << L) == 0 and (side >> L) >= 8 and L < 8:
        L += 1
    return L


class DeviceScene:
    """A session's fields on the device: fixed MAC velocities, and phi /
    cell_type rebuilt for each substep on the device, the level set shifted
    by 0.5 cell per substep along the session's direction: the union of the
    session's boxes and spheres (LevelSet.initialize_with_aabb / _sphere,
    level_set.py:40-64, moved by the shift), labels by apply_markers with
    the benchmark's phi < 0 rule over a SOLID ring (fluid_simulator.py:151-159,
    :337-341).  One launch per shape plus one for the labels, no allocation."""

    def __init__(self, sess, device):
        dim, side = sess["dim"], sess["side"]
        self.dim, self.side = dim, side
        self.res = (side,) * dim
        self.dx = 1.0 / side
        self.dt = 1.0 / 60.0
        self.rho, self.p0, self.gfm_clamp = 1000.0, 1e-3, 100.0
        self.scale_A = self.dt / (self.rho * self.dx * self.dx)
        self.scale_b = 1.0 / self.dx
        self.direction = np.asarray(sess["direction"], np.float64)
        shapes, vel_seed = mg_scenes.instance_shapes(dim, sess["scene_seed"])
        self.shapes = shapes
        rng = np.random.default_rng(vel_seed)
        self.vel = [torch.from_numpy(v).to(device)
                    for v in mg_scenes.random_velocity(rng, self.res, gravity_dt=-9.8 * self.dt)]
        self.phi = torch.empty(self.res, dtype=torch.float32, device=device)
        self.ct = torch.full(self.res, AIR, dtype=torch.int32, device=device)
        self._res = (mg_lib.ctypes.c_int32 * 3)(*(list(self.res) + [1] * (3 - dim)))
        self.lib = mg_lib.load()
        mg_lib.check(self.lib.mg_init_boundary(dim, self._res, self.ct.data_ptr(), mg_lib.stream_ptr(device)),
                     "mg_init_boundary")

    def build(self, step):
        """phi_t(x) = phi_0(x - 0.5 * step * dx * direction) and the labels, on
        the current stream."""
        shift = 0.5 * step * self.dx * self.direction
        st = mg_lib.stream_ptr(self.phi.device)
        f3 = mg_lib.ctypes.c_float * 3
        for i, (kind, centre, size) in enumerate(self.shapes):
            c = [float(centre[k] + shift[k]) for k in range(self.dim)]
            if kind == "box":
                a = f3(*[c[k] - float(size[k]) for k in range(self.dim)])
                b = f3(*[c[k] + float(size[k]) for k in range(self.dim)])
                sphere = 0
            else:
                a, b, sphere = f3(*c), f3(float(size)), 1
            mg_lib.check(self.lib.mg_level_set_shape(self.dim, self._res, self.phi.data_ptr(), self.dx, sphere, a, b,
                                                     int(i > 0), st), "mg_level_set_shape")
        mg_lib.check(self.lib.mg_apply_markers(self.dim, self._res, self.ct.data_ptr(), self.phi.data_ptr(), 1, st),
                     "mg_apply_markers")


class Session:
    def __init__(self, sid, spec):
        self.sid = sid
        self.spec = spec
        self.t_arrive = spec["t_arrive"]
        self.steps = spec["substeps"]
        self.step = 0
        self.scene = None
        self.solver = None
        self.key = None


class SolveServer:
    def __init__(self, storage="f16", streams=16, hbm_budget=120e9, device=None, max_iters=500, rel_tol=1e-12,
                 params=None):
        """``params(dim, side)`` -> (levels, pre_and_post_smoothing, bottom_smoothing)
        of a session's solver (e.g. from mg_tune); default: levels_for, 2, 50."""
        self.params = params or (lambda dim, side: (levels_for(dim, side), 2, 50))
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.storage = storage
        self.streams = [torch.cuda.Stream(self.device) for _ in range(streams)]
        self.budget = float(hbm_budget)
        self.max_iters = max_iters
        self.rel_tol = rel_tol
        self.pool = {}        # (dim, side, levels) -> free solvers (resident workspaces)
        self.in_use = 0.0     # bytes held by admitted sessions
        self.peak_in_use = 0.0
        self.admission_waits = 0  # sessions that arrived while the budget was full
        self.idle = 0.0       # bytes of pooled workspaces no session holds
        self.evictions = 0
        self.peak_resident = 0.0  # admitted + idle workspace bytes
        self.bytes_of = {}

    def warm(self, specs):
        """Fills the pool before serving: one resident solver per session of
        each shape that the HBM budget allows, each run once (workspace
        allocated, operator prepared, solve graph instantiated), so that no
        allocation or graph build synchronises the device while serving."""
        need = {}
        for sp in specs:
            key = (sp["dim"], sp["side"]) + tuple(self.params(sp["dim"], sp["side"]))
            need[key] = need.get(key, 0) + 1
        total = self.in_use + self.idle
        for key, n in sorted(need.items(), key=lambda kv: -kv[0][1]):
            dim, side, L, pp, bot = key
            if key not in self.bytes_of:
                self.bytes_of[key] = plan_bytes(dim, (side,) * dim, L, self.storage)
            spec = next(sp for sp in specs if (sp["dim"], sp["side"]) == (dim, side))
            scene = DeviceScene(spec, self.device)
            scene.build(0)
            have = len(self.pool.get(key, []))
            for _ in range(max(0, n - have)):
                if total + self.bytes_of[key] > self.budget:
                    break
                total += self.bytes_of[key]
                self.idle += self.bytes_of[key]
                solver = MGPCGPoissonSolver(dim, (side,) * dim, L, pp, bot, storage=self.storage, device=self.device)
                solver.pressure_solve_async(scene.ct, scene.vel, scene.phi, scene.p0, scene.scale_A, scene.scale_b,
                                            True, scene.gfm_clamp, max_iters=self.max_iters, rel_tol=self.rel_tol)
                self.pool.setdefault(key, []).append(solver)
        self.peak_resident = max(self.peak_resident, self.in_use + self.idle)
        torch.cuda.synchronize(self.device)

    def scenes_for(self, specs):
        """The sessions' payloads (velocities, phi / label buffers) on the device,
        in arrival order: what requests carry when they arrive."""
        return [DeviceScene(s, self.device) for s in sorted(specs, key=lambda s: s["t_arrive"])]

    def _acquire(self, dim, side):
        L, pp, bot = self.params(dim, side)
        key = (dim, side, L, pp, bot)
        if key not in self.bytes_of:
            self.bytes_of[key] = plan_bytes(dim, (side,) * dim, L, self.storage)
        need = self.bytes_of[key]
        if need > self.budget:
            raise ValueError(f"a {dim}D {side}-cell session needs {need} bytes, more than the whole "
                             f"HBM budget of {int(self.budget)}")
        if self.in_use + need > self.budget:
            return None, key
        free = self.pool.get(key)
        if free:
            self.in_use += need
            self.idle -= need
            self.peak_in_use = max(self.peak_in_use, self.in_use)
            return free.pop(), key
        # a new workspace: idle workspaces of other shapes are freed first when
        # resident bytes (admitted + idle) would pass the budget
        self._evict(self.budget - need)
        self.in_use += need
        self.peak_in_use = max(self.peak_in_use, self.in_use)
        self.peak_resident = max(self.peak_resident, self.in_use + self.idle)
        return MGPCGPoissonSolver(dim, (side,) * dim, L, pp, bot, storage=self.storage, device=self.device), key

    def _evict(self, limit):
        """Frees idle pooled workspaces, largest first, until admitted + idle
        bytes are at most ``limit``."""
        while self.in_use + self.idle > limit:
            keys = [k for k, v in self.pool.items() if v]
            if not keys:
                return
            k = max(keys, key=lambda k: self.bytes_of[k])
            solver = self.pool[k].pop()
            solver.close()
            self.idle -= self.bytes_of[k]
            self.evictions += 1

    def _release(self, sess):
        self.pool.setdefault(sess.key, []).append(sess.solver)
        self.in_use -= self.bytes_of[sess.key]
        self.idle += self.bytes_of[sess.key]
        sess.solver = None

    def run(self, specs, warm_start=True, on_complete=None, scenes=None):
        """Serves the sessions; returns per-request records and the wall time.
        ``on_complete(session_id, step, solver)`` is called after each request.
        ``scenes`` (from ``scenes_for``) supplies the payloads; without it each
        session's scene is built at admission, inside the served time."""
        sessions = [Session(i, s) for i, s in enumerate(sorted(specs, key=lambda s: s["t_arrive"]))]
        waiting = list(sessions)        # arrived or not yet, in arrival order
        active = []                     # admitted, with no request in flight
        inflight = []                   # (session, stream, event, t_issue)
        free_streams = list(range(len(self.streams)))
        records = []
        torch.cuda.synchronize(self.device)
        t0 = time.perf_counter()
        done = 0
        while done < len(sessions):
            now = time.perf_counter() - t0
            # admission in arrival order, against the HBM budget
            while waiting and waiting[0].t_arrive <= now:
                s = waiting[0]
                solver, key = self._acquire(s.spec["dim"], s.spec["side"])
                if solver is None:
                    if not getattr(s, "waited", False):
                        s.waited = True
                        self.admission_waits += 1
                    break
                waiting.pop(0)
                s.solver, s.key = solver, key
                s.scene = scenes[s.sid] if scenes is not None else DeviceScene(s.spec, self.device)
                s.t_ready = max(now, s.t_arrive)
                active.append(s)
            # issue every ready session's next substep on a free stream
            while active and free_streams:
                s = active.pop(0)
                k = free_streams.pop()
                st = self.streams[k]
                st.wait_stream(torch.cuda.current_stream(self.device))  # the session's uploads
                with torch.cuda.stream(st):
                    s.scene.build(s.step)
                    sc = s.scene
                    s.solver.pressure_solve_async(sc.ct, sc.vel, sc.phi, sc.p0, sc.scale_A, sc.scale_b, True,
                                                  sc.gfm_clamp, max_iters=self.max_iters, rel_tol=self.rel_tol,
                                                  warm_start=warm_start and s.step > 0, stream=st)
                    ev = torch.cuda.Event()
                    ev.record(st)
                inflight.append((s, k, ev, s.t_ready))
            # completions
            still = []
            for s, k, ev, t_issue in inflight:
                if ev.query():
                    t_done = time.perf_counter() - t0
                    stt = s.solver.stats(stream=self.streams[k])
                    records.append(dict(session=s.sid, step=s.step, dim=s.spec["dim"], side=s.spec["side"],
                                        latency_ms=(t_done - t_issue) * 1e3, iters=stt.iters,
                                        status=mg_lib.STATUS_NAMES.get(stt.status, str(stt.status)),
                                        rel=math.sqrt(stt.rTr / stt.bTb) if stt.bTb > 0 else 0.0))
                    if on_complete is not None:
                        on_complete(s.sid, s.step, s.solver)
                    free_streams.append(k)
                    s.step += 1
                    if s.step >= s.steps:
                        self._release(s)
                        done += 1
                    else:
                        s.t_ready = t_done
                        active.append(s)
                else:
                    still.append((s, k, ev, t_issue))
            inflight = still
            if not inflight and not active and waiting and waiting[0].t_arrive > now:
                time.sleep(min(0.001, waiting[0].t_arrive - now))
        torch.cuda.synchronize(self.device)
        wall = time.perf_counter() - t0
        return records, wall

    def run_one_at_a_time(self, specs, scenes=None):
        """The plain form: FIFO, one request at a time, FP32 grids, cold start,
        blocking reinitialize + solve through the drop-in API."""
        sessions = [Session(i, s) for i, s in enumerate(sorted(specs, key=lambda s: s["t_arrive"]))]
        records = []
        torch.cuda.synchronize(self.device)
        t0 = time.perf_counter()
        # requests are served in issue order; a session's next substep is
        # issued when its previous one completes
        heap = [(s.t_arrive, s.sid) for s in sessions]
        heapq.heapify(heap)
        solvers = self.__dict__.setdefault("_plain_solvers", {})  # one per shape, kept across runs
        while heap:
            t_issue, sid = heapq.heappop(heap)
            s = sessions[sid]
            now = time.perf_counter() - t0
            if now < t_issue:
                time.sleep(t_issue - now)
            if s.scene is None:
                s.scene = scenes[sid] if scenes is not None else DeviceScene(s.spec, self.device)
            L = levels_for(s.spec["dim"], s.spec["side"])
            key = (s.spec["dim"], s.spec["side"], L)
            if key not in solvers:
                solvers[key] = MGPCGPoissonSolver(s.spec["dim"], (s.spec["side"],) * s.spec["dim"], L, 2, 50,
                                                  device=self.device)
            solver = solvers[key]
            sc = s.scene
            sc.build(s.step)
            strat = PressureProjectStrategy(sc.dim, sc.vel, True, sc.phi, sc.p0, gfm_clamp=sc.gfm_clamp)
            strat.scale_A, strat.scale_b = sc.scale_A, sc.scale_b
            solver.reinitialize(sc.ct, strat)
            it = solver.solve(self.max_iters, rel_tol=self.rel_tol)
            t_done = time.perf_counter() - t0
            records.append(dict(session=sid, step=s.step, dim=s.spec["dim"], side=s.spec["side"],
                                latency_ms=(t_done - t_issue) * 1e3, iters=it, status=solver.last_status,
                                rel=solver.last_rel_resid))
            s.step += 1
            if s.step < s.steps:
                heapq.heappush(heap, (t_done, sid))
        torch.cuda.synchronize(self.device)
        return records, time.perf_counter() - t0


def summarize(records, wall):
    lat = np.array([r["latency_ms"] for r in records])
    return dict(solves=len(records), wall_s=round(wall, 4), solves_per_s=round(len(records) / wall, 2),
                p50_ms=round(float(np.percentile(lat, 50)), 3), p99_ms=round(float(np.percentile(lat, 99)), 3),
                iters_mean=round(float(np.mean([r["iters"] for r in records])), 2),
                converged=sum(r["status"] == "converged" for r in records),
                max_rel_resid=float(max(r["rel"] for r in records)))
