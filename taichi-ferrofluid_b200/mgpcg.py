"""Drop-in ``MGPCGPoissonSolver`` backed by hand-written sm_100a CUDA kernels.

Same module name, class name, constructor, methods and public fields as the
reference's ``mgpcg.py`` (mgpcg.py:4-238), so the simulators'
``from mgpcg import MGPCGPoissonSolver`` and their calls
``reinitialize(cell_type, strategy)`` / ``full_reinitialize(strategy)`` /
``solve(max_iters, verbose, rel_tol)`` / ``solver.x`` work unchanged.

Fields are PyTorch CUDA tensors that are views into ONE device workspace whose
layout the C library defines (``mg_plan_field``):

* ``b, x, p, Ap``: level 0, float32 (mgpcg.py:21, 39-41);
* ``r[l], z[l]``: the multigrid residual / correction (mgpcg.py:23-26);
  ``r[0]`` is float32, the rest use the V-cycle storage type;
* ``grid_type[l]``: int8 labels FLUID=0, AIR=1, SOLID=2 (mgpcg.py:29);
* ``Adiag[l]``: float32 diagonal (mgpcg.py:33);
* ``Ax[l]``: float32, shape ``(*shape_l, dim)``; ``Ax[l][I][k]`` is
  A(I, I + e_k) as in the reference (mgpcg.py:35).  Storage is SoA underneath.

A Strategy may write these tensors directly (the reference's protocol,
pressure_project.py:41-70) or call the library's build kernels, as
``PressureProjectStrategy`` does.

Differences from the reference, all outside the numbers it produces:
* ``solve`` runs the whole PCG loop on the device in one CUDA graph and
  returns the iteration count; ``last_iters``, ``last_status`` and
  ``last_rel_resid`` report the outcome (the reference returns nothing).
* ``verbose`` prints the initial and final residual only: per-iteration
  values never reach the host.
* inner products and the scalar steps (alpha, beta, the tolerance test) are
  FP64 on the device; the reference sums in float32 atomics.
* ``solve(x0=...)`` (an extension) warm-starts from a given pressure with
  r = b - A x0.
"""
import math

import torch

import mg_lib
from mg_lib import FLUID, AIR, SOLID, check

__all__ = ["MGPCGPoissonSolver", "FLUID", "AIR", "SOLID"]

_TORCH_STORE = {0: torch.float32, 1: torch.float16, 2: torch.bfloat16}


def _as_storage(real, storage):
    if storage is not None:
        key = storage if isinstance(storage, str) else {torch.float32: "f32", torch.float16: "f16",
                                                        torch.bfloat16: "bf16"}[storage]
        return mg_lib.STORE[key]
    return 0


class MGPCGPoissonSolver:
    """mgpcg.py:5-44.  ``real`` is accepted for compatibility and must be a
    32-bit float type (Taichi's ``float`` default).  ``storage`` selects the
    type of the V-cycle grids: "f32" (plain form), "f16" or "bf16" (mixed form:
    16-bit grids, float32 smoother arithmetic, float32 CG, FP64 inner
    products, and a true-residual refresh every ``refresh_every`` iterations).
    """

    def __init__(self, dim, res, n_mg_levels=4, pre_and_post_smoothing=2, bottom_smoothing=50,
                 real=float, *, storage=None, refresh_every=None, device=None, stored_kernels=False,
                 direct_launch=False):
        self.lib = mg_lib.load()
        self.FLUID = FLUID
        self.SOLID = SOLID
        self.AIR = AIR
        if real not in (float, torch.float32, "f32", "float32"):
            raise ValueError("the CUDA solver computes in float32 (real=float)")
        self.dim = int(dim)
        self.res = tuple(int(v) for v in res)[: self.dim]
        self.n_mg_levels = int(n_mg_levels)
        self.pre_and_post_smoothing = int(pre_and_post_smoothing)
        self.bottom_smoothing = int(bottom_smoothing)
        self.real = real
        self.storage = _as_storage(real, storage)
        if refresh_every is None:
            refresh_every = 10 if self.storage != 0 else 0
        self.refresh_every = int(refresh_every)
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())

        d = mg_lib.PlanDesc()
        d.dim = self.dim
        for k in range(3):
            d.res[k] = self.res[k] if k < self.dim else 1
        d.levels = self.n_mg_levels
        d.pre_post = self.pre_and_post_smoothing
        d.bottom = self.bottom_smoothing
        d.storage = self.storage
        d.refresh_every = self.refresh_every
        d.flags = (mg_lib.PLAN_STORED if stored_kernels else 0) | (mg_lib.PLAN_DIRECT if direct_launch else 0)
        plan = mg_lib.ctypes.c_void_p()
        check(self.lib.mg_plan_create(mg_lib.ctypes.byref(d), mg_lib.ctypes.byref(plan)), "mg_plan_create")
        self.plan = plan
        nbytes = int(self.lib.mg_plan_workspace_bytes(plan))
        with torch.cuda.device(self.device):
            self.workspace = torch.zeros(nbytes, dtype=torch.uint8, device=self.device)
            check(self.lib.mg_plan_bind(plan, self.workspace.data_ptr()), "mg_plan_bind")
        self._make_views()
        self.last_iters = None
        self.last_status = None
        self.last_rel_resid = None
        self.last_stats = None

    # ------------------------------------------------------------------ layout
    def shape(self, level=0):
        return tuple(v >> level for v in self.res)

    def _view(self, field, level, dtype, shape, comp=0, ncomp=1):
        off = mg_lib.ctypes.c_int64()
        nb = mg_lib.ctypes.c_int64()
        check(self.lib.mg_plan_field(self.plan, field, level, comp, mg_lib.ctypes.byref(off),
                                     mg_lib.ctypes.byref(nb)), "mg_plan_field")
        n = int(nb.value) * ncomp
        return self.workspace[off.value: off.value + n].view(dtype).view(shape)

    def _make_views(self):
        sd = _TORCH_STORE[self.storage]
        L = self.n_mg_levels
        self.b = self._view(mg_lib.FIELD_B, 0, torch.float32, self.shape(0))
        self.x = self._view(mg_lib.FIELD_X, 0, torch.float32, self.shape(0))
        self.p = self._view(mg_lib.FIELD_P, 0, torch.float32, self.shape(0))
        self.Ap = self._view(mg_lib.FIELD_AP, 0, torch.float32, self.shape(0))
        self.r = [self._view(mg_lib.FIELD_R, l, torch.float32 if l == 0 else sd, self.shape(l)) for l in range(L)]
        self.z = [self._view(mg_lib.FIELD_Z, l, sd, self.shape(l)) for l in range(L)]
        self.grid_type = [self._view(mg_lib.FIELD_TYPE, l, torch.int8, self.shape(l)) for l in range(L)]
        self.Adiag = [self._view(mg_lib.FIELD_ADIAG, l, torch.float32, self.shape(l)) for l in range(L)]
        self.Ax = [self._view(mg_lib.FIELD_AX, l, torch.float32, (self.dim,) + self.shape(l), 0, self.dim)
                   .movedim(0, -1) for l in range(L)]

    def _s(self):
        return mg_lib.stream_ptr(self.device)

    def close(self):
        plan = getattr(self, "plan", None)
        if plan is not None and plan.value:
            self.lib.mg_plan_destroy(plan)
            self.plan = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ----------------------------------------------------- reference methods
    def init_gridtype(self, grid0, grid):
        """mgpcg.py:46-60: grid = coarse labels of grid0 (consecutive levels)."""
        for l in range(1, self.n_mg_levels):
            if grid0 is self.grid_type[l - 1] and grid is self.grid_type[l]:
                check(self.lib.mg_init_gridtype(self.plan, l, self._s()), "mg_init_gridtype")
                return
        raise ValueError("init_gridtype expects grid_type[l-1], grid_type[l] of this solver")

    def initialize(self):
        """mgpcg.py:63-77: zeroes every field."""
        check(self.lib.mg_initialize(self.plan, self._s()), "mg_initialize")

    def _copy_cell_type(self, cell_type):
        ct = torch.as_tensor(cell_type, device=self.device)
        if tuple(ct.shape) != self.res:
            raise ValueError(f"cell_type shape {tuple(ct.shape)} != res {self.res}")
        ct = ct.to(torch.int32).contiguous()
        check(self.lib.mg_set_cell_type(self.plan, ct.data_ptr(), self._s()), "mg_set_cell_type")

    def prepare(self, strategy=None):
        """Chooses the V-cycle operator form for the A just built: the form a
        Strategy declares (``strategy.declared_operator(solver)`` returning
        ("uniform", off-diagonal magnitude per level) or ("whole", None)),
        checked on the device during the solve, else detected (one host
        synchronization)."""
        decl = getattr(strategy, "declared_operator", None) if strategy is not None else None
        form = decl(self) if decl is not None else None
        if form is None:
            check(self.lib.mg_plan_prepare(self.plan, self._s()), "mg_plan_prepare")
        elif form[0] == "uniform":
            od = (mg_lib.ctypes.c_float * self.n_mg_levels)(*[float(v) for v in form[1]])
            check(self.lib.mg_plan_prepare_declared(self.plan, od, self._s()), "mg_plan_prepare_declared")
        elif form[0] == "whole":
            check(self.lib.mg_plan_prepare_declared_whole(self.plan, self._s()), "mg_plan_prepare_declared_whole")
        else:
            raise ValueError(f"unknown declared operator form {form[0]!r}")

    def split_levels(self, bits=None):
        """(bits, streamed levels): the autotuner's per-level choice (bit l: level
        l runs the per-kernel passes); ``bits`` forces a choice until the next
        prepare."""
        b = mg_lib.ctypes.c_uint32(0 if bits is None else int(bits))
        n = mg_lib.ctypes.c_int32(0)
        check(self.lib.mg_plan_split(self.plan, 0 if bits is None else 1, mg_lib.ctypes.byref(b),
                                     mg_lib.ctypes.byref(n)), "mg_plan_split")
        return int(b.value), int(n.value)

    def step_planes(self, bits=None):
        """The autotuner's planes per step of the streamed sweeps: bit 2l (2l+1)
        set = level l's PRE (POST) sweep steps one plane at a time, else two;
        ``bits`` forces a choice until the next prepare."""
        b = mg_lib.ctypes.c_uint32(0 if bits is None else int(bits))
        check(self.lib.mg_plan_steps(self.plan, 0 if bits is None else 1, mg_lib.ctypes.byref(b)),
              "mg_plan_steps")
        return int(b.value)

    def grid_extra(self, bits=None):
        """The autotuner's grid per streamed level: bits 2l..2l+1 = blocks per SM,
        beyond those that fit its shared memory, that level's grid is sized for;
        ``bits`` forces a choice until the next prepare."""
        b = mg_lib.ctypes.c_uint32(0 if bits is None else int(bits))
        check(self.lib.mg_plan_grid(self.plan, 0 if bits is None else 1, mg_lib.ctypes.byref(b)),
              "mg_plan_grid")
        return int(b.value)

    def sweep_kernel(self, bits=None):
        """The autotuner's kernel per streamed level: bits 2l..2l+1 = 0 for the
        shared-memory ring sweep, 1..3 for the column-register sweep with a
        32x16, 32x32 or 64x16 tile; ``bits`` forces a choice until the next
        prepare."""
        b = mg_lib.ctypes.c_uint32(0 if bits is None else int(bits))
        check(self.lib.mg_plan_sweep_kernel(self.plan, 0 if bits is None else 1, mg_lib.ctypes.byref(b)),
              "mg_plan_sweep_kernel")
        return int(b.value)

    def resident(self, on=None, first_level=None):
        """(on, first level): whether the V-cycle runs its levels from the first
        brick level down as one thread-block-cluster launch (the autotuner's
        choice), and that level (-1: the shape has none); ``on`` forces a
        choice until the next prepare, ``first_level`` (with ``on``) the level
        the cluster starts at."""
        o = mg_lib.ctypes.c_int32(0 if on is None else int(bool(on)))
        lp = mg_lib.ctypes.c_int32(-1 if first_level is None else int(first_level))
        check(self.lib.mg_plan_resident(self.plan, 0 if on is None else 1, mg_lib.ctypes.byref(o),
                                        mg_lib.ctypes.byref(lp)), "mg_plan_resident")
        return bool(o.value), int(lp.value)

    def operator_form(self, level=0):
        f = mg_lib.ctypes.c_int32()
        check(self.lib.mg_plan_operator_form(self.plan, level, mg_lib.ctypes.byref(f)), "mg_plan_operator_form")
        return int(f.value)

    def reinitialize(self, cell_type, strategy):
        """mgpcg.py:79-87."""
        self.initialize()
        self._copy_cell_type(cell_type)
        strategy.build_b(self)
        strategy.build_A(self, 0)
        for l in range(1, self.n_mg_levels):
            self.init_gridtype(self.grid_type[l - 1], self.grid_type[l])
            strategy.build_A(self, l)
        self.prepare(strategy)

    def full_reinitialize(self, strategy):
        """mgpcg.py:89-94."""
        self.initialize()
        strategy.build_b(self)
        check(self.lib.mg_fill_fluid(self.plan, self._s()), "mg_fill_fluid")
        for l in range(self.n_mg_levels):
            strategy.build_A(self, l)
        self.prepare(strategy)

    def smooth(self, l, phase):
        """mgpcg.py:104-109."""
        check(self.lib.mg_smooth(self.plan, l, phase, self._s()), "mg_smooth")

    def restrict(self, l):
        """mgpcg.py:111-118 (also zeroes z[l+1], as v_cycle does before it)."""
        check(self.lib.mg_restrict(self.plan, l, self._s()), "mg_restrict")

    def prolongate(self, l):
        """mgpcg.py:120-123."""
        check(self.lib.mg_prolongate(self.plan, l, self._s()), "mg_prolongate")

    def v_cycle(self):
        """mgpcg.py:125-148: z[0] = M^-1 r[0]."""
        check(self.lib.mg_v_cycle(self.plan, self._s()), "mg_v_cycle")

    def compute_Ap(self):
        """mgpcg.py:218-224."""
        check(self.lib.mg_compute_Ap(self.plan, self._s()), "mg_compute_Ap")

    _FIELD_OF = {"b": mg_lib.FIELD_B, "x": mg_lib.FIELD_X, "p": mg_lib.FIELD_P, "Ap": mg_lib.FIELD_AP}

    def _field_id(self, t):
        for name, fid in self._FIELD_OF.items():
            if t is getattr(self, name):
                return fid
        if t is self.r[0]:
            return mg_lib.FIELD_R
        if t is self.z[0]:
            return mg_lib.FIELD_Z
        raise ValueError("reduce expects level-0 fields of this solver")

    def reduce(self, p, q):
        """mgpcg.py:211-216: sum of p*q over level-0 FLUID cells (FP64)."""
        out = mg_lib.ctypes.c_double()
        check(self.lib.mg_reduce(self.plan, self._field_id(p), self._field_id(q), mg_lib.ctypes.byref(out),
                                 self._s()), "mg_reduce")
        return out.value

    def solve(self, max_iters=-1, verbose=False, rel_tol=1e-12, abs_tol=1e-14, eps=1e-12, x0=None):
        """mgpcg.py:150-209 on the device.  Returns the reference's ``iter``."""
        self.solve_async(max_iters, rel_tol, abs_tol, eps, x0)
        st = self.stats()
        if verbose:
            print(f"init rtr = {st.rTr0}")
            print(f"iter {st.iters}, |residual|_2={math.sqrt(max(st.rTr, 0.0))} ({mg_lib.STATUS_NAMES[st.status]})")
        return st.iters

    def solve_async(self, max_iters=-1, rel_tol=1e-12, abs_tol=1e-14, eps=1e-12, x0=None):
        """Enqueues the solve on the current stream without waiting."""
        prm = mg_lib.SolveParams()
        prm.max_iters = int(max_iters)
        prm.rel_tol = float(rel_tol)
        prm.abs_tol = float(abs_tol)
        prm.eps = float(eps)
        prm.warm_start = 0
        if x0 is not None:
            self.x.copy_(torch.as_tensor(x0, device=self.device, dtype=torch.float32).reshape(self.res))
            prm.warm_start = 1
        check(self.lib.mg_pcg_solve_async(self.plan, mg_lib.ctypes.byref(prm), self._s()), "mg_pcg_solve_async")

    def pressure_solve_async(self, cell_type, velocity, phi, p0, scale_A, scale_b, ghost_fluid_method=True,
                             gfm_clamp=1e3, max_iters=500, rel_tol=1e-12, abs_tol=1e-14, eps=1e-12,
                             warm_start=False, stream=None):
        """reinitialize(cell_type, PressureProjectStrategy) + solve in ONE
        library call with no host synchronization (mg_pressure_solve_async):
        many of these can be in flight on different streams.  Inputs are
        device tensors in the layouts of PressureProjectStrategy; with
        ``warm_start`` the current ``x`` is the initial guess."""
        prm = mg_lib.SolveParams()
        prm.max_iters = int(max_iters)
        prm.rel_tol = float(rel_tol)
        prm.abs_tol = float(abs_tol)
        prm.eps = float(eps)
        prm.warm_start = 1 if warm_start else 0
        self._prm = prm  # the call copies it, but keep it alive for clarity
        v2 = velocity[2] if self.dim == 3 else None
        s = stream.cuda_stream if stream is not None else self._s()
        check(self.lib.mg_pressure_solve_async(
            self.plan, cell_type.data_ptr(), velocity[0].data_ptr(), velocity[1].data_ptr(), mg_lib.ptr(v2),
            mg_lib.ptr(phi), float(p0), float(scale_A), float(scale_b), int(bool(ghost_fluid_method)),
            float(gfm_clamp), mg_lib.ctypes.byref(prm), s), "mg_pressure_solve_async")

    def pressure_setup_async(self, cell_type, velocity, phi, p0, scale_A, scale_b, ghost_fluid_method=True,
                             gfm_clamp=1e3, warm_start=False, stream=None):
        """The system half of pressure_solve_async (labels, b, A, coarse
        labels, declared operator form) with no solve: a batch solve
        (mg_batch.BatchSolver.solve_batched) runs the PCG loops of many."""
        v2 = velocity[2] if self.dim == 3 else None
        s = stream.cuda_stream if stream is not None else self._s()
        check(self.lib.mg_pressure_setup_async(
            self.plan, cell_type.data_ptr(), velocity[0].data_ptr(), velocity[1].data_ptr(), mg_lib.ptr(v2),
            mg_lib.ptr(phi), float(p0), float(scale_A), float(scale_b), int(bool(ghost_fluid_method)),
            float(gfm_clamp), int(bool(warm_start)), s), "mg_pressure_setup_async")

    def launch_counts(self):
        """(kernels before the PCG loop, kernels per further iteration)."""
        a, b = mg_lib.ctypes.c_int32(), mg_lib.ctypes.c_int32()
        check(self.lib.mg_plan_launch_counts(self.plan, mg_lib.ctypes.byref(a), mg_lib.ctypes.byref(b)),
              "mg_plan_launch_counts")
        return int(a.value), int(b.value)

    def launch_stage(self, stage, level=0):
        """Launches one pipeline stage once (for timing; see mg_launch_stage)."""
        check(self.lib.mg_launch_stage(self.plan, int(stage), int(level), self._s()), "mg_launch_stage")

    def stats(self, stream=None):
        """Waits for the stream and returns the last solve's outcome."""
        st = mg_lib.SolveStats()
        s = stream.cuda_stream if stream is not None else self._s()
        check(self.lib.mg_pcg_stats(self.plan, mg_lib.ctypes.byref(st), s), "mg_pcg_stats")
        self.last_stats = st
        self.last_iters = st.iters
        self.last_status = mg_lib.STATUS_NAMES.get(st.status, str(st.status))
        self.last_rel_resid = math.sqrt(st.rTr / st.bTb) if st.bTb > 0 else 0.0
        return st
