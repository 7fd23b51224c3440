"""ctypes wrapper over the C++ restatement in ``mgpcg_oracle.cpp``.

TEST INFRASTRUCTURE ONLY (the oracle).  Mirrors the reference class
``MGPCGPoissonSolver`` (mgpcg.py:4-238) driven by ``PressureProjectStrategy``
(pressure_project.py:5-70).  Parity against the reference itself is unpinned
(Taichi is unavailable); see the header of ``mgpcg_oracle.cpp``.
"""
import ctypes
import numpy as np

from .build_oracle import build

FIELD = {"b": 0, "x": 1, "p": 2, "Ap": 3, "r": 4, "z": 5, "Adiag": 6, "Ax": 7, "grid_type": 8}

_lib = None


def _load():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(build())
        vp, ip, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
        lib.orc_create.restype = vp
        lib.orc_create.argtypes = [ctypes.c_int, ip, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        lib.orc_destroy.argtypes = [vp]
        lib.orc_set_threads.argtypes = [ctypes.c_int]
        lib.orc_max_threads.restype = ctypes.c_int
        lib.orc_field.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int]
        lib.orc_field.restype = ctypes.c_int
        for name in ("orc_initialize", "orc_v_cycle", "orc_compute_Ap", "orc_fill_fluid"):
            getattr(lib, name).argtypes = [vp]
        for name in ("orc_init_gridtype", "orc_restrict", "orc_prolongate"):
            getattr(lib, name).argtypes = [vp, ctypes.c_int]
        lib.orc_smooth.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        lib.orc_reinitialize_pressure.argtypes = [vp, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(vp), vp,
                                                  ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                  ctypes.c_int, ctypes.c_double]
        lib.orc_full_reinitialize_psi.argtypes = [vp, vp] + [ctypes.c_double] * 4 + [ctypes.c_int] * 3 + \
            [ctypes.c_double]
        lib.orc_reduce.restype = ctypes.c_double
        lib.orc_reduce.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        lib.orc_solve.restype = ctypes.c_int
        lib.orc_solve.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_int, dp, dp, ip]
        _lib = lib
    return _lib


def set_threads(n: int) -> None:
    _load().orc_set_threads(int(n))


def max_threads() -> int:
    return int(_load().orc_max_threads())


class OracleSolver:
    """CPU restatement of ``MGPCGPoissonSolver`` (mgpcg.py:6).

    ``real`` is ``np.float32`` (the reference's default ``real``) or
    ``np.float64`` (the FP64 solve that results are compared against).
    """

    def __init__(self, dim, res, n_mg_levels=4, pre_and_post_smoothing=2, bottom_smoothing=50,
                 real=np.float32):
        self.lib = _load()
        self.dim = dim
        self.res = tuple(int(v) for v in res)
        self.n_mg_levels = n_mg_levels
        self.real = np.dtype(real)
        arr = (ctypes.c_int * 3)(*(list(self.res) + [1] * (3 - dim)))
        self.h = self.lib.orc_create(dim, arr, n_mg_levels, pre_and_post_smoothing, bottom_smoothing,
                                     self.real.itemsize)
        if not self.h:
            raise ValueError(f"oracle rejected dim={dim} res={res} levels={n_mg_levels}")
        self.last_iters = None
        self.last_rTr0 = None
        self.last_rTr = None
        self.last_vcycles = None

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.lib.orc_destroy(h)
            self.h = None

    def shape(self, level=0):
        return tuple(v >> level for v in self.res)

    # ---- field access -------------------------------------------------
    def get(self, name, level=0):
        shp = self.shape(level)
        if name == "grid_type":
            out = np.empty(shp, np.int8)
        elif name == "Ax":
            out = np.empty((self.dim,) + shp, self.real)
        else:
            out = np.empty(shp, self.real)
        rc = self.lib.orc_field(self.h, FIELD[name], level, out.ctypes.data, 0)
        assert rc == 0
        return out

    def set(self, name, value, level=0):
        shp = self.shape(level)
        if name == "grid_type":
            buf = np.ascontiguousarray(value, dtype=np.int8).reshape(shp)
        elif name == "Ax":
            buf = np.ascontiguousarray(value, dtype=self.real).reshape((self.dim,) + shp)
        else:
            buf = np.ascontiguousarray(value, dtype=self.real).reshape(shp)
        rc = self.lib.orc_field(self.h, FIELD[name], level, buf.ctypes.data, 1)
        assert rc == 0

    # ---- reference methods ---------------------------------------------
    def initialize(self):
        self.lib.orc_initialize(self.h)

    def init_gridtype(self, level):
        """grid_type[level-1] -> grid_type[level] (mgpcg.py:46-60, :86)."""
        self.lib.orc_init_gridtype(self.h, level)

    def fill_fluid(self):
        self.lib.orc_fill_fluid(self.h)

    def smooth(self, level, phase):
        self.lib.orc_smooth(self.h, level, phase)

    def restrict(self, level):
        self.lib.orc_restrict(self.h, level)

    def prolongate(self, level):
        self.lib.orc_prolongate(self.h, level)

    def v_cycle(self):
        self.lib.orc_v_cycle(self.h)

    def compute_Ap(self):
        self.lib.orc_compute_Ap(self.h)

    def reduce(self, a, b, acc_mode=1):
        return self.lib.orc_reduce(self.h, FIELD[a], FIELD[b], acc_mode)

    def reinitialize_pressure(self, cell_type, velocity, phi, p0, scale_A, scale_b,
                              ghost_fluid_method=True, gfm_clamp=1e3):
        """reinitialize(cell_type, PressureProjectStrategy) (mgpcg.py:79-87)."""
        ct = np.ascontiguousarray(cell_type, dtype=np.int32)
        assert ct.shape == self.res
        vel = [np.ascontiguousarray(v, dtype=self.real) for v in velocity]
        for k, v in enumerate(vel):
            exp = list(self.res)
            exp[k] += 1
            assert v.shape == tuple(exp), (v.shape, exp)
        ph = np.ascontiguousarray(phi, dtype=self.real)
        ptrs = (ctypes.c_void_p * 3)(*([v.ctypes.data for v in vel] + [None] * (3 - self.dim)))
        self.lib.orc_reinitialize_pressure(self.h, ct.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                           ptrs, ph.ctypes.data, float(p0), float(scale_A),
                                           float(scale_b), int(bool(ghost_fluid_method)), float(gfm_clamp))

    def full_reinitialize_psi(self, chi, H=(0.0, 1.0, 0.0), dx=1.0, pin=(1, 1, 1), coarse_scale=0.5):
        """full_reinitialize (mgpcg.py:89-94) with the magnetic potential Strategy
        of the 3D substep benchmark (harmonic-mean mu faces, pinned cell,
        coarse levels coarse_scale * P^T A P for coarse_scale > 0; for 0 each
        coarse level rediscretised: chi the mean of the children, dx * 2^l)."""
        c = np.ascontiguousarray(chi, dtype=self.real)
        assert c.shape == self.res
        H = list(H) + [0.0] * (3 - len(H))
        pin = list(pin) + [0] * (3 - len(pin))
        self.lib.orc_full_reinitialize_psi(self.h, c.ctypes.data, float(H[0]), float(H[1]), float(H[2]),
                                           float(dx), int(pin[0]), int(pin[1]), int(pin[2]), float(coarse_scale))

    def set_system(self, grid_type, Adiag, Ax, b):
        """Writes a caller-built system (the Strategy protocol, pressure_project.py:41-70)."""
        self.initialize()
        for l in range(self.n_mg_levels):
            self.set("grid_type", grid_type[l], l)
            self.set("Adiag", Adiag[l], l)
            self.set("Ax", Ax[l], l)
        self.set("b", b)

    def solve(self, max_iters=-1, rel_tol=1e-12, abs_tol=1e-14, eps=1e-12, acc_mode=1):
        """PCG solve (mgpcg.py:150-209); returns the reference's ``iter`` count."""
        r0 = ctypes.c_double()
        rr = ctypes.c_double()
        vc = ctypes.c_int()
        it = self.lib.orc_solve(self.h, int(max_iters), float(rel_tol), float(abs_tol), float(eps),
                                int(acc_mode), ctypes.byref(r0), ctypes.byref(rr), ctypes.byref(vc))
        self.last_iters = it
        self.last_rTr0 = r0.value
        self.last_rTr = rr.value
        self.last_vcycles = vc.value
        return it
