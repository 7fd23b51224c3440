"""Drop-in ``LevelSet`` (level_set.py:10-64): the signed-distance field phi
of the fluid at cell centres, with the reference's initialisers.

``phi`` is a float32 CUDA tensor of shape res; ``eps`` = 5 dx is the
interface half width of the smoothed Heaviside / delta (level_set.py:22),
used by the volume-control, magnetic and surface-tension Strategies.
``initialize_with_aabb`` / ``initialize_with_sphere`` write phi on the device
(``mg_level_set_shape``); ``union=True`` takes the minimum with the current
phi instead of overwriting it (several shapes).
"""
import torch

import mg_lib
from mg_lib import check


class LevelSet:
    def __init__(self, dim, res, dx, real=float, device=None):
        if real not in (float, torch.float32, "f32", "float32"):
            raise ValueError("the level set is float32 (real=float)")
        self.dim = int(dim)
        self.res = tuple(int(v) for v in res)[: self.dim]
        self.dx = float(dx)
        self.real = real
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.phi = torch.zeros(self.res, dtype=torch.float32, device=self.device)
        self.eps = 5 * self.dx  # the "thickness" of the interface
        self.lib = mg_lib.load()
        self._res = (mg_lib.ctypes.c_int32 * 3)(*(list(self.res) + [1] * (3 - self.dim)))

    def _shape(self, sphere, a, b, union):
        f3 = mg_lib.ctypes.c_float * 3
        A = f3(*([float(v) for v in a][: self.dim] + [0.0] * (3 - self.dim)))
        B = f3(float(b), 0.0, 0.0) if sphere else f3(*([float(v) for v in b][: self.dim] + [0.0] * (3 - self.dim)))
        check(self.lib.mg_level_set_shape(self.dim, self._res, self.phi.data_ptr(), self.dx, int(sphere), A, B,
                                          int(bool(union)), mg_lib.stream_ptr(self.device)), "mg_level_set_shape")

    def initialize_with_aabb(self, x0, x1, union=False):
        """level_set.py:56-59: signed distance to the box [x0, x1]."""
        self._shape(False, x0, x1, union)

    def initialize_with_sphere(self, x0, r, union=False):
        """level_set.py:61-64: signed distance to the sphere of centre x0, radius r."""
        self._shape(True, x0, r, union)


class FastSweepingLevelSet(LevelSet):
    """FastSweepingLevelSet (level_set.py:258-334): ``redistance()`` turns phi
    into a signed distance with the same zero set - the crossing distances of
    the cells beside the interface (target_surface), then ``repeat_times``
    rounds of fast sweeping (H. Zhao, Math. Comp. 74:603-627, 2005) along each
    axis; ``valid`` and ``phi_temp`` are the reference's scratch fields."""

    def __init__(self, dim, res, dx, real=float, device=None):
        super().__init__(dim, res, dx, real, device)
        self.repeat_times = 2
        self.valid = torch.full(self.res, -1, dtype=torch.int32, device=self.device)
        self.phi_temp = torch.empty(self.res, dtype=torch.float32, device=self.device)

    def redistance(self):
        """level_set.py:329-333."""
        check(self.lib.mg_level_set_redistance(self.dim, self._res, self.phi.data_ptr(), self.phi_temp.data_ptr(),
                                               self.valid.data_ptr(), self.dx, int(self.repeat_times),
                                               mg_lib.stream_ptr(self.device)), "mg_level_set_redistance")

    def propagate(self):
        """level_set.py:283-327: the fast sweeping of phi_temp where valid is -1."""
        check(self.lib.mg_level_set_propagate(self.dim, self._res, self.phi.data_ptr(), self.phi_temp.data_ptr(),
                                              self.valid.data_ptr(), self.dx, int(self.repeat_times),
                                              mg_lib.stream_ptr(self.device)), "mg_level_set_propagate")

    def target_minus(self):
        """level_set.py:124-146 (after valid.fill(-1), which it includes)."""
        check(self.lib.mg_level_set_target_minus(self.dim, self._res, self.phi.data_ptr(), self.phi_temp.data_ptr(),
                                                 self.valid.data_ptr(), self.dx, mg_lib.stream_ptr(self.device)),
              "mg_level_set_target_minus")

    def smoothing(self, phi, phi_temp):
        """level_set.py:148-163: phi = min(mean of the axis neighbours of phi_temp, phi_temp)."""
        check(self.lib.mg_level_set_smooth(self.dim, self._res, phi.data_ptr(), phi_temp.data_ptr(),
                                           mg_lib.stream_ptr(self.device)), "mg_level_set_smooth")

    def build_from_markers(self, markers, total_mk=None):
        """level_set.py:381-392: phi from marker particles - the distance to the
        nearest marker near the markers (distance_to_markers, markers_propagate),
        minus the marker radius 0.99 dx, swept inward (target_minus, propagate),
        then three smoothing passes.  ``markers``: (N, dim) float32 CUDA tensor
        of positions; ``total_mk``: how many of them (default N)."""
        mk = markers.to(device=self.device, dtype=torch.float32).contiguous()
        n = int(mk.shape[0] if total_mk is None else total_mk)
        if mk.dim() != 2 or mk.shape[1] != self.dim or not 0 <= n <= mk.shape[0]:
            raise ValueError("markers must be (N, dim) with total_mk <= N")
        check(self.lib.mg_level_set_markers_distance(self.dim, self._res, self.phi.data_ptr(), self.valid.data_ptr(),
                                                     mk.data_ptr(), n, self.dx, int(self.repeat_times),
                                                     mg_lib.stream_ptr(self.device)), "mg_level_set_markers_distance")
        self.target_minus()
        self.propagate()
        self.smoothing(self.phi, self.phi_temp)
        self.smoothing(self.phi_temp, self.phi)
        self.smoothing(self.phi, self.phi_temp)
