"""Drop-in ``PressureProjectWithVolumeControlStrategy`` (volume_control.py:6-51).

The ghost-fluid pressure Strategy plus a PI controller on the fluid volume:
every ``build_b`` measures the smoothed volume of {phi < 0}, compares it with
the volume of the first step and adds the divergence ``c`` that pushes it back
to every FLUID cell of b.

Same constructor and Strategy protocol as the reference.  The volume sum, the
controller and ``b += c`` run on the device in one library call
(``mg_volume_control``), so a solve with volume control needs no host
synchronisation; the reference reads the volume back and prints it every
step (volume_control.py:47-50).  Here the controller state lives in a device
tensor of 8 doubles and is read only when asked for (``step``, ``vol_0``,
``y``, ``last_volume``, ``last_c``), or printed every step with
``verbose=True``.  The volume is summed over cells in FP64 (the reference sums
f32 atomically in an undefined order).
"""
import torch

import mg_lib
from mg_lib import check
from pressure_project import PressureProjectStrategy, _f32


class PressureProjectWithVolumeControlStrategy(PressureProjectStrategy):
    def __init__(self, dim, velocity, ghost_fluid_method, phi, p0, level_set, dt, gfm_clamp=1e3, verbose=False):
        super().__init__(dim, velocity, ghost_fluid_method, phi, p0, gfm_clamp)
        self.level_set = level_set
        self.dt = float(dt)
        self.verbose = verbose
        # proportional-integral controller (volume_control.py:14-20)
        self.n_p = 25
        self.k_p = 2.3 / (self.n_p * self.dt)  # proportional gain
        self.zeta = 2  # suppresses the noise of the volume computation
        self.k_i = (self.k_p / (2 * self.zeta)) ** 2  # integral gain
        self._state = None
        self._solver = None

    # ------------------------------------------------------------ state
    def _eps(self):
        eps = getattr(self.level_set, "eps", self.level_set)
        return float(eps)

    def _state_on(self, device):
        if self._state is None or self._state.device != device:
            st = torch.zeros(8, dtype=torch.float64, device=device)
            st[5], st[6], st[7] = self.k_p, self.k_i, self.dt
            self._state = st
        return self._state

    def _read(self, i):
        return float(self._state[i].item()) if self._state is not None else 0.0

    @property
    def step(self):
        return int(self._read(0))

    @property
    def vol_0(self):
        return self._read(1)

    @property
    def y(self):
        return self._read(2)

    @property
    def last_volume(self):
        return self._read(3)

    @property
    def last_c(self):
        return self._read(4)

    def _phi(self, solver):
        src = self.phi if self.phi is not None else getattr(self.level_set, "phi", None)
        if src is None:
            raise ValueError("volume control needs phi")
        phi = _f32(src, solver.device)
        if tuple(phi.shape) != solver.res:
            raise ValueError(f"phi shape {tuple(phi.shape)} != {solver.res}")
        return phi

    # ------------------------------------------------------- reference API
    def calc_volume(self, solver=None):
        """volume_control.py:22-31: the smoothed fluid volume (host float)."""
        solver = solver or self._solver
        if solver is None:
            raise ValueError("calc_volume needs a solver (geometry and scratch)")
        phi = self._phi(solver)
        out = torch.zeros(1, dtype=torch.float64, device=solver.device)
        check(solver.lib.mg_level_set_volume(solver.plan, phi.data_ptr(), self._eps(), out.data_ptr(),
                                             solver._s()), "mg_level_set_volume")
        return float(out.item())

    def build_b(self, solver):
        """volume_control.py:39-51."""
        super().build_b(solver)
        self._solver = solver
        phi = self._phi(solver)
        st = self._state_on(solver.device)
        check(solver.lib.mg_volume_control(solver.plan, phi.data_ptr(), self._eps(), st.data_ptr(), solver._s()),
              "mg_volume_control")
        self._keep_phi = phi
        if self.verbose:
            print(f"volume = {self.last_volume}, c = {self.last_c}")
