"""Drop-in ``PressureProjectStrategy``: the ghost-fluid pressure coefficients.

Same module, class, constructor and Strategy protocol as the reference's
``pressure_project.py`` (pressure_project.py:5-70): the caller sets
``scale_A`` and ``scale_b`` (fluid_simulator.py:178-179), the solver calls
``build_b(solver)`` and ``build_A(solver, level)``.  The work runs in the
library's CUDA kernels ``mg_build_pressure_b`` / ``mg_build_pressure_A``, with
the reference's operation order, so b and A match it bit for bit.

``velocity`` is a list of ``dim`` float32 tensors with shapes res + e_k (MAC
faces) and ``phi`` a float32 tensor of shape res, on the solver's device.
``gfm_clamp`` caps the ghost-fluid factor (phi_i - phi_j) / phi_i; the
reference hard-codes 1e3 (pressure_project.py:37, :62).
"""
import torch

import mg_lib
from mg_lib import check


def _f32(t, device):
    return torch.as_tensor(t, device=device).to(torch.float32).contiguous()


class PressureProjectStrategy:
    def __init__(self, dim, velocity, ghost_fluid_method, phi, p0, gfm_clamp=1e3):
        self.dim = dim
        self.velocity = velocity
        self.ghost_fluid_method = ghost_fluid_method
        self.phi = phi
        self.p0 = p0  # the standard atmospheric pressure
        self.gfm_clamp = gfm_clamp
        self.scale_A = None
        self.scale_b = None

    def _inputs(self, solver):
        dev = solver.device
        vel = [_f32(v, dev) for v in self.velocity]
        for k, v in enumerate(vel):
            exp = list(solver.res)
            exp[k] += 1
            if tuple(v.shape) != tuple(exp):
                raise ValueError(f"velocity[{k}] shape {tuple(v.shape)} != {tuple(exp)}")
        phi = _f32(self.phi, dev) if self.phi is not None else None
        if phi is not None and tuple(phi.shape) != solver.res:
            raise ValueError(f"phi shape {tuple(phi.shape)} != {solver.res}")
        return vel, phi

    def _scales(self):
        if self.scale_A is None or self.scale_b is None:
            raise ValueError("set strategy.scale_A and strategy.scale_b before the solve "
                             "(fluid_simulator.py:178-179)")
        return float(self.scale_A), float(self.scale_b)

    def build_b(self, solver):
        """pressure_project.py:15-43."""
        sA, sB = self._scales()
        vel, phi = self._inputs(solver)
        v2 = vel[2] if self.dim == 3 else None
        check(solver.lib.mg_build_pressure_b(solver.plan, vel[0].data_ptr(), vel[1].data_ptr(),
                                             mg_lib.ptr(v2), mg_lib.ptr(phi), float(self.p0), sA, sB,
                                             int(bool(self.ghost_fluid_method)), float(self.gfm_clamp),
                                             solver._s()), "mg_build_pressure_b")
        self._keep = (vel, phi)  # alive until the stream has consumed them

    def build_A(self, solver, level):
        """pressure_project.py:45-70."""
        sA, _ = self._scales()
        phi = None
        if level == 0 and self.ghost_fluid_method:
            _, phi = self._inputs(solver)
        check(solver.lib.mg_build_pressure_A(solver.plan, int(level), mg_lib.ptr(phi), sA,
                                             int(bool(self.ghost_fluid_method)), float(self.gfm_clamp),
                                             solver._s()), "mg_build_pressure_A")
        self._keep_A = phi

    def declared_operator(self, solver):
        """The form of the A this Strategy builds: label-uniform, off-diagonal
        -scale_A between FLUID cells on every level (pressure_project.py:56-58).
        The solver then prepares without the detection pass and its host
        synchronization; a device kernel still checks the declaration."""
        sA, _ = self._scales()
        return "uniform", [sA] * solver.n_mg_levels
