"""Drop-in ``MagneticForceStrategy`` (magnetic_force.py:6-38).

The pressure solve of the ferrofluid substep (ferrofluid_simulator.py:99-113):
the ghost-fluid pressure Strategy whose AIR faces carry the magnetic pressure
p0 + (k mu0 / 2) |H|^2 instead of p0, with H interpolated from the MAC field
``H`` at the AIR cell centre (ferrofluid_simulator.py:64-69).  ``build_A`` is
the pressure Strategy's (the reference inherits it).

``H`` is a list of ``dim`` float32 tensors with shapes res + e_k.  The
constant k mu0 / 2 is folded in double, as the reference's Python does.
"""
import mg_lib
from mg_lib import check
from pressure_project import PressureProjectStrategy, _f32


class MagneticForceStrategy(PressureProjectStrategy):
    def __init__(self, dim, velocity, ghost_fluid_method, phi, p0, mu0, k, H, simulator=None, gfm_clamp=1e3):
        super().__init__(dim, velocity, ghost_fluid_method, phi, p0, gfm_clamp)
        self.mu0 = mu0
        self.k = k
        self.H = H
        self.simulator = simulator

    @property
    def coef(self):
        return 1 / 2 * self.k * self.mu0

    def _H(self, solver):
        Hs = [_f32(h, solver.device) for h in self.H]
        for q, h in enumerate(Hs):
            exp = list(solver.res)
            exp[q] += 1
            if tuple(h.shape) != tuple(exp):
                raise ValueError(f"H[{q}] shape {tuple(h.shape)} != {tuple(exp)}")
        return Hs

    def build_b(self, solver):
        """magnetic_force.py:17-38."""
        sA, sB = self._scales()
        vel, _ = self._inputs(solver)
        Hs = self._H(solver)
        v2 = vel[2] if self.dim == 3 else None
        H2 = Hs[2] if self.dim == 3 else None
        check(solver.lib.mg_build_magnetic_b(solver.plan, vel[0].data_ptr(), vel[1].data_ptr(), mg_lib.ptr(v2),
                                             Hs[0].data_ptr(), Hs[1].data_ptr(), mg_lib.ptr(H2), float(self.p0),
                                             sA, sB, float(self.coef), solver._s()), "mg_build_magnetic_b")
        self._keep = (vel, Hs)
