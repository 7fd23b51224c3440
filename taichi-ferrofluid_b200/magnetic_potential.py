"""Magnetic potential Strategy of the 3D ferrofluid substep benchmark.

The reference solves for the magnetic potential psi with
``PotentialFunctionStrategy`` (potential_function.py:6-60) through
``full_reinitialize`` + ``solve`` (ferrofluid_simulator.py:77-87).  The
benchmark's form of that solve, implemented here on the CUDA library:

* permeability mu = 1 + chi, chi given at cell centres (1 inside the fluid);
* face coefficient = harmonic mean of the two cells' mu, over dx^2
  (symmetric positive definite; the reference's A is negative definite);
* right-hand side -div(mu H) for a constant external field H;
* Neumann at the domain boundary, psi pinned to 0 at cell ``pin``
  (the reference pins cell 0, potential_function.py:24, :48);
* coarse levels: the Galerkin operator P^T A P of the reference's transfer
  pair (the reference re-samples chi per level, potential_function.py:54-55).

The reference's own form is ``potential_function.PotentialFunctionStrategy``.

Use it with ``solver.full_reinitialize(strategy)`` as the reference does.
"""
import torch

import mg_lib
from mg_lib import check


class MagneticPotentialStrategy:
    def __init__(self, dim, chi, H_ext=(0.0, 1.0, 0.0), dx=1.0, pin=(1, 1, 1)):
        self.dim = dim
        self.chi = chi
        self.H_ext = tuple(float(h) for h in H_ext) + (0.0,) * (3 - len(H_ext))
        self.dx = float(dx)
        self.pin = tuple(int(p) for p in pin) + (0,) * (3 - len(pin))

    def _chi(self, solver):
        c = torch.as_tensor(self.chi, device=solver.device).to(torch.float32).contiguous()
        if tuple(c.shape) != solver.res:
            raise ValueError(f"chi shape {tuple(c.shape)} != {solver.res}")
        self._keep = c
        return c

    def build_b(self, solver):
        c = self._chi(solver)
        H, p = self.H_ext, self.pin
        check(solver.lib.mg_build_psi_b(solver.plan, c.data_ptr(), H[0], H[1], H[2], self.dx, p[0], p[1], p[2],
                                        solver._s()), "mg_build_psi_b")

    def build_A(self, solver, level):
        if level == 0:
            c = self._chi(solver)
            p = self.pin
            check(solver.lib.mg_build_psi_A(solver.plan, c.data_ptr(), self.dx, p[0], p[1], p[2], solver._s()),
                  "mg_build_psi_A")
        else:
            check(solver.lib.mg_galerkin_coarsen(solver.plan, int(level), solver._s()), "mg_galerkin_coarsen")
