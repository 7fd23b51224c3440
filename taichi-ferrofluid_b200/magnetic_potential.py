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
* coarse levels: half the Galerkin operator, A_l = P^T A_(l-1) P / 2, for the
  reference's transfer pair (piecewise-constant prolongation, child-sum
  restriction).  Plain Galerkin under-corrects with piecewise-constant
  prolongation; halving each level over-corrects by 2, which cuts the solve at
  128^3 from 38 to 8 PCG iterations.  ``coarse="rediscretise"`` builds each
  coarse level instead as the reference's potential Strategy does
  (potential_function.py:39-55): chi re-sampled per level (the mean of the
  children), spacing dx * 2^l.

The reference's own form is ``potential_function.PotentialFunctionStrategy``.

Use it with ``solver.full_reinitialize(strategy)`` as the reference does.
"""
import torch

import mg_lib
from mg_lib import check


class MagneticPotentialStrategy:
    coarse_scale = 0.5  # A_l = coarse_scale * P^T A_(l-1) P (a power of two)

    def __init__(self, dim, chi, H_ext=(0.0, 1.0, 0.0), dx=1.0, pin=(1, 1, 1), coarse="galerkin"):
        """``coarse``: "galerkin" (half the Galerkin operator, the default) or
        "rediscretise" (each coarse level built like level 0 from the mean of
        its children's chi at spacing dx * 2^l, as the reference's potential
        Strategy rebuilds its coarse levels, potential_function.py:39-55)."""
        if coarse not in ("galerkin", "rediscretise"):
            raise ValueError("coarse must be 'galerkin' or 'rediscretise'")
        self.dim = dim
        self.chi = chi
        self.H_ext = tuple(float(h) for h in H_ext) + (0.0,) * (3 - len(H_ext))
        self.dx = float(dx)
        self.pin = tuple(int(p) for p in pin) + (0,) * (3 - len(pin))
        self.coarse = coarse
        self._chi_levels = {}

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
        elif self.coarse == "galerkin":
            check(solver.lib.mg_galerkin_coarsen(solver.plan, int(level), float(self.coarse_scale), solver._s()),
                  "mg_galerkin_coarsen")
        else:
            fine = self._chi(solver) if level == 1 else self._chi_levels[level - 1]
            shp = solver.shape(level)
            out = self._chi_levels.get(level)
            if out is None or tuple(out.shape) != shp:
                out = torch.empty(shp, dtype=torch.float32, device=solver.device)
                self._chi_levels[level] = out
            p = self.pin
            check(solver.lib.mg_build_psi_A_level(solver.plan, int(level), fine.data_ptr(), out.data_ptr(), self.dx,
                                                  p[0], p[1], p[2], solver._s()), "mg_build_psi_A_level")

    def declared_operator(self, solver):
        """The form of the A this Strategy builds with full_reinitialize:
        every cell FLUID with stored couplings and a positive diagonal, on
        every level.  The solver then prepares without the detection pass and
        its host synchronization; a device kernel still checks it."""
        return "whole", None
