"""Drop-in ``PotentialFunctionStrategy`` (potential_function.py:6-60).

The reference's own form of the magnetic potential solve of the ferrofluid
substep (ferrofluid_simulator.py:77-87), used with ``full_reinitialize``:

* whole domain, every label FLUID;
* face coefficient (1 + chi)/dx with chi sampled at the face from the cell
  field ``chi`` (utils.sample), A negative definite;
* the origin cell pinned: Adiag = 1/dx, b = 0 (potential_function.py:24, :48);
* every level is rebuilt from the fine chi at (I + e_k/2) 2^level, and the
  in-domain test uses the fine ``res`` on every level (potential_function.py:
  17, 53), so the last cell of a coarse level couples to a cell beyond the
  level's edge; that neighbour reads as 0 in the V-cycle.

``H_ext`` is a list of ``dim`` float32 tensors with shapes res + e_k (MAC
faces), ``chi`` a float32 tensor of shape res.  For the symmetric positive
definite form with Galerkin coarse levels see ``magnetic_potential``.
"""
from mg_lib import check
from pressure_project import _f32


class PotentialFunctionStrategy:
    def __init__(self, dim, res, dx, H_ext, chi):
        self.dim = dim
        self.res = tuple(res)
        self.dx = dx
        self.H_ext = H_ext
        self.chi = chi

    def _chi(self, solver):
        c = _f32(self.chi, solver.device)
        if tuple(c.shape) != solver.res:
            raise ValueError(f"chi shape {tuple(c.shape)} != {solver.res}")
        return c

    def build_b(self, solver):
        """potential_function.py:19-39."""
        c = self._chi(solver)
        He = [_f32(h, solver.device) for h in self.H_ext]
        for k, h in enumerate(He):
            exp = list(solver.res)
            exp[k] += 1
            if tuple(h.shape) != tuple(exp):
                raise ValueError(f"H_ext[{k}] shape {tuple(h.shape)} != {tuple(exp)}")
        h2 = He[2].data_ptr() if self.dim == 3 else None
        check(solver.lib.mg_build_potential_b(solver.plan, c.data_ptr(), He[0].data_ptr(), He[1].data_ptr(), h2,
                                              solver._s()), "mg_build_potential_b")
        self._keep_b = (c, He)

    def build_A(self, solver, level):
        """potential_function.py:41-60."""
        c = self._chi(solver)
        check(solver.lib.mg_build_potential_A(solver.plan, int(level), c.data_ptr(), float(self.dx), solver._s()),
              "mg_build_potential_A")
        self._keep_A = c
