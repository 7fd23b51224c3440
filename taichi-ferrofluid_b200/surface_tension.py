"""Drop-in ``SurfaceTension`` and ``SurfaceTensionStrategy`` (surface_tension.py).

The implicit surface tension step: for each velocity axis d, the normal
n = grad phi / |grad phi| and curvature kappa = div n are computed at the
faces of axis d, then one whole-domain solve

    (1/dt + sigma dt L_delta) u_d = u_d / dt - sigma delta(phi) (kappa n_d
                                    + dt (n^T D2 n + kappa grad u_d . n))

replaces u_d (surface_tension.py:131-153).  delta is the level set's
smoothed Dirac delta of half width eps = 5 dx (level_set.py:22, 32-37).

``simulator`` is any object with the reference simulator's attributes used
here: ``dim``, ``res``, ``dt``, ``dx``, ``real``, ``verbose``, ``velocity``
(list of float32 CUDA tensors, shapes res + e_k), ``level_set`` (with ``phi``,
a float32 tensor of shape res, and ``eps``) and ``poisson_solver`` (an
``MGPCGPoissonSolver``).  ``n`` is held as ``dim`` planes of the cell grid
(``n[k]`` is component k); ``kappa`` has shape res.
"""
import torch

from mg_lib import check
from pressure_project import _f32


def _eps(level_set, dx):
    return float(getattr(level_set, "eps", 5 * dx))


class SurfaceTensionStrategy:
    def __init__(self, simulator, surface_tension):
        self.dim = simulator.dim
        self.res = tuple(simulator.res)
        self.dt = simulator.dt
        self.dx = simulator.dx
        self.real = simulator.real
        self.sigma = surface_tension.sigma
        self.simulator = simulator
        self.surface_tension = surface_tension
        self.d = 0

    def build_b(self, solver):
        """surface_tension.py:23-74."""
        sim, st = self.simulator, self.surface_tension
        u = _f32(sim.velocity[self.d], solver.device)
        phi = _f32(sim.level_set.phi, solver.device)
        check(solver.lib.mg_build_surface_tension_b(solver.plan, int(self.d), u.data_ptr(), phi.data_ptr(),
                                                    st.n.data_ptr(), st.kappa.data_ptr(), float(self.sigma),
                                                    float(self.dt), float(self.dx), _eps(sim.level_set, self.dx),
                                                    solver._s()), "mg_build_surface_tension_b")
        self._keep_b = (u, phi)

    def build_A(self, solver, level):
        """surface_tension.py:76-96."""
        sim = self.simulator
        phi = _f32(sim.level_set.phi, solver.device)
        check(solver.lib.mg_build_surface_tension_A(solver.plan, int(level), int(self.d), phi.data_ptr(),
                                                    float(self.sigma), float(self.dt), float(self.dx),
                                                    _eps(sim.level_set, self.dx), solver._s()),
              "mg_build_surface_tension_A")
        self._keep_A = phi


class SurfaceTension:
    def __init__(self, simulator):
        self.dim = simulator.dim
        self.res = tuple(simulator.res)
        self.dx = simulator.dx
        self.real = simulator.real
        self.sigma = 7.28e-2  # surface tension coefficient (surface_tension.py:105)
        self.simulator = simulator
        self.level_set = simulator.level_set
        self.poisson_solve_iterations = 500
        self.poisson_solver = simulator.poisson_solver
        dev = self.poisson_solver.device
        self.n = torch.zeros((self.dim,) + self.res, dtype=torch.float32, device=dev)  # n = grad phi / |grad phi|
        self.kappa = torch.zeros(self.res, dtype=torch.float32, device=dev)  # mean curvature, div n
        self.strategy = SurfaceTensionStrategy(simulator, self)

    def calc_n(self, d, phi):
        """surface_tension.py:108-121."""
        s = self.poisson_solver
        ph = _f32(phi, s.device)
        check(s.lib.mg_calc_surface_normal(s.plan, int(d), ph.data_ptr(), float(self.dx), self.n.data_ptr(), s._s()),
              "mg_calc_surface_normal")
        self._keep_phi = ph

    def calc_kappa(self, d, phi):
        """surface_tension.py:123-129 (d and phi are unused, as in the reference)."""
        s = self.poisson_solver
        check(s.lib.mg_calc_curvature(s.plan, self.n.data_ptr(), float(self.dx), self.kappa.data_ptr(), s._s()),
              "mg_calc_curvature")

    def solve_surface_tension(self):
        """surface_tension.py:131-153: one solve per velocity axis, x copied into u_d."""
        sim = self.simulator
        for k in range(self.dim):
            self.calc_n(k, self.level_set.phi)
            self.calc_kappa(k, self.level_set.phi)
            self.strategy.d = k
            self.poisson_solver.full_reinitialize(self.strategy)
            self.poisson_solver.solve(self.poisson_solve_iterations, getattr(sim, "verbose", False))
            idx = tuple(slice(0, r) for r in self.res)
            sim.velocity[k][idx].copy_(self.poisson_solver.x)
