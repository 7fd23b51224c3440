"""The simulator steps around the Poisson solves, on the device.

Free functions with the argument meaning of the reference's simulator
methods (the reference binds them to its ``FluidSimulator`` /
``FerrofluidSimulator`` objects):

* ``apply_pressure`` - FluidSimulator.apply_pressure (fluid_simulator.py:193-214),
  the ghost-fluid pressure-gradient update of the MAC velocity;
* ``apply_magnetic_force`` - FerrofluidSimulator.apply_magnetic_force
  (ferrofluid_simulator.py:115-137), the same update with the magnetic
  pressure on AIR faces;
* ``update_magnetic_susceptibility`` (ferrofluid_simulator.py:71-75) and
  ``update_magnetic_field`` (ferrofluid_simulator.py:89-97), the fields
  before and after the potential solve.

Every function takes the ``MGPCGPoissonSolver`` whose geometry (and, by
default, whose solution ``x`` and level-0 labels) it uses, so the pressure
goes from the solve to the velocity update without leaving the device.
Velocity and H lists are float32 CUDA tensors with shapes res + e_k and are
updated in place.
"""
import numpy as np
import torch

import mg_lib
from mg_lib import check
from pressure_project import _f32


def _faces(solver, fields, what):
    out = []
    for k in range(solver.dim):
        f = fields[k]
        exp = list(solver.res)
        exp[k] += 1
        if tuple(f.shape) != tuple(exp) or f.dtype != torch.float32 or not f.is_contiguous() \
                or f.device != solver.device:
            raise ValueError(f"{what}[{k}] must be a contiguous float32 tensor of shape {tuple(exp)} "
                             f"on {solver.device}")
        out.append(f)
    return out


def _labels(solver, cell_type):
    if cell_type is None:
        return None
    ct = torch.as_tensor(cell_type, device=solver.device).to(torch.int32).contiguous()
    if tuple(ct.shape) != solver.res:
        raise ValueError(f"cell_type shape {tuple(ct.shape)} != {solver.res}")
    return ct


def pressure_scale(dt, rho, dx):
    """scale = dt / (rho dx): dt is an f32 kernel argument, rho dx folded in double."""
    return float(np.float32(dt) / np.float32(rho * dx))


def apply_pressure(solver, velocity, dt, rho, dx, p0, phi=None, ghost_fluid_method=True, cell_type=None,
                   pressure=None, gfm_clamp=1e3):
    """fluid_simulator.py:193-214.  pressure None: the solver's x; cell_type
    None: the solver's level-0 labels (the simulator's cell_type after
    reinitialize)."""
    u = _faces(solver, velocity, "velocity")
    ct = _labels(solver, cell_type)
    pr = _f32(pressure, solver.device) if pressure is not None else None
    ph = _f32(phi, solver.device) if ghost_fluid_method else None
    if ghost_fluid_method and ph is None:
        raise ValueError("the ghost fluid method needs phi")
    u2 = u[2] if solver.dim == 3 else None
    check(solver.lib.mg_apply_pressure(solver.plan, u[0].data_ptr(), u[1].data_ptr(), mg_lib.ptr(u2),
                                       mg_lib.ptr(pr), mg_lib.ptr(ct), mg_lib.ptr(ph), pressure_scale(dt, rho, dx),
                                       float(p0), int(bool(ghost_fluid_method)), float(gfm_clamp), solver._s()),
          "mg_apply_pressure")
    solver._keep_apply = (ct, pr, ph)


def apply_magnetic_force(solver, velocity, H, dt, rho, dx, p0, k, mu0, cell_type=None, pressure=None):
    """ferrofluid_simulator.py:115-137."""
    u = _faces(solver, velocity, "velocity")
    Hs = [_f32(h, solver.device) for h in H]
    ct = _labels(solver, cell_type)
    pr = _f32(pressure, solver.device) if pressure is not None else None
    u2 = u[2] if solver.dim == 3 else None
    H2 = Hs[2] if solver.dim == 3 else None
    check(solver.lib.mg_apply_magnetic_force(solver.plan, u[0].data_ptr(), u[1].data_ptr(), mg_lib.ptr(u2),
                                             mg_lib.ptr(pr), mg_lib.ptr(ct), Hs[0].data_ptr(), Hs[1].data_ptr(),
                                             mg_lib.ptr(H2), pressure_scale(dt, rho, dx), float(p0),
                                             float(1 / 2 * k * mu0), solver._s()), "mg_apply_magnetic_force")
    solver._keep_apply = (ct, pr, Hs)


def update_magnetic_susceptibility(solver, phi, k, eps, chi):
    """ferrofluid_simulator.py:71-75: chi = k (1 - theta(phi)), in place."""
    ph = _f32(phi, solver.device)
    if tuple(chi.shape) != solver.res or not chi.is_contiguous():
        raise ValueError("chi must be a contiguous float32 tensor of shape res")
    check(solver.lib.mg_update_susceptibility(solver.plan, ph.data_ptr(), float(k), float(eps), chi.data_ptr(),
                                              solver._s()), "mg_update_susceptibility")
    solver._keep_chi = ph


def update_magnetic_field(solver, H_ext, dx, H, psi=None):
    """ferrofluid_simulator.py:89-97: H = H_ext - grad psi (psi None: the solver's x)."""
    He = [_f32(h, solver.device) for h in H_ext]
    Hs = _faces(solver, H, "H")
    ps = _f32(psi, solver.device) if psi is not None else None
    h2 = He[2] if solver.dim == 3 else None
    o2 = Hs[2] if solver.dim == 3 else None
    check(solver.lib.mg_update_magnetic_field(solver.plan, mg_lib.ptr(ps), He[0].data_ptr(), He[1].data_ptr(),
                                              mg_lib.ptr(h2), float(dx), Hs[0].data_ptr(), Hs[1].data_ptr(),
                                              mg_lib.ptr(o2), solver._s()), "mg_update_magnetic_field")
    solver._keep_H = (He, ps)


def _grid(cell_type):
    dim = cell_type.dim()
    return dim, (mg_lib.ctypes.c_int32 * 3)(*(list(cell_type.shape) + [1] * (3 - dim)))


def _i32(t, what):
    if t.dtype != torch.int32 or not t.is_contiguous() or not t.is_cuda:
        raise ValueError(f"{what} must be a contiguous int32 CUDA tensor (the simulator's labels)")
    return t


def apply_markers(cell_type, phi, strict=False):
    """fluid_simulator.py:151-159, in place: non-SOLID cells AIR, then FLUID
    where phi <= 0 (strict: phi < 0, the benchmark scenes' rule)."""
    ct = _i32(cell_type, "cell_type")
    ph = _f32(phi, ct.device)
    if ph.shape != ct.shape:
        raise ValueError("phi and cell_type shapes differ")
    dim, res = _grid(ct)
    lib = mg_lib.load()
    check(lib.mg_apply_markers(dim, res, ct.data_ptr(), ph.data_ptr(), int(bool(strict)),
                               mg_lib.stream_ptr(ct.device)), "mg_apply_markers")


def init_boundary(cell_type):
    """fluid_simulator.py:337-341, in place: SOLID on the outermost ring."""
    ct = _i32(cell_type, "cell_type")
    dim, res = _grid(ct)
    lib = mg_lib.load()
    check(lib.mg_init_boundary(dim, res, ct.data_ptr(), mg_lib.stream_ptr(ct.device)), "mg_init_boundary")


# ---- the velocity steps around the projection ----------------------------------
def _vel_grid(velocity):
    dim = len(velocity)
    shape = [int(s) - (k == 0) for k, s in enumerate(velocity[0].shape)]
    return dim, shape, (mg_lib.ctypes.c_int32 * 3)(*(shape + [1] * (3 - dim)))


def _check_faces(fields, shape, what):
    for k, f in enumerate(fields):
        exp = list(shape)
        exp[k] += 1
        if tuple(f.shape) != tuple(exp) or f.dtype != torch.float32 or not f.is_contiguous() or not f.is_cuda:
            raise ValueError(f"{what}[{k}] must be a contiguous float32 CUDA tensor of shape {tuple(exp)}")


def advect_quantity(velocity, velocity_backup, dx, dt, phi=None, phi_temp=None):
    """fluid_simulator.py:223-231: velocity_backup[k] (and phi_temp, when phi
    is given) = the semi-Lagrangian (midpoint) advection of velocity[k] (phi)
    through velocity."""
    dim, shape, res = _vel_grid(velocity)
    _check_faces(velocity, shape, "velocity")
    _check_faces(velocity_backup, shape, "velocity_backup")
    if (phi is None) != (phi_temp is None):
        raise ValueError("phi and phi_temp go together")
    u = [velocity[k].data_ptr() for k in range(dim)] + [None] * (3 - dim)
    o = [velocity_backup[k].data_ptr() for k in range(dim)] + [None] * (3 - dim)
    lib = mg_lib.load()
    check(lib.mg_advect_quantity(dim, res, u[0], u[1], u[2], mg_lib.ptr(phi), mg_lib.ptr(phi_temp), o[0], o[1], o[2],
                                 float(dx), float(dt), mg_lib.stream_ptr(velocity[0].device)), "mg_advect_quantity")


def update_quantity(velocity, velocity_backup, phi=None, phi_temp=None):
    """fluid_simulator.py:233-237: copy the advected fields back."""
    if phi is not None:
        phi.copy_(phi_temp)
    for v, b in zip(velocity, velocity_backup):
        v.copy_(b)


def extrap_velocity(velocity, cell_type, iterations=10):
    """fluid_simulator.py:268-272: per axis, faces beside a FLUID cell are
    valid and `iterations` rounds extend the velocity into the invalid faces
    (the mean of the valid faces of the 3^d box)."""
    dim, shape, res = _vel_grid(velocity)
    _check_faces(velocity, shape, "velocity")
    ct = _i32(cell_type, "cell_type")
    lib = mg_lib.load()
    st = mg_lib.stream_ptr(velocity[0].device)
    for k in range(dim):
        u = velocity[k]
        tmp = torch.empty_like(u)
        valid = torch.empty(u.shape, dtype=torch.int32, device=u.device)
        valid_tmp = torch.empty_like(valid)
        check(lib.mg_extrapolate_velocity(dim, res, k, u.data_ptr(), tmp.data_ptr(), valid.data_ptr(),
                                          valid_tmp.data_ptr(), ct.data_ptr(), int(iterations), st),
              "mg_extrapolate_velocity")


def enforce_boundary(velocity, cell_type):
    """fluid_simulator.py:168-174: zero velocity on the faces of SOLID cells."""
    dim, shape, res = _vel_grid(velocity)
    _check_faces(velocity, shape, "velocity")
    ct = _i32(cell_type, "cell_type")
    u = [velocity[k].data_ptr() for k in range(dim)] + [None] * (3 - dim)
    lib = mg_lib.load()
    check(lib.mg_enforce_boundary(dim, res, u[0], u[1], u[2], ct.data_ptr(), mg_lib.stream_ptr(ct.device)),
          "mg_enforce_boundary")


def add_gravity(velocity, gravity, dt):
    """fluid_simulator.py:160-166: velocity[k] += gravity[k] dt (nonzero k)."""
    dim, shape, res = _vel_grid(velocity)
    _check_faces(velocity, shape, "velocity")
    g = [float(v) for v in gravity] + [0.0] * (3 - len(gravity))
    u = [velocity[k].data_ptr() for k in range(dim)] + [None] * (3 - dim)
    lib = mg_lib.load()
    check(lib.mg_add_gravity(dim, res, u[0], u[1], u[2], g[0], g[1], g[2], float(dt),
                             mg_lib.stream_ptr(velocity[0].device)), "mg_add_gravity")
