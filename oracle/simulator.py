"""ctypes wrapper over ``simulator_oracle.cpp`` (test infrastructure only).

The oracle of the reference's other Strategies and of the pressure update:
``apply_pressure`` (fluid_simulator.py:193-214), ``apply_magnetic_force``
(ferrofluid_simulator.py:115-137), ``MagneticForceStrategy`` (magnetic_force.py),
``PotentialFunctionStrategy`` (potential_function.py),
``PressureProjectWithVolumeControlStrategy`` (volume_control.py) and
``SurfaceTension`` / ``SurfaceTensionStrategy`` (surface_tension.py).  Every
function takes and returns numpy arrays; the f32 inputs are copied, never
modified in place.  Parity against the reference itself is unpinned.
"""
import ctypes

import numpy as np

from .oracle import _load

_c = None


def _lib():
    global _c
    if _c is None:
        lib = _load()
        vp, dd, ff, ii = ctypes.c_void_p, ctypes.c_double, ctypes.c_float, ctypes.c_int
        lib.ors_apply_pressure.argtypes = [ii, vp, vp, vp, vp, vp, ff, ff, ii, ff, vp, ff]
        lib.ors_volume.restype = dd
        lib.ors_volume.argtypes = [ii, vp, vp, dd]
        lib.ors_volume_control.argtypes = [ii, vp, vp, dd, vp, vp, vp]
        lib.ors_build_magnetic_b.argtypes = [ii, vp, vp, vp, vp, ff, ff, ff, ff, vp]
        lib.ors_build_potential_b.argtypes = [ii, vp, vp, vp, vp]
        lib.ors_build_potential_A.argtypes = [ii, vp, ii, vp, dd, vp, vp]
        lib.ors_calc_n.argtypes = [ii, vp, ii, vp, ff, vp]
        lib.ors_calc_kappa.argtypes = [ii, vp, vp, ff, vp]
        lib.ors_build_st_b.argtypes = [ii, vp, ii, vp, vp, vp, vp, dd, dd, dd, dd, vp]
        lib.ors_build_st_A.argtypes = [ii, vp, ii, ii, vp, dd, dd, dd, dd, vp, vp]
        lib.ors_update_chi.argtypes = [ii, vp, vp, dd, dd, vp]
        lib.ors_update_H.argtypes = [ii, vp, ii, vp, vp, ff, vp]
        lib.ors_level_set_shape.argtypes = [ii, vp, vp, ff, ii, vp, vp, ii]
        lib.ors_apply_markers.argtypes = [ii, vp, vp, vp, ii]
        lib.ors_init_boundary.argtypes = [ii, vp, vp]
        lib.ors_redistance.argtypes = [ii, vp, vp, dd, ii, vp, vp]
        lib.ors_markers_distance.argtypes = [ii, vp, vp, ii, ff, ii, vp, vp]
        lib.ors_target_minus.argtypes = [ii, vp, vp, ff, vp, vp]
        lib.ors_fs_propagate.argtypes = [ii, vp, vp, vp, vp, dd, ii]
        lib.ors_ls_smooth.argtypes = [ii, vp, vp, vp]
        lib.ors_advect.argtypes = [ii, vp, vp, ii, vp, vp, ff, ff]
        lib.ors_extrapolate.argtypes = [ii, vp, ii, vp, vp, ii, vp]
        lib.ors_enforce_boundary.argtypes = [ii, vp, vp, vp]
        lib.ors_add_gravity.argtypes = [ii, vp, vp, vp, ff]
        _c = lib
    return _c


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32).copy()


def _res(shape):
    r = list(shape) + [1] * (3 - len(shape))
    return (ctypes.c_int * 3)(*r)


def _ptrs(arrs):
    return (ctypes.c_void_p * 3)(*([a.ctypes.data for a in arrs] + [None] * (3 - len(arrs))))


def apply_pressure(velocity, pressure, cell_type, phi, scale, p0, ghost_fluid_method=True, gfm_clamp=1e3):
    """FluidSimulator.apply_pressure; returns the updated face velocities."""
    ct = np.ascontiguousarray(cell_type, dtype=np.int32)
    u = [_f32(v) for v in velocity]
    p, ph = _f32(pressure), _f32(phi if phi is not None else np.zeros(ct.shape))
    _lib().ors_apply_pressure(ct.ndim, _res(ct.shape), _ptrs(u), p.ctypes.data, ct.ctypes.data, ph.ctypes.data,
                              float(scale), float(p0), int(bool(ghost_fluid_method)), float(gfm_clamp), None,
                              0.0)
    return u


def apply_magnetic_force(velocity, pressure, cell_type, H, scale, p0, coef):
    """FerrofluidSimulator.apply_magnetic_force; H is the MAC field (one array per axis)."""
    ct = np.ascontiguousarray(cell_type, dtype=np.int32)
    u = [_f32(v) for v in velocity]
    Hs = [_f32(h) for h in H]
    p = _f32(pressure)
    _lib().ors_apply_pressure(ct.ndim, _res(ct.shape), _ptrs(u), p.ctypes.data, ct.ctypes.data, None,
                              float(scale), float(p0), 0, 0.0, _ptrs(Hs), float(coef))
    return u


def volume(phi, eps):
    """PressureProjectWithVolumeControlStrategy.calc_volume (FP64 sum)."""
    ph = _f32(phi)
    return float(_lib().ors_volume(ph.ndim, _res(ph.shape), ph.ctypes.data, float(eps)))


def volume_control(phi, eps, grid_type, b, state):
    """One controller step plus add_c; returns (b, state) updated copies."""
    ph, bb = _f32(phi), _f32(b)
    t = np.ascontiguousarray(grid_type, dtype=np.int8)
    st = np.ascontiguousarray(state, dtype=np.float64).copy()
    _lib().ors_volume_control(ph.ndim, _res(ph.shape), ph.ctypes.data, float(eps), t.ctypes.data,
                              bb.ctypes.data, st.ctypes.data)
    return bb, st


def build_magnetic_b(grid_type, velocity, H, p0, scale_A, scale_b, coef):
    """MagneticForceStrategy.build_b_kernel on a zeroed b."""
    t = np.ascontiguousarray(grid_type, dtype=np.int8)
    v = [_f32(a) for a in velocity]
    Hs = [_f32(h) for h in H]
    b = np.zeros(t.shape, np.float32)
    _lib().ors_build_magnetic_b(t.ndim, _res(t.shape), t.ctypes.data, _ptrs(v), _ptrs(Hs), float(p0),
                                float(scale_A), float(scale_b), float(coef), b.ctypes.data)
    return b


def build_potential_b(chi, H_ext):
    c = _f32(chi)
    Hs = [_f32(h) for h in H_ext]
    b = np.zeros(c.shape, np.float32)
    _lib().ors_build_potential_b(c.ndim, _res(c.shape), c.ctypes.data, _ptrs(Hs), b.ctypes.data)
    return b


def build_potential_A(chi, level, dx):
    """One level; returns (Adiag, Ax) with Ax of shape (dim, *level_shape)."""
    c = _f32(chi)
    shp = tuple(v >> level for v in c.shape)
    Ad = np.zeros(shp, np.float32)
    Ax = np.zeros((c.ndim,) + shp, np.float32)
    _lib().ors_build_potential_A(c.ndim, _res(c.shape), int(level), c.ctypes.data, float(dx), Ad.ctypes.data,
                                 Ax.ctypes.data)
    return Ad, Ax


def calc_n(phi, d, dx):
    ph = _f32(phi)
    n = np.zeros((ph.ndim,) + ph.shape, np.float32)
    _lib().ors_calc_n(ph.ndim, _res(ph.shape), int(d), ph.ctypes.data, float(dx), n.ctypes.data)
    return n


def calc_kappa(n, dx):
    nn = _f32(n)
    shp = nn.shape[1:]
    k = np.zeros(shp, np.float32)
    _lib().ors_calc_kappa(len(shp), _res(shp), nn.ctypes.data, float(dx), k.ctypes.data)
    return k


def build_st_b(d, u_d, phi, n, kappa, sigma, dt, dx, eps):
    ph, u, nn, ka = _f32(phi), _f32(u_d), _f32(n), _f32(kappa)
    b = np.zeros(ph.shape, np.float32)
    _lib().ors_build_st_b(ph.ndim, _res(ph.shape), int(d), u.ctypes.data, ph.ctypes.data, nn.ctypes.data,
                          ka.ctypes.data, float(sigma), float(dt), float(dx), float(eps), b.ctypes.data)
    return b


def build_st_A(phi, level, d, sigma, dt, dx, eps):
    ph = _f32(phi)
    shp = tuple(v >> level for v in ph.shape)
    Ad = np.zeros(shp, np.float32)
    Ax = np.zeros((ph.ndim,) + shp, np.float32)
    _lib().ors_build_st_A(ph.ndim, _res(ph.shape), int(level), int(d), ph.ctypes.data, float(sigma), float(dt),
                          float(dx), float(eps), Ad.ctypes.data, Ax.ctypes.data)
    return Ad, Ax


def update_chi(phi, k, eps):
    """FerrofluidSimulator.update_magnetic_susceptibility."""
    ph = _f32(phi)
    chi = np.zeros(ph.shape, np.float32)
    _lib().ors_update_chi(ph.ndim, _res(ph.shape), ph.ctypes.data, float(k), float(eps), chi.ctypes.data)
    return chi


def update_H(psi, H_ext, dx):
    """FerrofluidSimulator.update_magnetic_field; returns one face array per axis."""
    ps = _f32(psi)
    out = []
    for k, he in enumerate(H_ext):
        h = _f32(he)
        H = np.zeros(h.shape, np.float32)
        _lib().ors_update_H(ps.ndim, _res(ps.shape), k, ps.ctypes.data, h.ctypes.data, float(dx), H.ctypes.data)
        out.append(H)
    return out


def level_set_shape(shape, dx, sphere, a, b, phi=None):
    """LevelSet.initialize_with_aabb (sphere False: box [a, b]) or
    initialize_with_sphere (centre a, radius b); with phi: union (min)."""
    out = np.zeros(shape, np.float32) if phi is None else _f32(phi)
    A = (ctypes.c_float * 3)(*(list(a) + [0.0] * (3 - len(a))))
    bb = [b] if sphere else list(b)
    B = (ctypes.c_float * 3)(*(bb + [0.0] * (3 - len(bb))))
    _lib().ors_level_set_shape(len(shape), _res(shape), out.ctypes.data, float(dx), int(bool(sphere)), A, B,
                               int(phi is not None))
    return out


def apply_markers(cell_type, phi, strict=False):
    ct = np.ascontiguousarray(cell_type, dtype=np.int32).copy()
    ph = _f32(phi)
    _lib().ors_apply_markers(ct.ndim, _res(ct.shape), ct.ctypes.data, ph.ctypes.data, int(bool(strict)))
    return ct


def init_boundary(cell_type):
    ct = np.ascontiguousarray(cell_type, dtype=np.int32).copy()
    _lib().ors_init_boundary(ct.ndim, _res(ct.shape), ct.ctypes.data)
    return ct


def redistance(phi, dx, repeat_times=2):
    """FastSweepingLevelSet.redistance, lines swept one after another;
    returns (phi, valid)."""
    ph = _f32(phi)
    valid = np.zeros(ph.shape, np.int32)
    _lib().ors_redistance(ph.ndim, _res(ph.shape), ph.ctypes.data, float(dx), int(repeat_times), None,
                          valid.ctypes.data)
    return ph, valid


def markers_distance(shape, markers, dx, repeat_times=2):
    """FastSweepingLevelSet.build_from_markers' first part: distance_to_markers
    and markers_propagate from phi = 1e20, valid = -1; returns (phi, valid)."""
    mk = _f32(markers).reshape(-1, len(shape))
    phi = np.zeros(shape, np.float32)
    valid = np.zeros(shape, np.int32)
    _lib().ors_markers_distance(len(shape), _res(shape), mk.ctypes.data, int(mk.shape[0]), float(np.float32(dx)),
                                int(repeat_times), phi.ctypes.data, valid.ctypes.data)
    return phi, valid


def target_minus(phi, dx):
    """LevelSet.target_minus after valid.fill(-1); returns (phi, phi_temp, valid)."""
    ph = _f32(phi)
    temp = np.zeros(ph.shape, np.float32)
    valid = np.zeros(ph.shape, np.int32)
    _lib().ors_target_minus(ph.ndim, _res(ph.shape), ph.ctypes.data, float(np.float32(0.99 * dx)), temp.ctypes.data,
                            valid.ctypes.data)
    return ph, temp, valid


def fs_propagate(phi, phi_temp, valid, dx, repeat_times=2):
    """FastSweepingLevelSet.propagate (lines one after another); returns phi_temp."""
    ph = _f32(phi)
    t = _f32(phi_temp)
    v = np.ascontiguousarray(valid, dtype=np.int32)
    _lib().ors_fs_propagate(ph.ndim, _res(ph.shape), ph.ctypes.data, t.ctypes.data, v.ctypes.data, float(dx),
                            int(repeat_times))
    return t


def ls_smooth(src):
    """LevelSet.smoothing: returns min(mean of the axis neighbours of src, src)."""
    a = _f32(src)
    out = np.zeros(a.shape, np.float32)
    _lib().ors_ls_smooth(a.ndim, _res(a.shape), out.ctypes.data, a.ctypes.data)
    return out


def build_from_markers(shape, markers, dx, repeat_times=2):
    """FastSweepingLevelSet.build_from_markers (level_set.py:381-392); returns phi."""
    phi, _ = markers_distance(shape, markers, dx, repeat_times)
    phi, temp, valid = target_minus(phi, dx)
    temp = fs_propagate(phi, temp, valid, dx, repeat_times)
    phi = ls_smooth(temp)
    temp = ls_smooth(phi)
    return ls_smooth(temp)


def advect(velocity, src, field, dx, dt):
    """FluidSimulator.advect of one field (field -1: cell field, k: faces of axis k)."""
    u = [_f32(v) for v in velocity]
    sr = _f32(src)
    shape = tuple(s - (k == field) for k, s in enumerate(sr.shape)) if field >= 0 else sr.shape
    out = np.zeros(sr.shape, np.float32)
    _lib().ors_advect(len(shape), _res(shape), _ptrs(u), int(field), sr.ctypes.data, out.ctypes.data, float(dx),
                      float(dt))
    return out


def extrapolate(u_k, k, cell_type, iterations=10):
    """FluidSimulator.extrap_velocity for axis k; returns (u_k, valid)."""
    ct = np.ascontiguousarray(cell_type, dtype=np.int32)
    u = _f32(u_k)
    valid = np.zeros(u.shape, np.int32)
    _lib().ors_extrapolate(ct.ndim, _res(ct.shape), int(k), u.ctypes.data, ct.ctypes.data, int(iterations),
                           valid.ctypes.data)
    return u, valid


def enforce_boundary(velocity, cell_type):
    ct = np.ascontiguousarray(cell_type, dtype=np.int32)
    u = [_f32(v) for v in velocity]
    _lib().ors_enforce_boundary(ct.ndim, _res(ct.shape), _ptrs(u), ct.ctypes.data)
    return u


def add_gravity(velocity, gravity, dt):
    u = [_f32(v) for v in velocity]
    shape = tuple(s - (k == 0) for k, s in enumerate(u[0].shape))
    g = (ctypes.c_double * 3)(*(list(gravity) + [0.0] * (3 - len(gravity))))
    _lib().ors_add_gravity(len(shape), _res(shape), _ptrs(u), g, float(dt))
    return u
