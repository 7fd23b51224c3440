// The step before the solve: level-set initialisation from shapes and the
// cell labels derived from it (the simulators' label production).  f32 with
// explicit round-to-nearest intrinsics in the reference's operation order.
#pragma once
#include "mg_common.cuh"

namespace mg {

// Cell-centre position (I + 0.5) dx of axis k (level_set.py:59, :64).
__device__ __forceinline__ float centre(int c, float dx) { return __fmul_rn(__fadd_rn((float)c, 0.5f), dx); }

// LevelSet.distance_of_aabb (level_set.py:40-54) at the centre of cell c:
// inside the open box the largest (negative) per-axis distance to a face,
// outside the distance to the closest point of the box.
__device__ __forceinline__ float distance_of_aabb(const int c[3], int dim, float dx, const float x0[3],
                                                  const float x1[3]) {
  float x[3];
  bool inside = true;
  for (int k = 0; k < dim; ++k) {
    x[k] = centre(c[k], dx);
    inside = inside && x[k] > x0[k] && x[k] < x1[k];
  }
  if (inside) {
    float m = fmaxf(__fsub_rn(x0[0], x[0]), __fsub_rn(x[0], x1[0]));
    for (int k = 1; k < dim; ++k) m = fmaxf(m, fmaxf(__fsub_rn(x0[k], x[k]), __fsub_rn(x[k], x1[k])));
    return m;
  }
  float s = 0.0f;
  for (int k = 0; k < dim; ++k) {
    const float p = x[k] < x0[k] ? x0[k] : (x[k] > x1[k] ? x1[k] : x[k]);
    const float d = __fsub_rn(x[k], p);
    s = k == 0 ? __fmul_rn(d, d) : __fadd_rn(s, __fmul_rn(d, d));
  }
  return __fsqrt_rn(s);
}

// LevelSet.initialize_with_aabb (level_set.py:56-59) and initialize_with_sphere
// (level_set.py:61-64): phi = the shape's signed distance at cell centres.
// combine != 0 keeps min(phi, distance) instead (the union of several shapes).
__global__ void k_ls_shape(Geom g, float* __restrict__ phi, float dx, int sphere, float a0, float a1, float a2,
                           float b0, float b1, float b2, int combine) {
  const float x0[3] = {a0, a1, a2}, x1[3] = {b0, b1, b2};
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < g.count;
       i += (long long)gridDim.x * blockDim.x) {
    int c[3];
    g.coords(i, c);
    float v;
    if (sphere) {  // centre x0, radius b0
      float s = 0.0f;
      for (int k = 0; k < g.dim; ++k) {
        const float d = __fsub_rn(centre(c[k], dx), x0[k]);
        s = k == 0 ? __fmul_rn(d, d) : __fadd_rn(s, __fmul_rn(d, d));
      }
      v = __fsub_rn(__fsqrt_rn(s), b0);
    } else {
      v = distance_of_aabb(c, g.dim, dx, x0, x1);
    }
    phi[i] = combine ? fminf(phi[i], v) : v;
  }
}

// FluidSimulator.apply_markers (fluid_simulator.py:151-159): every non-SOLID
// cell becomes AIR, then FLUID where phi <= 0 (strict != 0: phi < 0, the
// benchmark scenes' rule).
__global__ void k_apply_markers(Geom g, int32_t* __restrict__ ct, const float* __restrict__ phi, int strict) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < g.count;
       i += (long long)gridDim.x * blockDim.x) {
    if (ct[i] == SOLID) continue;
    const float p = phi[i];
    ct[i] = (strict ? p < 0.0f : p <= 0.0f) ? FLUID : AIR;
  }
}

// FluidSimulator.init_boundary (fluid_simulator.py:337-341): SOLID on the
// outermost ring of cells.
__global__ void k_init_boundary(Geom g, int32_t* __restrict__ ct) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < g.count;
       i += (long long)gridDim.x * blockDim.x) {
    int c[3];
    g.coords(i, c);
    bool edge = false;
    for (int k = 0; k < g.dim; ++k) edge = edge || c[k] == 0 || c[k] + 1 == g.n[k];
    if (edge) ct[i] = SOLID;
  }
}

// ---------------------------------------------------------------------------
// FastSweepingLevelSet.redistance (level_set.py:260-334)
// ---------------------------------------------------------------------------

// GLSL sign (taichi_glsl's ts.sign): -1, 0 or +1.
__device__ __forceinline__ float gsign(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }

// valid.fill(-1) and LevelSet.target_surface (level_set.py:66-86): cells with
// a neighbour of the other sign get phi_temp = the signed distance to the
// linearly interpolated crossing nearest to them (valid 0); the others 1e20.
__global__ void k_target_surface(Geom g, const float* __restrict__ phi, float* __restrict__ phi_temp,
                                 int32_t* __restrict__ valid, float dx) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < g.count;
       i += (long long)gridDim.x * blockDim.x) {
    int c[3];
    g.coords(i, c);
    const float p = phi[i], sp = gsign(p);
    bool change = false;
    float est = 1e20f;
    for (int k = 0; k < g.dim; ++k)
      for (int s = -1; s <= 1; s += 2) {
        const int v = c[k] + s;
        if (v < 0 || v >= g.n[k]) continue;
        const float q = phi[i + s * g.stride(k)];
        if (sp != gsign(q)) {
          const float theta = __fdiv_rn(p, __fsub_rn(p, q));
          const float est0 = __fmul_rn(__fmul_rn(sp, theta), dx);
          est = fabsf(est0) < fabsf(est) ? est0 : est;
          change = true;
        }
      }
    phi_temp[i] = change ? est : 1e20f;
    valid[i] = change ? 0 : -1;
  }
}

// LevelSet.update_from_neighbor (level_set.py:88-112): the upwind Eikonal
// update of cell i from the smaller |phi_temp| neighbour per axis, sorted;
// dx1 = dx, two_dx2 = 2 dx^2, dx2 = dx^2, third = 1/3 folded on the host.
__device__ __forceinline__ float eikonal(const Geom& g, const float* t, long long i, const int c[3], float dx1,
                                         float two_dx2, float dx2, float third) {
  float nb[3];
  for (int k = 0; k < g.dim; ++k) {
    const long long st = g.stride(k);
    const float up = c[k] + 1 < g.n[k] ? fabsf(t[i + st]) : 0.0f;
    if (c[k] == 0 || (c[k] < g.n[k] - 1 && up < fabsf(t[i - st]))) nb[k] = fabsf(t[i + st]);
    else nb[k] = fabsf(t[i - st]);
  }
  for (int a = 0; a < g.dim - 1; ++a)  // the reference's bubble sort
    for (int b = 0; b < g.dim - 1 - a; ++b)
      if (nb[b] > nb[b + 1]) {
        const float tmp = nb[b];
        nb[b] = nb[b + 1];
        nb[b + 1] = tmp;
      }
  float d = __fadd_rn(nb[0], dx1);
  if (d > nb[1]) {
    const float e = __fsub_rn(nb[1], nb[0]);
    d = __fmul_rn(0.5f, __fadd_rn(__fadd_rn(nb[0], nb[1]), __fsqrt_rn(__fsub_rn(two_dx2, __fmul_rn(e, e)))));
    if (g.dim == 3 && d > nb[2]) {
      const float s = __fadd_rn(__fadd_rn(nb[0], nb[1]), nb[2]);
      const float q = __fsub_rn(
          __fadd_rn(__fadd_rn(__fmul_rn(nb[0], nb[0]), __fmul_rn(nb[1], nb[1])), __fmul_rn(nb[2], nb[2])), dx2);
      const float inner = fmaxf(0.0f, __fsub_rn(__fmul_rn(s, s), __fmul_rn(3.0f, q)));
      d = __fmul_rn(third, __fadd_rn(s, __fsqrt_rn(inner)));
    }
  }
  return d;
}

// One sweep of FastSweepingLevelSet.propagate (level_set.py:284-327): every
// line along `axis` is walked by one thread, forward (dir > 0) or backward,
// applying propagate_update (level_set.py:267-271) to its cells in order.
// As in the reference, the lines run in parallel and read each other's cells
// while they change.  Consecutive threads take consecutive cells of the
// fastest other axis.
__global__ void k_fs_sweep(Geom g, int axis, int dir, float* phi_temp, const float* __restrict__ phi,
                           const int32_t* __restrict__ valid, float dx1, float two_dx2, float dx2, float third) {
  int oa[2], no = 0;
  for (int k = 0; k < g.dim; ++k)
    if (k != axis) oa[no++] = k;
  const long long lines = g.count / g.n[axis];
  const int nfast = no == 2 ? g.n[oa[1]] : 1;
  for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < lines;
       l += (long long)gridDim.x * blockDim.x) {
    int c[3] = {0, 0, 0};
    if (no == 2) {
      c[oa[0]] = (int)(l / nfast);
      c[oa[1]] = (int)(l % nfast);
    } else {
      c[oa[0]] = (int)l;
    }
    const int n = g.n[axis];
    for (int step = 0; step < n; ++step) {
      c[axis] = dir > 0 ? step : n - 1 - step;
      const long long i = g.index(c[0], c[1], c[2]);
      if (valid[i] != -1) continue;
      const float d = eikonal(g, phi_temp, i, c, dx1, two_dx2, dx2, third);
      if (fabsf(d) < fabsf(phi_temp[i])) phi_temp[i] = __fmul_rn(d, gsign(phi[i]));
    }
  }
}

// ---- FastSweepingLevelSet.build_from_markers (level_set.py:381-392) --------

// The cell of a marker (coordinates / dx truncated toward zero, the
// reference's cast) and its distance to the cell centre (I + 0.5) dx; false
// when the cell is outside the grid or a coordinate is not finite.
__device__ __forceinline__ bool marker_cell(const Geom& g, const float* m, float dx, int c[3], float* d) {
  float s = 0.0f;
  bool in = true;
  c[0] = c[1] = c[2] = 0;
  for (int a = 0; a < g.dim; ++a) {
    const float q = __fdiv_rn(m[a], dx);
    if (!isfinite(q) || fabsf(q) > 2.0e9f) return false;
    const int I = (int)q;  // truncation toward zero
    c[a] = I;
    in = in && I >= 0 && I < g.n[a];
    const float diff = __fsub_rn(m[a], __fmul_rn(__fadd_rn((float)I, 0.5f), dx));
    s = a == 0 ? __fmul_rn(diff, diff) : __fadd_rn(s, __fmul_rn(diff, diff));
  }
  *d = __fsqrt_rn(s);
  return in;
}

// phi.fill(1e20); valid holds INT_MAX until k_marker_owner has run.
__global__ void k_markers_init(Geom g, float* __restrict__ phi, int32_t* __restrict__ valid) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < g.count;
       i += (long long)gridDim.x * blockDim.x) {
    phi[i] = 1e20f;
    valid[i] = 0x7fffffff;
  }
}

// LevelSet.distance_to_markers (level_set.py:114-122), pass 1: every cell
// keeps the smallest distance of its markers (non-negative floats order as
// their bit patterns).  The reference's parallel loop races between markers
// of one cell; the smallest distance, then the smallest marker index (pass
// 2), is what its loop gives when the markers run in index order.
__global__ void k_marker_min_d(Geom g, const float* __restrict__ markers, int n, float dx, float* phi) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    int c[3];
    float d;
    if (!marker_cell(g, markers + (long long)p * g.dim, dx, c, &d)) continue;
    atomicMin(reinterpret_cast<unsigned int*>(phi) + g.index(c[0], c[1], c[2]), __float_as_uint(d));
  }
}

// Pass 2: the smallest index among the markers at that distance.
__global__ void k_marker_owner(Geom g, const float* __restrict__ markers, int n, float dx,
                               const float* __restrict__ phi, int32_t* valid) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    int c[3];
    float d;
    if (!marker_cell(g, markers + (long long)p * g.dim, dx, c, &d)) continue;
    const long long i = g.index(c[0], c[1], c[2]);
    if (__float_as_uint(d) == __float_as_uint(phi[i])) atomicMin(valid + i, p);
  }
}

__global__ void k_marker_valid_fix(Geom g, int32_t* __restrict__ valid) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < g.count;
       i += (long long)gridDim.x * blockDim.x)
    if (valid[i] == 0x7fffffff) valid[i] = -1;
}

// One sweep of FastSweepingLevelSet.markers_propagate (level_set.py:336-379)
// along `axis`: a thread walks each line in direction dir; a cell whose
// neighbour one step ahead (index + dir) is in the grid and owns a marker
// takes that marker's distance when smaller, and the marker.  A line reads
// only its own cells, so the result is that of the reference's serial walk.
// A neighbour without a marker (valid -1) is skipped (the reference indexes
// markers[-1] there).
__global__ void k_marker_sweep(Geom g, int axis, int dir, const float* __restrict__ markers, float dx,
                               float* __restrict__ phi, int32_t* __restrict__ valid) {
  int oa[2], no = 0;
  for (int k = 0; k < g.dim; ++k)
    if (k != axis) oa[no++] = k;
  const long long lines = g.count / g.n[axis];
  const int nfast = no == 2 ? g.n[oa[1]] : 1;
  const long long st = g.stride(axis) * dir;
  for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < lines;
       l += (long long)gridDim.x * blockDim.x) {
    int c[3] = {0, 0, 0};
    if (no == 2) {
      c[oa[0]] = (int)(l / nfast);
      c[oa[1]] = (int)(l % nfast);
    } else {
      c[oa[0]] = (int)l;
    }
    const int n = g.n[axis];
    for (int step = 0; step < n; ++step) {
      c[axis] = dir > 0 ? step : n - 1 - step;
      const int na = c[axis] + dir;
      if (na < 0 || na >= n) continue;
      const long long i = g.index(c[0], c[1], c[2]);
      const int32_t v = valid[i + st];
      if (v < 0) continue;
      float s = 0.0f;
      for (int a = 0; a < g.dim; ++a) {
        const float diff = __fsub_rn(markers[(long long)v * g.dim + a], __fmul_rn(__fadd_rn((float)c[a], 0.5f), dx));
        s = a == 0 ? __fmul_rn(diff, diff) : __fadd_rn(s, __fmul_rn(diff, diff));
      }
      const float d = __fsqrt_rn(s);
      if (d < phi[i]) {
        phi[i] = d;
        valid[i] = v;
      }
    }
  }
}

// LevelSet.target_minus (level_set.py:124-146), first loop (after
// valid.fill(-1)): phi -= r, the marker radius (0.99 dx folded in double).
__global__ void k_target_minus_a(Geom g, float* __restrict__ phi, int32_t* __restrict__ valid, float r) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < g.count;
       i += (long long)gridDim.x * blockDim.x) {
    phi[i] = __fsub_rn(phi[i], r);
    valid[i] = -1;
  }
}

// Second loop: cells with a sign change and phi <= 0 are known (valid 0,
// phi_temp = phi), other phi <= 0 cells get phi_temp = -1 (swept later),
// phi > 0 cells are known with phi_temp = phi.
__global__ void k_target_minus_b(Geom g, const float* __restrict__ phi, float* __restrict__ phi_temp,
                                 int32_t* __restrict__ valid) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < g.count;
       i += (long long)gridDim.x * blockDim.x) {
    int c[3];
    g.coords(i, c);
    const float p = phi[i];
    bool change = false;
    for (int k = 0; k < g.dim; ++k)
      for (int s = -1; s <= 1; s += 2) {
        const int v = c[k] + s;
        if (v >= 0 && v < g.n[k] && gsign(p) != gsign(phi[i + s * g.stride(k)])) change = true;
      }
    if (change && p <= 0.0f) {
      valid[i] = 0;
      phi_temp[i] = p;
    } else if (p <= 0.0f) {
      phi_temp[i] = -1.0f;
    } else {
      phi_temp[i] = p;
      valid[i] = 0;
    }
  }
}

// LevelSet.smoothing (level_set.py:148-163): out = min(mean of the in-range
// axis neighbours of in (summed axis by axis, lower then upper), in).
__global__ void k_ls_smooth(Geom g, float* __restrict__ out, const float* __restrict__ in) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < g.count;
       i += (long long)gridDim.x * blockDim.x) {
    int c[3];
    g.coords(i, c);
    float avg = 0.0f;
    int tot = 0;
    for (int k = 0; k < g.dim; ++k)
      for (int s = -1; s <= 1; s += 2) {
        const int v = c[k] + s;
        if (v >= 0 && v < g.n[k]) {
          avg = __fadd_rn(avg, in[i + s * g.stride(k)]);
          ++tot;
        }
      }
    avg = __fdiv_rn(avg, (float)tot);
    out[i] = avg < in[i] ? avg : in[i];
  }
}

}  // namespace mg
