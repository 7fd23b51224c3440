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

}  // namespace mg
