// The simulator's velocity steps around the projection: semi-Lagrangian
// advection, velocity extrapolation, gravity and the solid boundary.  f32 with
// explicit round-to-nearest intrinsics in the reference's operation order.
#pragma once
#include "mg_strategies.cuh"

namespace mg {

// Geometry of the MAC face field of axis k (shape res + e_k).
__device__ __forceinline__ Geom face_geom(const Geom& g, int k) {
  Geom f = g;
  f.n[k] += 1;
  f.count = (long long)f.n[0] * f.n[1] * f.n[2];
  return f;
}

struct Vel {
  const float* u[3];
};

// FluidSimulator.vel_interp (fluid_simulator.py:138-143): component q sampled
// at pos / dx - 0.5 (1 - e_q).
__device__ __forceinline__ void vel_interp(const Vel& V, const Geom& g, float dx, const float pos[3], float v[3]) {
  for (int q = 0; q < g.dim; ++q) {
    float s[3] = {0.0f, 0.0f, 0.0f};
    for (int a = 0; a < g.dim; ++a) s[a] = __fsub_rn(__fdiv_rn(pos[a], dx), a == q ? 0.0f : 0.5f);
    v[q] = sample(face_field(V.u[q], g, q), s);
  }
}

// FluidSimulator.advect (fluid_simulator.py:216-221) into dst for every index
// of the field (cells: field = -1, offset 0.5; faces of axis k: field = k,
// offset 0.5 (1 - e_k)): a midpoint (RK2) backtrace through the velocity and
// a sample of src at the departure point.
__global__ void k_advect(Geom g, int field, Vel V, const float* __restrict__ src, float* __restrict__ dst, float dx,
                         float dt) {
  const Geom f = field < 0 ? g : face_geom(g, field);
  Field fs;
  fs.v = src;
  fs.dim = g.dim;
  fs.n[0] = f.n[0];
  fs.n[1] = f.n[1];
  fs.n[2] = f.n[2];
  const float half_dt = __fmul_rn(0.5f, dt);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < f.count;
       i += (long long)gridDim.x * blockDim.x) {
    int c[3];
    f.coords(i, c);
    float off[3], pos[3], v[3], mid[3], p0[3], s[3];
    for (int a = 0; a < 3; ++a) off[a] = (a >= g.dim || (field >= 0 && a == field)) ? 0.0f : 0.5f;
    for (int a = 0; a < g.dim; ++a) pos[a] = __fmul_rn(__fadd_rn((float)c[a], off[a]), dx);
    vel_interp(V, g, dx, pos, v);
    for (int a = 0; a < g.dim; ++a) mid[a] = __fsub_rn(pos[a], __fmul_rn(v[a], half_dt));
    vel_interp(V, g, dx, mid, v);
    for (int a = 0; a < g.dim; ++a) p0[a] = __fsub_rn(pos[a], __fmul_rn(v[a], dt));
    for (int a = 0; a < 3; ++a) s[a] = a < g.dim ? __fsub_rn(__fdiv_rn(p0[a], dx), off[a]) : 0.0f;
    dst[i] = sample(fs, s);
  }
}

// FluidSimulator.mark_valid(k) (fluid_simulator.py:244-252): a face is valid
// when a cell on either side is FLUID.
__global__ void k_mark_valid(Geom g, int k, const int32_t* __restrict__ ct, int32_t* __restrict__ valid) {
  const Geom f = face_geom(g, k);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < f.count;
       i += (long long)gridDim.x * blockDim.x) {
    int c[3];
    f.coords(i, c);
    const bool in1 = c[k] >= 1, in0 = c[k] < g.n[k];
    const bool fl1 = in1 && ct[g.index(c[0] - (k == 0), c[1] - (k == 1), c[2] - (k == 2))] == FLUID;
    const bool fl0 = in0 && ct[g.index(c[0], c[1], c[2])] == FLUID;
    valid[i] = (fl1 || fl0) ? 1 : 0;
  }
}

// One round of FluidSimulator.diffuse_quantity (fluid_simulator.py:254-266)
// for the faces of axis k, ping-ponged: an invalid face with valid neighbours
// in its 3^d box (offsets in row-major order) takes their mean and becomes
// valid; every other face is copied.  A neighbour outside the face field
// counts as invalid.
__global__ void k_diffuse(Geom g, int k, const float* __restrict__ src, float* __restrict__ dst,
                          const int32_t* __restrict__ vsrc, int32_t* __restrict__ vdst) {
  const Geom f = face_geom(g, k);
  const int d = g.dim;
  const int span = d == 3 ? 27 : 9;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < f.count;
       i += (long long)gridDim.x * blockDim.x) {
    if (vsrc[i] != 0) {
      dst[i] = src[i];
      vdst[i] = vsrc[i];
      continue;
    }
    int c[3];
    f.coords(i, c);
    float tot = 0.0f;
    int cnt = 0;
    for (int o = 0; o < span; ++o) {
      int n[3] = {c[0], c[1], c[2]};
      if (d == 3) {
        n[0] += o / 9 - 1;
        n[1] += (o / 3) % 3 - 1;
        n[2] += o % 3 - 1;
      } else {
        n[0] += o / 3 - 1;
        n[1] += o % 3 - 1;
      }
      bool in = true;
      for (int a = 0; a < d; ++a) in = in && n[a] >= 0 && n[a] < f.n[a];
      if (!in) continue;
      const long long j = f.index(n[0], n[1], n[2]);
      if (vsrc[j] == 1) {
        tot = __fadd_rn(tot, src[j]);
        ++cnt;
      }
    }
    dst[i] = cnt > 0 ? __fdiv_rn(tot, (float)cnt) : src[i];
    vdst[i] = cnt > 0 ? 1 : vsrc[i];
  }
}

// FluidSimulator.enforce_boundary (fluid_simulator.py:168-174): both faces of
// every SOLID cell along every axis get velocity 0.
__global__ void k_enforce_boundary(Geom g, Vel V, const int32_t* __restrict__ ct) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < g.count;
       i += (long long)gridDim.x * blockDim.x) {
    if (ct[i] != SOLID) continue;
    int c[3];
    g.coords(i, c);
    for (int k = 0; k < g.dim; ++k) {
      const Geom f = face_geom(g, k);
      float* u = const_cast<float*>(V.u[k]);
      u[f.index(c[0], c[1], c[2])] = 0.0f;
      u[f.index(c[0] + (k == 0), c[1] + (k == 1), c[2] + (k == 2))] = 0.0f;
    }
  }
}

// FluidSimulator.add_gravity (fluid_simulator.py:160-166) for axis k:
// u += g * dt on every face, with g (a Python constant, rounded to f32) times
// the f32 argument dt formed in f32 as the reference does.
__global__ void k_add_gravity(Geom g, int k, float* __restrict__ u, float gk, float dt) {
  const Geom f = face_geom(g, k);
  const float gdt = __fmul_rn(gk, dt);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < f.count;
       i += (long long)gridDim.x * blockDim.x)
    u[i] = __fadd_rn(u[i], gdt);
}

}  // namespace mg
