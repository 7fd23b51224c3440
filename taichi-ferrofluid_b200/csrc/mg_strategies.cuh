// Strategy kernels beyond the ghost-fluid pressure: the whole-domain magnetic
// potential solve of the 3D ferrofluid substep, and Galerkin coarsening of a
// stored-coefficient operator.
#pragma once
#include "mg_common.cuh"

namespace mg {

__device__ __forceinline__ bool is_pin(const int c[3], const int pin[3], int dim) {
  return c[0] == pin[0] && c[1] == pin[1] && (dim == 2 || c[2] == pin[2]);
}

// Harmonic mean of the permeabilities mu = 1 + chi of two cells.
__device__ __forceinline__ float mu_face(float chi_a, float chi_b) {
  const float ma = __fadd_rn(1.0f, chi_a), mb = __fadd_rn(1.0f, chi_b);
  return __fdiv_rn(__fmul_rn(2.0f, __fmul_rn(ma, mb)), __fadd_rn(ma, mb));
}

// k_build_psi_b for a compile-time dim (its per-axis arrays and the level's
// extents indexed by constants, so nothing is kept in local memory).
template <int DIM>
__device__ __forceinline__ void k_build_psi_b_dim(Level L, float* b, const float* __restrict__ chi, float H0, float H1, float H2,
                              float dx, int p0, int p1, int p2) {
  const float Hk[3] = {H0, H1, H2};
  const int pin[3] = {p0, p1, p2};
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < L.g.count;
       i += (long long)gridDim.x * blockDim.x) {
    int c[3];
    L.g.coords(i, c);
    if (is_pin(c, pin, DIM)) {
      b[i] = 0.0f;
      continue;
    }
    float acc = 0.0f;
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
      const long long s = L.g.stride(k);
      if (c[k] + 1 < L.g.n[k]) acc = __fadd_rn(acc, __fmul_rn(Hk[k], mu_face(chi[i], chi[i + s])));
      if (c[k] > 0) acc = __fsub_rn(acc, __fmul_rn(Hk[k], mu_face(chi[i - s], chi[i])));
    }
    b[i] = -__fdiv_rn(acc, dx);
  }
}

// Magnetic potential right-hand side on level 0:
//   b_I = -(1/dx) sum_k H_k (mu(I, I+e_k) - mu(I-e_k, I))
// over faces inside the domain (no flux through the boundary), b = 0 at the
// pinned cell.  H is constant (the external field).
__global__ void k_build_psi_b(Level L, float* b, const float* __restrict__ chi, float H0, float H1, float H2,
                              float dx, int p0, int p1, int p2) {
  if (L.g.dim == 3) k_build_psi_b_dim<3>(L, b, chi, H0, H1, H2, dx, p0, p1, p2);
  else k_build_psi_b_dim<2>(L, b, chi, H0, H1, H2, dx, p0, p1, p2);
}

// k_build_psi_A for a compile-time dim (its per-axis arrays and the level's
// extents indexed by constants, so nothing is kept in local memory).
template <int DIM>
__device__ __forceinline__ void k_build_psi_A_dim(Level L, const float* __restrict__ chi, float dx, int p0, int p1, int p2) {
  const int pin[3] = {p0, p1, p2};
  const float dx2 = __fmul_rn(dx, dx);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < L.g.count;
       i += (long long)gridDim.x * blockDim.x) {
    int c[3];
    L.g.coords(i, c);
    if (is_pin(c, pin, DIM)) {
      L.Adiag[i] = __fdiv_rn(1.0f, dx2);
#pragma unroll
      for (int k = 0; k < DIM; ++k) L.Ax[k][i] = 0.0f;
      continue;
    }
    float d = 0.0f;
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
      const long long s = L.g.stride(k);
      float up = 0.0f;
      if (c[k] > 0) d = __fadd_rn(d, __fdiv_rn(mu_face(chi[i - s], chi[i]), dx2));
      if (c[k] + 1 < L.g.n[k]) {
        const float cf = __fdiv_rn(mu_face(chi[i], chi[i + s]), dx2);
        d = __fadd_rn(d, cf);
        int cn[3] = {c[0], c[1], c[2]};
        cn[k] += 1;
        up = is_pin(cn, pin, DIM) ? 0.0f : -cf;
      }
      L.Ax[k][i] = up;
    }
    L.Adiag[i] = d;
  }
}

// Magnetic potential operator on level 0: face coefficient mu(I, J) / dx^2
// (symmetric positive definite), Neumann at the domain boundary, Dirichlet
// psi = 0 at the pinned cell (its couplings removed, its row the identity
// times 1/dx^2).
__global__ void k_build_psi_A(Level L, const float* __restrict__ chi, float dx, int p0, int p1, int p2) {
  if (L.g.dim == 3) k_build_psi_A_dim<3>(L, chi, dx, p0, p1, p2);
  else k_build_psi_A_dim<2>(L, chi, dx, p0, p1, p2);
}

// chi of a coarse level: the mean of the 2^dim children of the finer level,
// summed in lexicographic order from 0 and multiplied by 2^-dim (exact) - the
// coarse coefficient field of a rediscretised level.
__global__ void k_mean_children(Geom gf, const float* __restrict__ fine, Geom gc, float* __restrict__ coarse) {
  const float w = gc.dim == 3 ? 0.125f : 0.25f;
  for (long long ic = (long long)blockIdx.x * blockDim.x + threadIdx.x; ic < gc.count;
       ic += (long long)gridDim.x * blockDim.x) {
    int cc[3];
    gc.coords(ic, cc);
    float acc = 0.0f;
    for (int o0 = 0; o0 < 2; ++o0)
      for (int o1 = 0; o1 < 2; ++o1)
        for (int o2 = 0; o2 < (gc.dim == 3 ? 2 : 1); ++o2)
          acc = __fadd_rn(acc, fine[gf.index(2 * cc[0] + o0, 2 * cc[1] + o1, gc.dim == 3 ? 2 * cc[2] + o2 : 0)]);
    coarse[ic] = __fmul_rn(acc, w);
  }
}

// k_galerkin for a compile-time dim (its per-axis arrays and the level's
// extents indexed by constants, so nothing is kept in local memory).
template <int DIM>
__device__ __forceinline__ void k_galerkin_dim(Level F, Level C, float scale) {
  for (long long ic = (long long)blockIdx.x * blockDim.x + threadIdx.x; ic < C.g.count;
       ic += (long long)gridDim.x * blockDim.x) {
    int cc[3];
    C.g.coords(ic, cc);
    constexpr int dim = DIM;
    float d = 0.0f, ax[3] = {0.0f, 0.0f, 0.0f};
    for (int o0 = 0; o0 < 2; ++o0)
      for (int o1 = 0; o1 < 2; ++o1)
        for (int o2 = 0; o2 < (dim == 3 ? 2 : 1); ++o2) {
          const int o[3] = {o0, o1, o2};
          const long long i = F.g.index(2 * cc[0] + o0, 2 * cc[1] + o1, dim == 3 ? 2 * cc[2] + o2 : 0);
          d = __fadd_rn(d, F.Adiag[i]);
#pragma unroll
          for (int k = 0; k < dim; ++k) {
            const float a = F.Ax[k][i];
            if (o[k] == 0) d = __fadd_rn(d, __fmul_rn(2.0f, a));  // internal face
            else ax[k] = __fadd_rn(ax[k], a);                       // face to the next block
          }
        }
    C.Adiag[ic] = __fmul_rn(scale, d);
#pragma unroll
    for (int k = 0; k < dim; ++k) C.Ax[k][ic] = (cc[k] + 1 < C.g.n[k]) ? __fmul_rn(scale, ax[k]) : 0.0f;
  }
}

// Galerkin coarse operator A_c = P^T A P for the reference's transfer pair
// (prolongation: piecewise constant, mgpcg.py:120-123; restriction: the
// unweighted sum of the 2^d children, mgpcg.py:111-118):
//   Ax_c[J][k] = sum of Ax[i][k] over the children i of J on its +k face
//   Adiag_c[J] = sum of Adiag[i] over the children + 2 * sum of the Ax of the
//                faces between two children of J
// Children are visited in lexicographic order.  Both sums are then multiplied
// by `scale` (a power of two, so the product is exact): 1 gives P^T A P, 1/2
// the over-corrected coarse operator of the magnetic potential Strategy.
__global__ void k_galerkin(Level F, Level C, float scale) {
  if (C.g.dim == 3) k_galerkin_dim<3>(F, C, scale);
  else k_galerkin_dim<2>(F, C, scale);
}

// ---------------------------------------------------------------------------
// The reference's other Strategies and the step after the solve
// ---------------------------------------------------------------------------

// utils.sample (utils.py:8-33): bi/trilinear interpolation of a cell-centred
// field at a position in index units, indices clamped to the grid, weights to
// [0, 1]; int() truncates toward zero as Taichi's cast does.
struct Field {
  const float* v;
  int n[3];
  int dim;
  __device__ __forceinline__ float at(int i, int j, int k) const {
    return v[dim == 3 ? ((long long)i * n[1] + j) * n[2] + k : (long long)i * n[1] + j];
  }
};

__device__ __forceinline__ int clampi(int v, int a, int b) { return v < a ? a : (v > b ? b : v); }
__device__ __forceinline__ float clampf(float v, float a, float b) { return fmaxf(a, fminf(b, v)); }

__device__ float sample(const Field& f, const float pos[3]) {
  const int i = clampi((int)pos[0], 0, f.n[0] - 1), j = clampi((int)pos[1], 0, f.n[1] - 1);
  const int ip = clampi(i + 1, 0, f.n[0] - 1), jp = clampi(j + 1, 0, f.n[1] - 1);
  const float s = clampf(__fsub_rn(pos[0], (float)i), 0.0f, 1.0f), t = clampf(__fsub_rn(pos[1], (float)j), 0.0f, 1.0f);
  const float os = __fsub_rn(1.0f, s), ot = __fsub_rn(1.0f, t);
  if (f.dim == 2) {
    const float a = __fadd_rn(__fmul_rn(f.at(i, j, 0), os), __fmul_rn(f.at(ip, j, 0), s));
    const float b = __fadd_rn(__fmul_rn(f.at(i, jp, 0), os), __fmul_rn(f.at(ip, jp, 0), s));
    return __fadd_rn(__fmul_rn(a, ot), __fmul_rn(b, t));
  }
  const int k = clampi((int)pos[2], 0, f.n[2] - 1), kp = clampi(k + 1, 0, f.n[2] - 1);
  const float u = clampf(__fsub_rn(pos[2], (float)k), 0.0f, 1.0f), ou = __fsub_rn(1.0f, u);
  const float a0 = __fadd_rn(__fmul_rn(f.at(i, j, k), os), __fmul_rn(f.at(ip, j, k), s));
  const float b0 = __fadd_rn(__fmul_rn(f.at(i, jp, k), os), __fmul_rn(f.at(ip, jp, k), s));
  const float a1 = __fadd_rn(__fmul_rn(f.at(i, j, kp), os), __fmul_rn(f.at(ip, j, kp), s));
  const float b1 = __fadd_rn(__fmul_rn(f.at(i, jp, kp), os), __fmul_rn(f.at(ip, jp, kp), s));
  const float lo = __fadd_rn(__fmul_rn(a0, ot), __fmul_rn(b0, t));
  const float hi = __fadd_rn(__fmul_rn(a1, ot), __fmul_rn(b1, t));
  return __fadd_rn(__fmul_rn(lo, ou), __fmul_rn(hi, u));
}

// MAC face field k (shape res + e_k) as a sampled Field.
__device__ __forceinline__ Field face_field(const float* v, const Geom& g, int k) {
  Field f;
  f.v = v;
  f.dim = g.dim;
  f.n[0] = g.n[0] + (k == 0);
  f.n[1] = g.n[1] + (k == 1);
  f.n[2] = g.dim == 3 ? g.n[2] + (k == 2) : 1;
  return f;
}

// |H_interp(c + 0.5)|^2 (ferrofluid_simulator.py:64-69): component q of the
// MAC field H sampled at c + 0.5 - 0.5 (1 - e_q); squares summed in axis order.
__device__ __forceinline__ float h2_at(const float* const Hs[3], const Geom& g, const int c[3]) {
  float hh = 0.0f;
  for (int q = 0; q < g.dim; ++q) {
    float pos[3] = {0.0f, 0.0f, 0.0f};
    for (int a = 0; a < g.dim; ++a) pos[a] = __fsub_rn(__fadd_rn((float)c[a], 0.5f), a == q ? 0.0f : 0.5f);
    const float h = sample(face_field(Hs[q], g, q), pos);
    hh = __fadd_rn(hh, __fmul_rn(h, h));
  }
  return hh;
}

// k_apply_pressure for a compile-time dim (its per-axis arrays and the level's
// extents indexed by constants, so nothing is kept in local memory).
template <int DIM>
__device__ __forceinline__ void k_apply_pressure_dim(Level L, int k, float* __restrict__ u, const float* __restrict__ pr,
                                 const int32_t* __restrict__ ct32, const float* __restrict__ phi, float scale,
                                 float p0, int ghost, float clamp, const float* H0, const float* H1,
                                 const float* H2, float coef) {
  const Geom& g = L.g;
  const float* const Hs[3] = {H0, H1, H2};
  const int nu1 = g.n[1] + (k == 1), nu2 = DIM == 3 ? g.n[2] + (k == 2) : 1;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < g.count;
       i += (long long)gridDim.x * blockDim.x) {
    int c[3];
    g.coords(i, c);
    const bool v1 = c[k] >= 1;  // I - e_k inside the grid (I always is)
    const long long i1 = i - g.stride(k);
    const int t = ct32 ? ct32[i] : L.type[i];
    const int t1 = v1 ? (ct32 ? ct32[i1] : L.type[i1]) : SOLID;
    if (!(t1 == FLUID || t == FLUID)) continue;
    const long long f = ((long long)c[0] * nu1 + c[1]) * nu2 + c[2];
    if (t1 == SOLID || t == SOLID) {
      u[f] = 0.0f;
    } else if (t == AIR) {  // fluid-air
      if (H0) {
        const float pa = __fadd_rn(p0, __fmul_rn(coef, h2_at(Hs, g, c)));
        u[f] = __fsub_rn(u[f], __fmul_rn(scale, __fsub_rn(pa, pr[i1])));
      } else if (ghost) {
        const float cc = __fdiv_rn(__fsub_rn(phi[i1], phi[i]), phi[i1]);
        u[f] = __fsub_rn(u[f], __fmul_rn(__fmul_rn(scale, __fsub_rn(p0, pr[i1])), fminf(cc, clamp)));
      } else {
        u[f] = __fsub_rn(u[f], __fmul_rn(scale, __fsub_rn(p0, pr[i1])));
      }
    } else if (t1 == AIR) {  // air-fluid
      if (H0) {
        int c1[3] = {c[0], c[1], c[2]};
        c1[k] -= 1;
        const float pa = __fadd_rn(p0, __fmul_rn(coef, h2_at(Hs, g, c1)));
        u[f] = __fsub_rn(u[f], __fmul_rn(scale, __fsub_rn(pr[i], pa)));
      } else if (ghost) {
        const float cc = __fdiv_rn(__fsub_rn(phi[i], phi[i1]), phi[i]);
        u[f] = __fsub_rn(u[f], __fmul_rn(__fmul_rn(scale, __fsub_rn(pr[i], p0)), fminf(cc, clamp)));
      } else {
        u[f] = __fsub_rn(u[f], __fmul_rn(scale, __fsub_rn(pr[i], p0)));
      }
    } else {  // fluid-fluid
      u[f] = __fsub_rn(u[f], __fmul_rn(scale, __fsub_rn(pr[i], pr[i1])));
    }
  }
}

// FluidSimulator.apply_pressure (fluid_simulator.py:193-214) and, with H given,
// FerrofluidSimulator.apply_magnetic_force (ferrofluid_simulator.py:115-137)
// for axis k: the pressure-gradient update of the MAC velocity u_k on face I
// (between cells I - e_k and I) of every cell I.  Out-of-range cells are SOLID
// (fluid_simulator.py:123-136).  With H the AIR side pressure is
// p0 + coef |H(air cell + 0.5)|^2 and no ghost-fluid factor applies.
// Cell labels come from ct32 (the simulator's int32 field) or, when it is
// null, from the plan's level-0 labels.  scale = dt / (rho dx).
__global__ void k_apply_pressure(Level L, int k, float* __restrict__ u, const float* __restrict__ pr,
                                 const int32_t* __restrict__ ct32, const float* __restrict__ phi, float scale,
                                 float p0, int ghost, float clamp, const float* H0, const float* H1,
                                 const float* H2, float coef) {
  if (L.g.dim == 3) k_apply_pressure_dim<3>(L, k, u, pr, ct32, phi, scale, p0, ghost, clamp, H0, H1, H2, coef);
  else k_apply_pressure_dim<2>(L, k, u, pr, ct32, phi, scale, p0, ghost, clamp, H0, H1, H2, coef);
}

// LevelSet.theta (level_set.py:24-30): smoothed Heaviside of half width eps.
// The constants are folded on the host in double and rounded once to f32:
// two_eps = 2 eps, pi, inv_2pi = 1 / (2 pi).
struct ThetaK {
  float eps, two_eps, pi, inv_2pi;
};

__device__ __forceinline__ float theta_h(float phi, const ThetaK& t) {
  if (phi <= -t.eps) return 0.0f;
  if (phi >= t.eps) return 1.0f;
  return __fadd_rn(__fadd_rn(0.5f, __fdiv_rn(phi, t.two_eps)),
                   __fmul_rn(t.inv_2pi, sinf(__fdiv_rn(__fmul_rn(t.pi, phi), t.eps))));
}

// PressureProjectWithVolumeControlStrategy.calc_volume (volume_control.py:22-31):
// sum over cells of the mean over the 2^d cell corners of theta(-phi(corner)),
// phi sampled at I + offset - 0.5, corners in row-major offset order.  The
// cell terms are f32 as in the reference; the sum over cells is FP64.
//
// With `state` (the controller of volume_control.py:8-20, 39-51, in FP64:
// state[0] step, [1] vol_0, [2] y, [3] volume, [4] c, [5] k_p, [6] k_i,
// [7] dt) the last block also runs one controller step: the first step takes
// the volume as vol_0; later steps integrate the normalised error and set
// the divergence c = (-k_p x - k_i y) / (x + 1).  The volume goes to *out.
__global__ void __launch_bounds__(kRedThreads) k_volume(Geom g, const float* __restrict__ phi, ThetaK th,
                                                        double* partials, unsigned int* counter, double* out,
                                                        double* state) {
  __shared__ double sh[32];
  Field f;
  f.v = phi;
  f.dim = g.dim;
  f.n[0] = g.n[0];
  f.n[1] = g.n[1];
  f.n[2] = g.n[2];
  const int corners = g.dim == 3 ? 8 : 4;
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < g.count;
       i += (long long)gridDim.x * blockDim.x) {
    int c[3];
    g.coords(i, c);
    float cv = 0.0f;
    for (int o = 0; o < corners; ++o) {
      const float pos[3] = {__fsub_rn((float)(c[0] + ((o >> (g.dim - 1)) & 1)), 0.5f),
                            __fsub_rn((float)(c[1] + ((o >> (g.dim - 2)) & 1)), 0.5f),
                            g.dim == 3 ? __fsub_rn((float)(c[2] + (o & 1)), 0.5f) : 0.0f};
      cv = __fadd_rn(cv, theta_h(-sample(f, pos), th));
    }
    acc += (double)__fdiv_rn(cv, (float)corners);
  }
  double tot;
  if (last_block_total<kRedThreads>(acc, partials, counter, sh, &tot) && threadIdx.x == 0) {
    *out = tot;
    if (state) {
      const double step = state[0] + 1.0;
      state[0] = step;
      state[3] = tot;
      if (step == 1.0) {
        state[1] = tot;
      } else {
        const double x = (tot - state[1]) / state[1];
        const double y = state[2] + x * state[7];
        state[2] = y;
        state[4] = (-state[5] * x - state[6] * y) / (x + 1.0);
      }
    }
  }
}

// PressureProjectWithVolumeControlStrategy.add_c (volume_control.py:33-37,
// 51): b += c (rounded to f32) on FLUID cells, skipped on the controller's
// first step, with c read from the controller state on the device.
__global__ void k_add_c(Level L, float* b, const double* __restrict__ state) {
  if (state[0] == 1.0) return;
  const float c = (float)state[4];
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < L.g.count;
       i += (long long)gridDim.x * blockDim.x)
    if (L.type[i] == FLUID) b[i] = __fadd_rn(b[i], c);
}

// k_build_magnetic_b for a compile-time dim (its per-axis arrays and the level's
// extents indexed by constants, so nothing is kept in local memory).
template <int DIM>
__device__ __forceinline__ void k_build_magnetic_b_dim(Level L, const float* __restrict__ v0, const float* __restrict__ v1,
                                   const float* __restrict__ v2, const float* __restrict__ H0,
                                   const float* __restrict__ H1, const float* __restrict__ H2, float p0, float sA,
                                   float sB, float coef, float* b) {
  const float* vel[3] = {v0, v1, v2};
  const float* Hs[3] = {H0, H1, H2};
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < L.g.count;
       i += (long long)gridDim.x * blockDim.x) {
    if (L.type[i] != FLUID) continue;
    int c[3];
    L.g.coords(i, c);
    float bi = b[i];
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
      int cp[3] = {c[0], c[1], c[2]};
      cp[k] += 1;
      bi = __fadd_rn(bi, __fsub_rn(vel_at(vel[k], L.g, k, c[0], c[1], c[2]), vel_at(vel[k], L.g, k, cp[0], cp[1], cp[2])));
    }
    bi = __fmul_rn(bi, sB);
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
#pragma unroll
      for (int s = -1; s <= 1; s += 2) {
        const int8_t nt = nb_type(L, i, c, k, s);
        if (nt == SOLID) {
          if (s < 0) {
            bi = __fsub_rn(bi, __fmul_rn(sB, __fsub_rn(vel_at(vel[k], L.g, k, c[0], c[1], c[2]), 0.0f)));
          } else {
            int cp[3] = {c[0], c[1], c[2]};
            cp[k] += 1;
            bi = __fadd_rn(bi, __fmul_rn(sB, __fsub_rn(vel_at(vel[k], L.g, k, cp[0], cp[1], cp[2]), 0.0f)));
          }
        } else if (nt == AIR) {
          int cn[3] = {c[0], c[1], c[2]};
          cn[k] += s;
          bi = __fadd_rn(bi, __fmul_rn(sA, __fadd_rn(p0, __fmul_rn(coef, h2_at(Hs, L.g, cn)))));
        }
      }
    }
    b[i] = bi;
  }
}

// MagneticForceStrategy.build_b_kernel (magnetic_force.py:17-38): the pressure
// right-hand side whose AIR faces carry the magnetic pressure
// p0 + (k mu0 / 2) |H|^2, H sampled from the MAC field H at the face
// (FerrofluidSimulator.H_interp, ferrofluid_simulator.py:64-69); no ghost
// fluid factor in b.  coef = 0.5 * k * mu0.
__global__ void k_build_magnetic_b(Level L, const float* __restrict__ v0, const float* __restrict__ v1,
                                   const float* __restrict__ v2, const float* __restrict__ H0,
                                   const float* __restrict__ H1, const float* __restrict__ H2, float p0, float sA,
                                   float sB, float coef, float* b) {
  if (L.g.dim == 3) k_build_magnetic_b_dim<3>(L, v0, v1, v2, H0, H1, H2, p0, sA, sB, coef, b);
  else k_build_magnetic_b_dim<2>(L, v0, v1, v2, H0, H1, H2, p0, sA, sB, coef, b);
}

// PotentialFunctionStrategy (potential_function.py:19-55), the reference's
// form: whole domain, A negative definite, cell 0 pinned, in_domain tested
// against the FINE resolution on every level, chi sampled at the faces.
__device__ __forceinline__ bool in_domain(const int c[3], const int res[3], int dim) {
  for (int k = 0; k < dim; ++k)
    if (c[k] < 0 || c[k] + 1 > res[k]) return false;
  return true;
}

// k_build_potential_b for a compile-time dim (its per-axis arrays and the level's
// extents indexed by constants, so nothing is kept in local memory).
template <int DIM>
__device__ __forceinline__ void k_build_potential_b_dim(Level L, float* b, const float* __restrict__ chi, const float* __restrict__ Hx0,
                                    const float* __restrict__ Hx1, const float* __restrict__ Hx2, int r0, int r1,
                                    int r2) {
  const int res[3] = {r0, r1, r2};
  const float* Hx[3] = {Hx0, Hx1, Hx2};
  Field fc;
  fc.v = chi;
  fc.dim = DIM;
  fc.n[0] = L.g.n[0];
  fc.n[1] = L.g.n[1];
  fc.n[2] = L.g.n[2];
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < L.g.count;
       i += (long long)gridDim.x * blockDim.x) {
    int c[3];
    L.g.coords(i, c);
    const bool origin = c[0] == 0 && c[1] == 0 && (DIM == 2 || c[2] == 0);
    if (origin) {
      b[i] = 0.0f;
      continue;
    }
    if (!in_domain(c, res, DIM)) continue;
    float bi = b[i];
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
      int up[3] = {c[0], c[1], c[2]}, dn[3] = {c[0], c[1], c[2]};
      up[k] += 1;
      dn[k] -= 1;
      if (in_domain(up, res, DIM)) {
        float pos[3];
        for (int a = 0; a < 3; ++a) pos[a] = __fadd_rn((float)up[a], a == k ? 0.0f : 0.5f);
        bi = __fadd_rn(bi, __fmul_rn(sample(fc, pos), vel_at(Hx[k], L.g, k, up[0], up[1], up[2])));
      }
      if (in_domain(dn, res, DIM)) {
        float pos[3];
        for (int a = 0; a < 3; ++a) pos[a] = __fadd_rn((float)c[a], a == k ? 0.0f : 0.5f);
        bi = __fsub_rn(bi, __fmul_rn(sample(fc, pos), vel_at(Hx[k], L.g, k, c[0], c[1], c[2])));
      }
    }
    b[i] = bi;
  }
}

__global__ void k_build_potential_b(Level L, float* b, const float* __restrict__ chi, const float* __restrict__ Hx0,
                                    const float* __restrict__ Hx1, const float* __restrict__ Hx2, int r0, int r1,
                                    int r2) {
  if (L.g.dim == 3) k_build_potential_b_dim<3>(L, b, chi, Hx0, Hx1, Hx2, r0, r1, r2);
  else k_build_potential_b_dim<2>(L, b, chi, Hx0, Hx1, Hx2, r0, r1, r2);
}

// k_build_potential_A for a compile-time dim (its per-axis arrays and the level's
// extents indexed by constants, so nothing is kept in local memory).
template <int DIM>
__device__ __forceinline__ void k_build_potential_A_dim(Level L, int level, const float* __restrict__ chi, Geom fine, float dx_l,
                                    float inv_dx_l, int r0, int r1, int r2) {
  const int res[3] = {r0, r1, r2};
  Field fc;
  fc.v = chi;
  fc.dim = fine.dim;
  fc.n[0] = fine.n[0];
  fc.n[1] = fine.n[1];
  fc.n[2] = fine.n[2];
  const float sc = (float)(1 << level);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < L.g.count;
       i += (long long)gridDim.x * blockDim.x) {
    int c[3];
    L.g.coords(i, c);
    const bool origin = c[0] == 0 && c[1] == 0 && (DIM == 2 || c[2] == 0);
    if (origin) {
      L.Adiag[i] = inv_dx_l;
      continue;
    }
    if (!in_domain(c, res, DIM)) continue;
    float d = L.Adiag[i];
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
#pragma unroll
      for (int s = -1; s <= 1; s += 2) {
        int nb[3] = {c[0], c[1], c[2]};
        nb[k] += s;
        if (!in_domain(nb, res, DIM)) continue;
        float pos[3];
        for (int a = 0; a < 3; ++a)
          pos[a] = __fmul_rn(__fadd_rn((float)c[a], a == k ? 0.5f * (float)s : 0.0f), sc);
        const float cf = __fdiv_rn(__fadd_rn(1.0f, sample(fc, pos)), dx_l);
        d = __fsub_rn(d, cf);
        if (s > 0) L.Ax[k][i] = cf;
      }
    }
    L.Adiag[i] = d;
  }
}

// dx_l = dx 2^level and inv_dx_l = 1 / dx_l are folded on the host (the
// reference computes both in double before they meet f32 values).
__global__ void k_build_potential_A(Level L, int level, const float* __restrict__ chi, Geom fine, float dx_l,
                                    float inv_dx_l, int r0, int r1, int r2) {
  if (L.g.dim == 3) k_build_potential_A_dim<3>(L, level, chi, fine, dx_l, inv_dx_l, r0, r1, r2);
  else k_build_potential_A_dim<2>(L, level, chi, fine, dx_l, inv_dx_l, r0, r1, r2);
}

// FerrofluidSimulator.update_magnetic_susceptibility (ferrofluid_simulator.py:
// 71-75): chi = k (1 - theta(phi)).
__global__ void k_update_chi(Geom g, const float* __restrict__ phi, float kk, ThetaK th, float* __restrict__ chi) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < g.count;
       i += (long long)gridDim.x * blockDim.x)
    chi[i] = __fmul_rn(kk, __fsub_rn(1.0f, theta_h(phi[i], th)));
}

// FerrofluidSimulator.update_magnetic_field (ferrofluid_simulator.py:89-97)
// for axis k over the faces (shape res + e_k): H = H_ext - d psi / dx on
// interior faces, H = H_ext on the two boundary faces of the axis.
__global__ void k_update_H(Geom g, int k, const float* __restrict__ psi, const float* __restrict__ Hext, float dx,
                           float* __restrict__ H) {
  Geom f = g;
  f.n[k] += 1;
  f.count = (long long)f.n[0] * f.n[1] * f.n[2];
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < f.count;
       i += (long long)gridDim.x * blockDim.x) {
    int c[3];
    f.coords(i, c);
    float h = 0.0f;
    if (c[k] - 1 >= 0 && c[k] < g.n[k]) {
      const long long ic = g.index(c[0], c[1], c[2]);
      h = __fsub_rn(h, __fdiv_rn(__fsub_rn(psi[ic], psi[ic - g.stride(k)]), dx));
    }
    H[i] = __fadd_rn(h, Hext[i]);
  }
}

// ---------------------------------------------------------------------------
// SurfaceTension / SurfaceTensionStrategy (surface_tension.py:10-153): one
// implicit viscosity-like solve per velocity axis d on the whole domain.
// ---------------------------------------------------------------------------

// LevelSet.delta (level_set.py:32-37): smoothed Dirac delta of half width eps.
__device__ __forceinline__ float delta_h(float phi, const ThetaK& t) {
  if (phi <= -t.eps || phi >= t.eps) return 0.0f;
  return __fdiv_rn(__fadd_rn(1.0f, cosf(__fdiv_rn(__fmul_rn(t.pi, phi), t.eps))), t.two_eps);
}

__device__ __forceinline__ Field cell_field(const float* v, const Geom& g) {
  Field f;
  f.v = v;
  f.dim = g.dim;
  f.n[0] = g.n[0];
  f.n[1] = g.n[1];
  f.n[2] = g.n[2];
  return f;
}

// Position c + h (in half cells, h[a] in {-1, 0, 1}) + 0.5 (1 - e_d), times m.
__device__ __forceinline__ void face_pos(const int c[3], const int h[3], int d, int dim, float m, float pos[3]) {
  for (int a = 0; a < 3; ++a) {
    const float v = __fadd_rn(__fadd_rn((float)c[a], 0.5f * (float)h[a]), a == d || a >= dim ? 0.0f : 0.5f);
    pos[a] = __fmul_rn(v, m);
  }
}

// k_calc_n for a compile-time dim (its per-axis arrays and the level's
// extents indexed by constants, so nothing is kept in local memory).
template <int DIM>
__device__ __forceinline__ void k_calc_n_dim(Geom g, int d, const float* __restrict__ phi, float dx, float* __restrict__ n) {
  const Field fp = cell_field(phi, g);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < g.count;
       i += (long long)gridDim.x * blockDim.x) {
    int c[3];
    g.coords(i, c);
    float v[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
      int hp[3] = {0, 0, 0}, hm[3] = {0, 0, 0};
      hp[k] = 1;
      hm[k] = -1;
      float pp[3], pm[3];
      face_pos(c, hp, d, DIM, 1.0f, pp);
      face_pos(c, hm, d, DIM, 1.0f, pm);
      v[k] = __fdiv_rn(__fsub_rn(sample(fp, pp), sample(fp, pm)), dx);
    }
    float nn = __fmul_rn(v[0], v[0]);
    for (int k = 1; k < DIM; ++k) nn = __fadd_rn(nn, __fmul_rn(v[k], v[k]));
    const float norm = __fsqrt_rn(nn);
#pragma unroll
    for (int k = 0; k < DIM; ++k) n[k * g.count + i] = norm > 0.0f ? __fdiv_rn(v[k], norm) : v[k];
  }
}

// SurfaceTension.calc_n (surface_tension.py:108-121): n = grad phi / |grad phi|
// at I + 0.5 (1 - e_d) by central differences of sampled phi; |n| = 0 leaves
// the unnormalised gradient.  n is stored as dim planes of the cell grid.
__global__ void k_calc_n(Geom g, int d, const float* __restrict__ phi, float dx, float* __restrict__ n) {
  if (g.dim == 3) k_calc_n_dim<3>(g, d, phi, dx, n);
  else k_calc_n_dim<2>(g, d, phi, dx, n);
}

// SurfaceTension.calc_kappa (surface_tension.py:123-129): kappa = div n by
// central differences of the sampled component planes.
__global__ void k_calc_kappa(Geom g, const float* __restrict__ n, float dx, float* __restrict__ kappa) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < g.count;
       i += (long long)gridDim.x * blockDim.x) {
    int c[3];
    g.coords(i, c);
    float acc = 0.0f;
    for (int k = 0; k < g.dim; ++k) {
      const Field fk = cell_field(n + k * g.count, g);
      float pp[3], pm[3];
      for (int a = 0; a < 3; ++a) {
        pp[a] = __fadd_rn((float)c[a], a == k ? 0.5f : 0.0f);
        pm[a] = __fsub_rn((float)c[a], a == k ? 0.5f : 0.0f);
      }
      acc = __fadd_rn(acc, __fdiv_rn(__fsub_rn(sample(fk, pp), sample(fk, pm)), dx));
    }
    kappa[i] = acc;
  }
}

// k_build_st_b for a compile-time dim (its per-axis arrays and the level's
// extents indexed by constants, so nothing is kept in local memory).
template <int DIM>
__device__ __forceinline__ void k_build_st_b_dim(Geom g, int d, const float* __restrict__ u, const float* __restrict__ phi,
                             const float* __restrict__ n, const float* __restrict__ kappa, float sigma, float dt,
                             float dx, float dx2, ThetaK th, float* __restrict__ b) {
  const Field fp = cell_field(phi, g);
  const Field fu = face_field(u, g, d);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < g.count;
       i += (long long)gridDim.x * blockDim.x) {
    int c[3];
    g.coords(i, c);
    float bi = __fdiv_rn(vel_at(u, g, d, c[0], c[1], c[2]), dt);
    float pos[3];
    const int h0[3] = {0, 0, 0};
    face_pos(c, h0, d, DIM, 1.0f, pos);
    const float scale = __fmul_rn(sigma, delta_h(sample(fp, pos), th));
    float nv[3];
#pragma unroll
    for (int k = 0; k < DIM; ++k) nv[k] = n[k * g.count + i];
    // Du/Dn
    float du = 0.0f;
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
      float pp[3], pm[3];
      for (int a = 0; a < 3; ++a) {
        pp[a] = __fadd_rn((float)c[a], a == k ? 0.5f : 0.0f);
        pm[a] = __fsub_rn((float)c[a], a == k ? 0.5f : 0.0f);
      }
      const float gk = __fadd_rn(0.0f, __fdiv_rn(__fsub_rn(sample(fu, pp), sample(fu, pm)), dx));
      du = k == 0 ? __fmul_rn(gk, nv[0]) : __fadd_rn(du, __fmul_rn(gk, nv[k]));
    }
    // D2u/Dn2 = (n^T D2) n, accumulated in index order
    float D2[3][3];
    for (int k1 = 0; k1 < DIM; ++k1)
      for (int k2 = 0; k2 < DIM; ++k2) {
        float p00[3], p10[3], p01[3], p11[3];
        for (int a = 0; a < 3; ++a) {
          const float h1 = a == k1 ? 0.5f : 0.0f, h2 = a == k2 ? 0.5f : 0.0f;
          const float ca = (float)c[a];
          p00[a] = __fsub_rn(__fsub_rn(ca, h1), h2);
          p10[a] = __fsub_rn(__fadd_rn(ca, h1), h2);
          p01[a] = __fadd_rn(__fsub_rn(ca, h1), h2);
          p11[a] = __fadd_rn(__fadd_rn(ca, h1), h2);
        }
        const float v00 = sample(fu, p00), v10 = sample(fu, p10), v01 = sample(fu, p01), v11 = sample(fu, p11);
        D2[k1][k2] = __fdiv_rn(__fsub_rn(__fsub_rn(__fadd_rn(v11, v00), v10), v01), dx2);
      }
    float d2 = 0.0f;
    for (int j = 0; j < DIM; ++j) {
      float t = __fmul_rn(nv[0], D2[0][j]);
      for (int k = 1; k < DIM; ++k) t = __fadd_rn(t, __fmul_rn(nv[k], D2[k][j]));
      d2 = j == 0 ? __fmul_rn(t, nv[0]) : __fadd_rn(d2, __fmul_rn(t, nv[j]));
    }
    const float kap = kappa[i];
    const float inner = __fadd_rn(__fmul_rn(kap, nv[d]), __fmul_rn(dt, __fadd_rn(d2, __fmul_rn(kap, du))));
    b[i] = __fsub_rn(bi, __fmul_rn(scale, inner));
  }
}

// SurfaceTensionStrategy.build_b_kernel (surface_tension.py:23-71) for axis d:
// b = u_d / dt - sigma delta(phi) (kappa n_d + dt (n^T D2 n + kappa grad u . n))
// with grad u and the Hessian D2 of u_d from samples of the face field at
// half-cell offsets.  dx2 = dx^2 folded on the host.  Whole domain.
__global__ void k_build_st_b(Geom g, int d, const float* __restrict__ u, const float* __restrict__ phi,
                             const float* __restrict__ n, const float* __restrict__ kappa, float sigma, float dt,
                             float dx, float dx2, ThetaK th, float* __restrict__ b) {
  if (g.dim == 3) k_build_st_b_dim<3>(g, d, u, phi, n, kappa, sigma, dt, dx, dx2, th, b);
  else k_build_st_b_dim<2>(g, d, u, phi, n, kappa, sigma, dt, dx, dx2, th, b);
}

// k_build_st_A for a compile-time dim (its per-axis arrays and the level's
// extents indexed by constants, so nothing is kept in local memory).
template <int DIM>
__device__ __forceinline__ void k_build_st_A_dim(Level L, int level, Geom fine, int d, const float* __restrict__ phi, float inv_dt,
                             float scale, ThetaK th) {
  const Field fp = cell_field(phi, fine);
  const float m = (float)(1 << level);
  const float nscale = -scale;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < L.g.count;
       i += (long long)gridDim.x * blockDim.x) {
    int c[3];
    L.g.coords(i, c);
    float ad = inv_dt;
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
      int hp[3] = {0, 0, 0}, hm[3] = {0, 0, 0};
      hp[k] = 1;
      hm[k] = -1;
      if (c[k] + 1 < fine.n[k]) {
        float pos[3];
        face_pos(c, hp, d, DIM, m, pos);
        const float dl = delta_h(sample(fp, pos), th);
        L.Ax[k][i] = __fmul_rn(nscale, dl);
        ad = __fadd_rn(ad, __fmul_rn(scale, dl));
      }
      if (c[k] - 1 >= 0) {
        float pos[3];
        face_pos(c, hm, d, DIM, m, pos);
        ad = __fadd_rn(ad, __fmul_rn(scale, delta_h(sample(fp, pos), th)));
      }
    }
    L.Adiag[i] = ad;
  }
}

// SurfaceTensionStrategy.build_A_kernel (surface_tension.py:76-95) on one
// level: Adiag = 1/dt + scale sum of delta over the faces, Ax = -scale delta
// on the + faces, phi sampled at the face times 2^level; the face tests use
// the fine resolution res on every level.  inv_dt = 1/dt and
// scale = sigma dt / (dx 2^level)^2 are folded on the host.
__global__ void k_build_st_A(Level L, int level, Geom fine, int d, const float* __restrict__ phi, float inv_dt,
                             float scale, ThetaK th) {
  if (L.g.dim == 3) k_build_st_A_dim<3>(L, level, fine, d, phi, inv_dt, scale, th);
  else k_build_st_A_dim<2>(L, level, fine, d, phi, inv_dt, scale, th);
}

}  // namespace mg
