// Reference-structured kernels: one CUDA kernel per Taichi kernel of
// mgpcg.py and pressure_project.py, with the reference's operation order.
// They back the per-kernel C entry points (mg_smooth, mg_restrict, ...) used by
// the parity tests, and the stored-coefficient ("generic") operator form of
// the solve.  The label-uniform fast path lives in mg_fused.cuh.
#pragma once
#include "mg_common.cuh"

namespace mg {

__device__ __forceinline__ long long gtid() { return (long long)blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ long long gstride() { return (long long)gridDim.x * blockDim.x; }

// grid_type[0].copy_from(cell_type) (mgpcg.py:81)
__global__ void k_set_cell_type(const int32_t* __restrict__ in, int8_t* __restrict__ out, long long n) {
  for (long long i = gtid(); i < n; i += gstride()) out[i] = (int8_t)in[i];
}

// init_gridtype (mgpcg.py:46-60): AIR if any child is AIR, else FLUID if any
// child is FLUID, else SOLID.
__global__ void k_init_gridtype(Level F, Level C) {
  for (long long i = gtid(); i < C.g.count; i += gstride()) {
    int c[3];
    C.g.coords(i, c);
    int tot_fluid = 0, tot_air = 0;
    const int o2max = C.g.dim == 3 ? 2 : 1;
    for (int o0 = 0; o0 < 2; ++o0)
      for (int o1 = 0; o1 < 2; ++o1)
        for (int o2 = 0; o2 < o2max; ++o2) {
          int attr = F.type[F.g.index(2 * c[0] + o0, 2 * c[1] + o1, C.g.dim == 3 ? 2 * c[2] + o2 : 0)];
          if (attr == AIR) tot_air++;
          else if (attr == FLUID) tot_fluid++;
        }
    C.type[i] = tot_air > 0 ? AIR : (tot_fluid > 0 ? FLUID : SOLID);
  }
}

__device__ __forceinline__ int8_t nb_type(const Level& L, long long idx, const int c[3], int axis, int s) {
  int v = c[axis] + s;
  if (v < 0 || v >= L.g.n[axis]) return SOLID;  // rule H1
  return L.type[idx + s * L.g.stride(axis)];
}

// Face velocity of axis k at cell coordinates c (shape res + e_k).
__device__ __forceinline__ float vel_at(const float* v, const Geom& g, int k, int c0, int c1, int c2) {
  int n1 = g.n[1] + (k == 1), n2 = g.dim == 3 ? g.n[2] + (k == 2) : 1;
  return v[((long long)c0 * n1 + c1) * n2 + c2];
}

// PressureProjectStrategy.build_b_kernel (pressure_project.py:15-39).  The two
// passes of the reference touch only b[I] of the cell itself, so one thread
// runs pass 1 then pass 2 for its cell with the same operation order.
__global__ void k_build_pressure_b(Level L, const float* __restrict__ v0, const float* __restrict__ v1,
                                   const float* __restrict__ v2, const float* __restrict__ phi,
                                   float p0, float sA, float sB, int ghost, float clamp, float* b) {
  const float* vel[3] = {v0, v1, v2};
  for (long long i = gtid(); i < L.g.count; i += gstride()) {
    if (L.type[i] != FLUID) continue;
    int c[3];
    L.g.coords(i, c);
    float bi = b[i];
    for (int k = 0; k < L.g.dim; ++k) {
      int cp[3] = {c[0], c[1], c[2]};
      cp[k] += 1;
      float a = vel_at(vel[k], L.g, k, c[0], c[1], c[2]);
      float bb = vel_at(vel[k], L.g, k, cp[0], cp[1], cp[2]);
      bi = __fadd_rn(bi, __fsub_rn(a, bb));
    }
    bi = __fmul_rn(bi, sB);
    for (int k = 0; k < L.g.dim; ++k) {
      for (int s = -1; s <= 1; s += 2) {
        int8_t nt = nb_type(L, i, c, k, s);
        if (nt == SOLID) {
          if (s < 0) {
            bi = __fsub_rn(bi, __fmul_rn(sB, __fsub_rn(vel_at(vel[k], L.g, k, c[0], c[1], c[2]), 0.0f)));
          } else {
            int cp[3] = {c[0], c[1], c[2]};
            cp[k] += 1;
            bi = __fadd_rn(bi, __fmul_rn(sB, __fsub_rn(vel_at(vel[k], L.g, k, cp[0], cp[1], cp[2]), 0.0f)));
          }
        } else if (nt == AIR) {
          if (ghost) {
            float phin = phi[i + s * L.g.stride(k)];
            float cc = __fdiv_rn(__fsub_rn(phi[i], phin), phi[i]);
            bi = __fadd_rn(bi, __fmul_rn(__fmul_rn(sA, fminf(cc, clamp)), p0));
          } else {
            bi = __fadd_rn(bi, __fmul_rn(sA, p0));
          }
        }
      }
    }
    b[i] = bi;
  }
}

// PressureProjectStrategy.build_A_kernel (pressure_project.py:45-64).
__global__ void k_build_pressure_A(Level L, int level, const float* __restrict__ phi, float sA,
                                   int ghost, float clamp) {
  for (long long i = gtid(); i < L.g.count; i += gstride()) {
    if (L.type[i] != FLUID) continue;
    int c[3];
    L.g.coords(i, c);
    float d = L.Adiag[i];
    for (int k = 0; k < L.g.dim; ++k) {
      for (int s = -1; s <= 1; s += 2) {
        int8_t nt = nb_type(L, i, c, k, s);
        if (nt == FLUID) {
          d = __fadd_rn(d, sA);
          if (s > 0) L.Ax[k][i] = -sA;
        } else if (nt == AIR) {
          if (ghost && level == 0) {
            float phin = phi[i + s * L.g.stride(k)];
            float cc = __fdiv_rn(__fsub_rn(phi[i], phin), phi[i]);
            d = __fadd_rn(d, __fmul_rn(sA, fminf(cc, clamp)));
          } else {
            d = __fadd_rn(d, sA);
          }
        }
      }
    }
    L.Adiag[i] = d;
  }
}

// b += c * src (or += c) on FLUID cells (volume_control.py:33-37).
__global__ void k_add_rhs(Level L, float* b, const float* __restrict__ src, float c) {
  for (long long i = gtid(); i < L.g.count; i += gstride()) {
    if (L.type[i] != FLUID) continue;
    b[i] = __fadd_rn(b[i], src ? __fmul_rn(c, src[i]) : c);
  }
}

// ---- generic (stored-coefficient) V-cycle kernels, f32 ---------------------

// smooth(l, phase) (mgpcg.py:104-109).  One thread per cell of the colour:
// along the last axis the colour's cells are every other cell.
__device__ __forceinline__ void smooth_cell(const Level& L, long long j, int phase) {
  const Geom& g = L.g;
  // j enumerates cells of one colour: (row, k) with the last axis index
  // x = 2k + ((phase - rowsum) & 1); a row is (i0, i1) in 3D or (i0) in 2D.
  const int nl = g.dim == 3 ? g.n[2] : g.n[1];
  const int half = (nl + 1) >> 1;
  long long row = j / half;
  int k = (int)(j - row * half);
  int c[3];
  int rowsum;
  if (g.dim == 3) {
    c[0] = (int)(row / g.n[1]);
    c[1] = (int)(row - (long long)c[0] * g.n[1]);
    rowsum = c[0] + c[1];
    c[2] = 2 * k + ((phase - rowsum) & 1);
    if (c[2] >= g.n[2]) return;
  } else {
    c[0] = (int)row;
    rowsum = c[0];
    c[1] = 2 * k + ((phase - rowsum) & 1);
    c[2] = 0;
    if (c[1] >= g.n[1]) return;
  }
  long long idx = g.index(c[0], c[1], c[2]);
  if (L.type[idx] != FLUID) return;
  float* z = (float*)L.z;
  const float* r = (const float*)L.r;
  z[idx] = __fdiv_rn(__fsub_rn(r[idx], nbr_sum_f32(L, z, idx, c)), L.Adiag[idx]);
}

__device__ __forceinline__ long long colour_cells(const Geom& g) {
  const int nl = g.dim == 3 ? g.n[2] : g.n[1];
  return g.count / nl * ((nl + 1) >> 1);
}

__global__ void k_smooth(Level L, int phase) {
  pdl_enter();
  const long long n = colour_cells(L.g);
  for (long long j = gtid(); j < n; j += gstride()) smooth_cell(L, j, phase);
}

// restrict(l) (mgpcg.py:111-118) as a gather: coarse r = 0 + sum of the FLUID
// children's (r - (Adiag z + nbr_sum)) in lexicographic child order.  Also
// zeroes the coarse z (the r[l+1].fill(0), z[l+1].fill(0) of mgpcg.py:132-133).
__global__ void k_restrict(Level F, Level C) {
  pdl_enter();
  const float* zf = (const float*)F.z;
  const float* rf = (const float*)F.r;
  for (long long ic = gtid(); ic < C.g.count; ic += gstride()) {
    int cc[3];
    C.g.coords(ic, cc);
    float acc = 0.0f;
    const int o2max = F.g.dim == 3 ? 2 : 1;
    for (int o0 = 0; o0 < 2; ++o0)
      for (int o1 = 0; o1 < 2; ++o1)
        for (int o2 = 0; o2 < o2max; ++o2) {
          int c[3] = {2 * cc[0] + o0, 2 * cc[1] + o1, F.g.dim == 3 ? 2 * cc[2] + o2 : 0};
          long long i = F.g.index(c[0], c[1], c[2]);
          if (F.type[i] == FLUID) {
            float Az = __fmul_rn(F.Adiag[i], zf[i]);
            Az = __fadd_rn(Az, nbr_sum_f32(F, zf, i, c));
            acc = __fadd_rn(acc, __fsub_rn(rf[i], Az));
          }
        }
    ((float*)C.r)[ic] = acc;
    ((float*)C.z)[ic] = 0.0f;
  }
}

// prolongate(l) (mgpcg.py:120-123): z[l][I] += z[l+1][I // 2], every cell.
__global__ void k_prolongate(Level F, Level C) {
  pdl_enter();
  float* zf = (float*)F.z;
  const float* zc = (const float*)C.z;
  for (long long i = gtid(); i < F.g.count; i += gstride()) {
    int c[3];
    F.g.coords(i, c);
    zf[i] = __fadd_rn(zf[i], zc[C.g.index(c[0] >> 1, c[1] >> 1, c[2] >> 1)]);
  }
}

// The bottom solve of v_cycle (mgpcg.py:136-142) in ONE thread block: nhalf
// sweeps in colour order (0, 1) then nhalf in order (1, 0), block-synchronised
// between half sweeps.  Used for levels small enough for one block.
__global__ void k_bottom(Level L, int nhalf) {
  pdl_enter();
  const long long n = colour_cells(L.g);
  for (int it = 0; it < 2 * nhalf; ++it) {
    for (int h = 0; h < 2; ++h) {
      int phase = it < nhalf ? h : 1 - h;
      for (long long j = threadIdx.x; j < n; j += blockDim.x) smooth_cell(L, j, phase);
      __syncthreads();
    }
  }
}

}  // namespace mg
