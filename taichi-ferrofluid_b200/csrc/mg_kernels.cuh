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

// k_build_pressure_b for a compile-time dim (its per-axis arrays and the level's
// extents indexed by constants, so nothing is kept in local memory).
template <int DIM>
__device__ __forceinline__ void k_build_pressure_b_dim(Level L, const float* __restrict__ v0, const float* __restrict__ v1,
                                   const float* __restrict__ v2, const float* __restrict__ phi,
                                   float p0, float sA, float sB, int ghost, float clamp, float* b) {
  const float* vel[3] = {v0, v1, v2};
  for (long long i = gtid(); i < L.g.count; i += gstride()) {
    if (L.type[i] != FLUID) continue;
    int c[3];
    L.g.coords(i, c);
    float bi = b[i];
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
      int cp[3] = {c[0], c[1], c[2]};
      cp[k] += 1;
      float a = vel_at(vel[k], L.g, k, c[0], c[1], c[2]);
      float bb = vel_at(vel[k], L.g, k, cp[0], cp[1], cp[2]);
      bi = __fadd_rn(bi, __fsub_rn(a, bb));
    }
    bi = __fmul_rn(bi, sB);
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
#pragma unroll
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

// PressureProjectStrategy.build_b_kernel (pressure_project.py:15-39).  The two
// passes of the reference touch only b[I] of the cell itself, so one thread
// runs pass 1 then pass 2 for its cell with the same operation order.
__global__ void k_build_pressure_b(Level L, const float* __restrict__ v0, const float* __restrict__ v1,
                                   const float* __restrict__ v2, const float* __restrict__ phi,
                                   float p0, float sA, float sB, int ghost, float clamp, float* b) {
  if (L.g.dim == 3) k_build_pressure_b_dim<3>(L, v0, v1, v2, phi, p0, sA, sB, ghost, clamp, b);
  else k_build_pressure_b_dim<2>(L, v0, v1, v2, phi, p0, sA, sB, ghost, clamp, b);
}

// k_build_pressure_A for a compile-time dim (its per-axis arrays and the level's
// extents indexed by constants, so nothing is kept in local memory).
template <int DIM>
__device__ __forceinline__ void k_build_pressure_A_dim(Level L, int level, const float* __restrict__ phi, float sA,
                                   int ghost, float clamp) {
  for (long long i = gtid(); i < L.g.count; i += gstride()) {
    if (L.type[i] != FLUID) continue;
    int c[3];
    L.g.coords(i, c);
    float d = L.Adiag[i];
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
#pragma unroll
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

// PressureProjectStrategy.build_A_kernel (pressure_project.py:45-64).
__global__ void k_build_pressure_A(Level L, int level, const float* __restrict__ phi, float sA,
                                   int ghost, float clamp) {
  if (L.g.dim == 3) k_build_pressure_A_dim<3>(L, level, phi, sA, ghost, clamp);
  else k_build_pressure_A_dim<2>(L, level, phi, sA, ghost, clamp);
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
  long long row;
  int k;
  if (g.count < (1LL << 31)) {  // 32-bit division (a 64-bit one is a long emulated sequence)
    const unsigned ur = (unsigned)j / (unsigned)half;
    row = ur;
    k = (int)((unsigned)j - ur * (unsigned)half);
  } else {
    row = j / half;
    k = (int)(j - row * half);
  }
  int c[3];
  int rowsum;
  if (g.dim == 3) {
    c[0] = g.count < (1LL << 31) ? (int)((unsigned)row / (unsigned)g.n[1]) : (int)(row / g.n[1]);
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

// The stencil data of one 4-cell group along the fastest axis of a 3D f32
// level (row (i0, i1), cells x .. x+3, x a multiple of 4): z and its six
// neighbour directions, the couplings, r and Adiag, with 16-byte loads.
struct Group4 {
  float Z[4], Z0l[4], Z0h[4], Z1l[4], Z1h[4], zxl, zxh;
  float A0l[4], A0h[4], A1l[4], A1h[4], A2c[4], a2l;
  float R[4], D[4];
  bool h0l, h0h, h1l, h1h;
  int x, n2;
};

__device__ __forceinline__ void unpack4(const float4 v, float o[4]) {
  o[0] = v.x;
  o[1] = v.y;
  o[2] = v.z;
  o[3] = v.w;
}

__device__ __forceinline__ void load_group4(const Level& L, const float* z, int i0, int i1, int x, Group4& g) {
  const int n0 = L.g.n[0], n1 = L.g.n[1], n2 = L.g.n[2];
  const long long s0 = (long long)n1 * n2;
  const int s1 = n2;
  const long long idx = ((long long)i0 * n1 + i1) * n2 + x;
  const float4 f0 = make_float4(0.f, 0.f, 0.f, 0.f);
  g.x = x;
  g.n2 = n2;
  g.h0l = i0 > 0;
  g.h0h = i0 + 1 < n0;
  g.h1l = i1 > 0;
  g.h1h = i1 + 1 < n1;
  unpack4(*reinterpret_cast<const float4*>(z + idx), g.Z);
  unpack4(g.h0l ? *reinterpret_cast<const float4*>(z + idx - s0) : f0, g.Z0l);
  unpack4(g.h0h ? *reinterpret_cast<const float4*>(z + idx + s0) : f0, g.Z0h);
  unpack4(g.h1l ? *reinterpret_cast<const float4*>(z + idx - s1) : f0, g.Z1l);
  unpack4(g.h1h ? *reinterpret_cast<const float4*>(z + idx + s1) : f0, g.Z1h);
  g.zxl = x > 0 ? z[idx - 1] : 0.0f;
  g.zxh = x + 4 < n2 ? z[idx + 4] : 0.0f;
  unpack4(g.h0l ? __ldg(reinterpret_cast<const float4*>(L.Ax[0] + idx - s0)) : f0, g.A0l);
  unpack4(__ldg(reinterpret_cast<const float4*>(L.Ax[0] + idx)), g.A0h);
  unpack4(g.h1l ? __ldg(reinterpret_cast<const float4*>(L.Ax[1] + idx - s1)) : f0, g.A1l);
  unpack4(__ldg(reinterpret_cast<const float4*>(L.Ax[1] + idx)), g.A1h);
  unpack4(__ldg(reinterpret_cast<const float4*>(L.Ax[2] + idx)), g.A2c);
  g.a2l = x > 0 ? __ldg(L.Ax[2] + idx - 1) : 0.0f;
  unpack4(__ldg(reinterpret_cast<const float4*>((const float*)L.r + idx)), g.R);
  unpack4(__ldg(reinterpret_cast<const float4*>(L.Adiag + idx)), g.D);
}

// nbr_sum_f32 of the group's cell e, in its order (axis 0, 1, 2; lower + upper).
__device__ __forceinline__ float group4_nsum(const Group4& g, int e) {
  float ret = 0.0f;
  ret = __fadd_rn(ret, __fadd_rn(g.h0l ? __fmul_rn(g.A0l[e], g.Z0l[e]) : 0.0f,
                                 g.h0h ? __fmul_rn(g.A0h[e], g.Z0h[e]) : 0.0f));
  ret = __fadd_rn(ret, __fadd_rn(g.h1l ? __fmul_rn(g.A1l[e], g.Z1l[e]) : 0.0f,
                                 g.h1h ? __fmul_rn(g.A1h[e], g.Z1h[e]) : 0.0f));
  const float lo = g.x + e > 0 ? __fmul_rn(e == 0 ? g.a2l : g.A2c[e - 1], e == 0 ? g.zxl : g.Z[e - 1]) : 0.0f;
  const float hi = g.x + e + 1 < g.n2 ? __fmul_rn(g.A2c[e], e == 3 ? g.zxh : g.Z[e + 1]) : 0.0f;
  return __fadd_rn(ret, __fadd_rn(lo, hi));
}

// Row (axis 0 and 1) and first column of 4-cell group q of a 3D level with
// q2 groups a row: 32-bit division where the level has fewer than 2^31
// groups (a 64-bit integer division is a long emulated sequence).
__device__ __forceinline__ void group4_coords(long long q, int q2, int n1, long long groups, long long& row, int& x,
                                              int& i1, int& i0) {
  if (groups < (1LL << 31)) {
    const unsigned uq = (unsigned)q, ur = uq / (unsigned)q2, u0 = ur / (unsigned)n1;
    row = ur;
    x = (int)(uq - ur * (unsigned)q2) * 4;
    i1 = (int)(ur - u0 * (unsigned)n1);
    i0 = (int)u0;
    return;
  }
  row = q / q2;
  x = (int)(q - row * q2) * 4;
  i1 = (int)(row % n1);
  i0 = (int)(row / n1);
}

// smooth(l, phase) on a whole-domain level (every cell FLUID with a nonzero
// diagonal: the stored form's levels), 3D with the fastest extent a multiple
// of 4: one thread per 4-cell group, which holds two cells of the colour.
// The same float32 operations in the same order as smooth_cell.  z of the
// other colour (all a cell's neighbours) is not written during the half
// sweep, so the group's loads see final values; each thread stores only its
// two cells.
__global__ void k_smooth_w4(Level L, int phase) {
  pdl_enter();
  const int n1 = L.g.n[1], n2 = L.g.n[2];
  const int q2 = n2 >> 2;
  const long long groups = L.g.count >> 2;
  float* z = (float*)L.z;
  for (long long q = gtid(); q < groups; q += gstride()) {
    long long row;
    int x, i1, i0;
    group4_coords(q, q2, n1, groups, row, x, i1, i0);
    const int e0 = (phase - i0 - i1 - x) & 1;  // first cell of the colour in the group
    Group4 g;
    load_group4(L, z, i0, i1, x, g);
    float out[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float v = 0.0f;
#pragma unroll
      for (int ee = 0; ee < 2; ++ee) {  // unrolled over both values of e0
        const int e = ee + 2 * h;
        if (ee == e0) v = div_pos(__fsub_rn(g.R[e], group4_nsum(g, e)), g.D[e]);
      }
      out[h] = v;
    }
    const long long idx = row * n2 + x;
    z[idx + e0] = out[0];
    z[idx + e0 + 2] = out[1];
  }
}

// The first half sweep of pre-smoothing (colour 0 from z = 0) on a
// whole-domain level of 4-cell groups: with every neighbour 0 the neighbour
// sum is +0, so z = (r - 0) / Adiag = r / Adiag on colour 0 (the same float32
// value, -0 included), and z = 0 on colour 1 - the z.fill(0) before the sweep
// written in the same pass.
__global__ void k_smooth_first_w4(Level L) {
  pdl_enter();
  const int n1 = L.g.n[1], n2 = L.g.n[2];
  const int q2 = n2 >> 2;
  const long long groups = L.g.count >> 2;
  float* z = (float*)L.z;
  for (long long q = gtid(); q < groups; q += gstride()) {
    long long row;
    int x, i1, i0;
    group4_coords(q, q2, n1, groups, row, x, i1, i0);
    const int e0 = (0 - i0 - i1 - x) & 1;  // first colour-0 cell of the group
    float R[4], D[4];
    unpack4(__ldg(reinterpret_cast<const float4*>((const float*)L.r) + q), R);
    unpack4(__ldg(reinterpret_cast<const float4*>(L.Adiag) + q), D);
    float v[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int e = 0; e < 4; ++e)
      if (((e - e0) & 1) == 0) v[e] = div_pos(__fsub_rn(R[e], 0.0f), D[e]);
    reinterpret_cast<float4*>(z)[q] = make_float4(v[0], v[1], v[2], v[3]);
  }
}

// restrict(l) as k_restrict for a whole-domain fine level halving exactly
// onto the coarse one, 3D, fine fastest extent a multiple of 4: one thread
// per pair of coarse cells along the fastest axis, i.e. one 4-cell fine group
// in each of the 2 x 2 fine rows; children summed in k_restrict's
// lexicographic order.
__global__ void k_restrict_w4(Level F, Level C) {
  pdl_enter();
  const float* zf = (const float*)F.z;
  const int cn1 = C.g.n[1], cn2 = C.g.n[2];
  const int pr = cn2 >> 1;  // coarse pairs per coarse row
  const long long pairs = C.g.count >> 1;
  for (long long t = gtid(); t < pairs; t += gstride()) {
    long long crow;
    int cx, c1, c0;
    group4_coords(t, pr, cn1, pairs, crow, cx, c1, c0);
    cx >>= 1;  // pairs, not groups of 4: the first coarse column of the pair is 2 (t mod pr)
    float acc[2] = {0.0f, 0.0f};
#pragma unroll
    for (int o0 = 0; o0 < 2; ++o0)
#pragma unroll
      for (int o1 = 0; o1 < 2; ++o1) {
        Group4 g;
        load_group4(F, zf, 2 * c0 + o0, 2 * c1 + o1, 2 * cx, g);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const float Az = __fadd_rn(__fmul_rn(g.D[e], g.Z[e]), group4_nsum(g, e));
          acc[e >> 1] = __fadd_rn(acc[e >> 1], __fsub_rn(g.R[e], Az));
        }
      }
    const long long ic = crow * cn2 + cx;
    ((float*)C.r)[ic] = acc[0];
    ((float*)C.r)[ic + 1] = acc[1];
    ((float*)C.z)[ic] = 0.0f;
    ((float*)C.z)[ic + 1] = 0.0f;
  }
}

// prolongate(l) as k_prolongate for a fine level halving exactly onto the
// coarse one, 3D, fine fastest extent a multiple of 4: one 4-cell group per
// thread, two coarse values.
__global__ void k_prolongate4(Level F, Level C) {
  pdl_enter();
  float* zf = (float*)F.z;
  const float* zc = (const float*)C.z;
  const int n1 = F.g.n[1], n2 = F.g.n[2], q2 = n2 >> 2;
  const long long groups = F.g.count >> 2;
  for (long long q = gtid(); q < groups; q += gstride()) {
    long long row;
    int x, i1, i0;
    group4_coords(q, q2, n1, groups, row, x, i1, i0);
    const long long ic = C.g.index(i0 >> 1, i1 >> 1, x >> 1);
    const float a = zc[ic], b = zc[ic + 1];
    float4 v = reinterpret_cast<float4*>(zf)[q];
    v.x = __fadd_rn(v.x, a);
    v.y = __fadd_rn(v.y, a);
    v.z = __fadd_rn(v.z, b);
    v.w = __fadd_rn(v.w, b);
    reinterpret_cast<float4*>(zf)[q] = v;
  }
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
