// The coarse V-cycle of the fused path: every level from lc down in ONE
// thread block with all grids in shared memory.
#pragma once
#include "mg_fused.cuh"

namespace mg {

// ---------------------------------------------------------------------------
// k_coarse: the coarse V-cycle in one thread block
// ---------------------------------------------------------------------------

constexpr int kCoarseThreads = 512;
constexpr int kBottomPerThread = 4;  // cached bottom cells per colour and thread

struct CoarseArgs {
  int dim, nlev, pre_post, bottom;
  int n[kMaxLevels][3];     // shapes of the levels handled (lc .. L-1); 2D: (n0, n1, 1)
  int off[kMaxLevels];      // cell offset of each level inside the shared arrays
  float s[kMaxLevels];      // kappa * s_l
  const int8_t* type[kMaxLevels];
  const void* Ad[kMaxLevels];
  const void* r0;           // r of level lc (float if r_f32)
  void* z0;                 // z of level lc (written)
  int r_f32;
  float rho, pi;            // per-level restriction / prolongation factors
  const Control* ctl;
  int total;                // total cells
};

// Cell of colour `phase` number j of a level (row-major rows, every other
// cell along the last axis).  Returns false when j runs past a short row.
__device__ __forceinline__ bool colour_cell(const int n[3], int dim, int j, int phase, int c[3]) {
  const int nl = dim == 3 ? n[2] : n[1];
  const int half = (nl + 1) >> 1;
  const int row = j / half, k = j - row * half;
  if (dim == 3) {
    c[0] = row / n[1];
    c[1] = row - c[0] * n[1];
    c[2] = 2 * k + ((phase - c[0] - c[1]) & 1);
    return c[2] < n[2];
  }
  c[0] = row;
  c[1] = 2 * k + ((phase - c[0]) & 1);
  c[2] = 0;
  return c[1] < n[1];
}

__device__ __forceinline__ int colour_count(const int n[3], int dim) {
  const int nl = dim == 3 ? n[2] : n[1];
  return (n[0] * n[1] * n[2] / nl) * ((nl + 1) >> 1);
}

// Neighbour sum of cell (c0,c1,c2) of level l with FLUID checks (the coarse
// kernel keeps unmasked z: non-FLUID z reaches finer levels by prolongation).
__device__ __forceinline__ float coarse_nsum(const CoarseArgs& A, int l, const int c[3], int g, const float* sz,
                                             const int8_t* sl) {
  const int n0 = A.n[l][0], n1 = A.n[l][1], n2 = A.n[l][2];
  const float ms = -A.s[l];
  const int s0 = n1 * n2, s1 = n2;
  float ret = 0.0f;
  float l0 = (c[0] > 0 && sl[g - s0] == FLUID) ? __fmul_rn(ms, sz[g - s0]) : 0.0f;
  float h0 = (c[0] + 1 < n0 && sl[g + s0] == FLUID) ? __fmul_rn(ms, sz[g + s0]) : 0.0f;
  ret = __fadd_rn(ret, __fadd_rn(l0, h0));
  float l1 = (c[1] > 0 && sl[g - s1] == FLUID) ? __fmul_rn(ms, sz[g - s1]) : 0.0f;
  float h1 = (c[1] + 1 < n1 && sl[g + s1] == FLUID) ? __fmul_rn(ms, sz[g + s1]) : 0.0f;
  ret = __fadd_rn(ret, __fadd_rn(l1, h1));
  if (A.dim == 3) {
    float l2 = (c[2] > 0 && sl[g - 1] == FLUID) ? __fmul_rn(ms, sz[g - 1]) : 0.0f;
    float h2 = (c[2] + 1 < n2 && sl[g + 1] == FLUID) ? __fmul_rn(ms, sz[g + 1]) : 0.0f;
    ret = __fadd_rn(ret, __fadd_rn(l2, h2));
  }
  return ret;
}

__device__ void coarse_smooth(const CoarseArgs& A, int l, int phase, float* sz, const float* sr, const float* sa,
                              const int8_t* sl) {
  const int cnt = colour_count(A.n[l], A.dim);
  for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
    int c[3];
    if (!colour_cell(A.n[l], A.dim, j, phase, c)) continue;
    const int g = A.off[l] + (c[0] * A.n[l][1] + c[1]) * A.n[l][2] + c[2];
    if (sl[g] != FLUID) continue;
    sz[g] = __fdiv_rn(__fsub_rn(sr[g], coarse_nsum(A, l, c, g, sz, sl)), sa[g]);
  }
}

// Shared layout: z[total] f32, r[total] f32, Ad[total] f32, type[total] i8.
template <typename ST>
__global__ void __launch_bounds__(kCoarseThreads) k_coarse(CoarseArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  float* sz = (float*)smem;
  float* sr = sz + A.total;
  float* sa = sr + A.total;
  int8_t* sl = (int8_t*)(sa + A.total);
  const float sigma = A.r_f32 ? (float)A.ctl->scale_r : 1.0f;
  for (int l = 0; l < A.nlev; ++l) {
    const int cnt = A.n[l][0] * A.n[l][1] * A.n[l][2];
    const int o = A.off[l];
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
      sl[o + i] = A.type[l][i];
      sa[o + i] = to_f<ST>(((const ST*)A.Ad[l])[i]);
      sz[o + i] = 0.0f;
      sr[o + i] = l == 0 ? load_r<ST>(A.r0, i, A.r_f32, sigma) : 0.0f;
    }
  }
  __syncthreads();
  const int L = A.nlev;
  for (int l = 0; l < L - 1; ++l) {
    for (int i = 0; i < A.pre_post; ++i) {
      coarse_smooth(A, l, 0, sz, sr, sa, sl);
      __syncthreads();
      coarse_smooth(A, l, 1, sz, sr, sa, sl);
      __syncthreads();
    }
    // restrict: coarse r = rho * sum over FLUID children (lexicographic order)
    const int m1 = A.n[l + 1][1], m2 = A.n[l + 1][2];
    const int cnt = A.n[l + 1][0] * m1 * m2;
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
      const int c2 = i % m2, t = i / m2, c1 = t % m1, c0 = t / m1;
      float acc = 0.0f;
      for (int o0 = 0; o0 < 2; ++o0)
        for (int o1 = 0; o1 < 2; ++o1)
          for (int o2 = 0; o2 < (A.dim == 3 ? 2 : 1); ++o2) {
            const int f[3] = {2 * c0 + o0, 2 * c1 + o1, A.dim == 3 ? 2 * c2 + o2 : 0};
            const int g = A.off[l] + (f[0] * A.n[l][1] + f[1]) * A.n[l][2] + f[2];
            if (sl[g] == FLUID) {
              const float Az = __fadd_rn(__fmul_rn(sa[g], sz[g]), coarse_nsum(A, l, f, g, sz, sl));
              acc = __fadd_rn(acc, __fsub_rn(sr[g], Az));
            }
          }
      sr[A.off[l + 1] + i] = __fmul_rn(A.rho, acc);
    }
    __syncthreads();
  }
  // bottom sweeps (mgpcg.py:136-142)
  const int nh = A.bottom / 2;
  const int lb = L - 1;
  const int cntb = colour_count(A.n[lb], A.dim);
  if (cntb <= kBottomPerThread * kCoarseThreads) {
    // cache each owned cell's index, r, Adiag and neighbour-coupling mask in
    // registers: the 2*bottom half sweeps then touch shared memory only for z
    int gi[2][kBottomPerThread], mk[2][kBottomPerThread];
    float rr[2][kBottomPerThread], aa[2][kBottomPerThread];
    const int n0 = A.n[lb][0], n1 = A.n[lb][1], n2 = A.n[lb][2];
    const int s0 = n1 * n2, s1 = n2;
#pragma unroll
    for (int ph = 0; ph < 2; ++ph) {
#pragma unroll
      for (int k = 0; k < kBottomPerThread; ++k) {
        const int j = threadIdx.x + k * kCoarseThreads;
        int c[3];
        gi[ph][k] = -1;
        mk[ph][k] = 0;
        rr[ph][k] = 0.0f;
        aa[ph][k] = 1.0f;
        if (j < cntb && colour_cell(A.n[lb], A.dim, j, ph, c)) {
          const int g = A.off[lb] + (c[0] * n1 + c[1]) * n2 + c[2];
          if (sl[g] == FLUID) {
            int m = 0;
            if (c[0] > 0 && sl[g - s0] == FLUID) m |= 1;
            if (c[0] + 1 < n0 && sl[g + s0] == FLUID) m |= 2;
            if (c[1] > 0 && sl[g - s1] == FLUID) m |= 4;
            if (c[1] + 1 < n1 && sl[g + s1] == FLUID) m |= 8;
            if (A.dim == 3 && c[2] > 0 && sl[g - 1] == FLUID) m |= 16;
            if (A.dim == 3 && c[2] + 1 < n2 && sl[g + 1] == FLUID) m |= 32;
            gi[ph][k] = g;
            mk[ph][k] = m;
            rr[ph][k] = sr[g];
            aa[ph][k] = sa[g];
          }
        }
      }
    }
    const float ms = -A.s[lb];
    for (int i = 0; i < 2 * nh; ++i) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int ph = i < nh ? h : 1 - h;
#pragma unroll
        for (int k = 0; k < kBottomPerThread; ++k) {
          const int g = ph ? gi[1][k] : gi[0][k];
          const int m = ph ? mk[1][k] : mk[0][k];
          if (g >= 0) {
            float ret = 0.0f;
            float l0 = (m & 1) ? __fmul_rn(ms, sz[g - s0]) : 0.0f;
            float h0 = (m & 2) ? __fmul_rn(ms, sz[g + s0]) : 0.0f;
            ret = __fadd_rn(ret, __fadd_rn(l0, h0));
            float l1 = (m & 4) ? __fmul_rn(ms, sz[g - s1]) : 0.0f;
            float h1 = (m & 8) ? __fmul_rn(ms, sz[g + s1]) : 0.0f;
            ret = __fadd_rn(ret, __fadd_rn(l1, h1));
            if (A.dim == 3) {
              float l2 = (m & 16) ? __fmul_rn(ms, sz[g - 1]) : 0.0f;
              float h2 = (m & 32) ? __fmul_rn(ms, sz[g + 1]) : 0.0f;
              ret = __fadd_rn(ret, __fadd_rn(l2, h2));
            }
            const float r_ = ph ? rr[1][k] : rr[0][k];
            const float a_ = ph ? aa[1][k] : aa[0][k];
            sz[g] = __fdiv_rn(__fsub_rn(r_, ret), a_);
          }
        }
        __syncthreads();
      }
    }
  } else {
    for (int i = 0; i < 2 * nh; ++i) {
      for (int h = 0; h < 2; ++h) {
        coarse_smooth(A, lb, i < nh ? h : 1 - h, sz, sr, sa, sl);
        __syncthreads();
      }
    }
  }
  for (int l = L - 2; l >= 0; --l) {
    const int cnt = A.n[l][0] * A.n[l][1] * A.n[l][2];
    const int n1 = A.n[l][1], n2 = A.n[l][2];
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
      const int c2 = i % n2, t = i / n2, c1 = t % n1, c0 = t / n1;
      const int gc = A.off[l + 1] + ((c0 >> 1) * A.n[l + 1][1] + (c1 >> 1)) * A.n[l + 1][2] + (c2 >> 1);
      sz[A.off[l] + i] = __fadd_rn(sz[A.off[l] + i], __fmul_rn(A.pi, sz[gc]));
    }
    __syncthreads();
    for (int i = 0; i < A.pre_post; ++i) {
      coarse_smooth(A, l, 1, sz, sr, sa, sl);
      __syncthreads();
      coarse_smooth(A, l, 0, sz, sr, sa, sl);
      __syncthreads();
    }
  }
  const int cnt0 = A.n[0][0] * A.n[0][1] * A.n[0][2];
  for (int i = threadIdx.x; i < cnt0; i += blockDim.x) ((ST*)A.z0)[i] = from_f<ST>(sz[i]);
}

}  // namespace mg
