// The coarse V-cycle of the fused path: every level from lc down in ONE
// thread block with all grids in shared memory.
#pragma once
#include <type_traits>

#include "mg_fused.cuh"

namespace mg {

// ---------------------------------------------------------------------------
// k_coarse: the coarse V-cycle in one thread block
// ---------------------------------------------------------------------------
//
// Shared memory, per level, a PADDED grid (one ring of cells around it) of
//   zm: z masked - the value on FLUID cells, 0 on every other cell and on the
//       ring, so a neighbour term is (-s) * zm for every neighbour (the same
//       float32 result as the reference's Ax * z, see k_sweep);
//   sr: r on FLUID cells; on non-FLUID cells the UNMASKED z, which the
//       smoother never touches but prolongation carries to the finer level
//       (mgpcg.py:120-123 adds to every cell); their r is never read;
//   sa: Adiag (nonzero exactly on FLUID cells; mg_plan_prepare checks it);
//   sx: (STO, the whole-domain stored form) the dim coupling arrays Ax[k],
//       0 on the ring, so a neighbour outside a level reads as z = 0, Ax = 0.

// Cached bottom cells per colour and thread, and the block size (compile-time
// tuning constants).
#ifndef MG_BOTTOM_CELLS_PER_THREAD
#define MG_BOTTOM_CELLS_PER_THREAD 1  // 8 warps for 8^3: 37 vs 48 us a V-cycle at 128^3 (2 cells)
#endif
#ifndef MG_COARSE_THREADS
#define MG_COARSE_THREADS 1024
#endif
constexpr int kBottomPerThread = MG_BOTTOM_CELLS_PER_THREAD;
constexpr int kCoarseThreads = MG_COARSE_THREADS;

struct CoarseArgs {
  int dim, nlev, pre_post, bottom;
  int n[kMaxLevels][3];     // shapes of the levels handled (lc .. L-1); 2D: (n0, n1, 1)
  int off[kMaxLevels];      // offset of each PADDED level inside the shared arrays
  float s[kMaxLevels];      // kappa * s_l
  const void* Ad[kMaxLevels];
  const float* Ax[kMaxLevels][3];  // STO: the stored couplings of each level
  const void* r0;           // r of level lc (float if r_f32)
  void* z0;                 // z of level lc (written)
  int r_f32;
  float rho, pi;            // per-level restriction / prolongation factors
  const Control* ctl;
  int total;                // padded cells of all levels
};

// Padded geometry of one level: P = n + 2 per axis (2D: no padding along the
// absent third axis).
struct PGeom {
  int n0, n1, n2, P1, P2, o;   // sizes, padded strides, level offset
  float r1, r2;                // 1 / n1, 1 / n2 (rounded; cell_coords)
  int s0, s1, s2;              // neighbour strides in the padded grid
  __device__ __forceinline__ int at(int c0, int c1, int c2) const {
    return o + ((c0 + 1) * P1 + (c1 + 1)) * P2 + c2 + (P2 > 1 ? 1 : 0);
  }
};

__device__ __forceinline__ PGeom pgeom(const CoarseArgs& A, int l) {
  PGeom g;
  g.n0 = A.n[l][0];
  g.n1 = A.n[l][1];
  g.n2 = A.n[l][2];
  g.P1 = g.n1 + 2;
  g.P2 = A.dim == 3 ? g.n2 + 2 : 1;
  g.o = A.off[l];
  g.s0 = g.P1 * g.P2;
  g.s1 = g.P2;
  g.s2 = 1;
  g.r1 = 1.0f / (float)g.n1;
  g.r2 = 1.0f / (float)g.n2;
  return g;
}

// Cell i of a level as (c0, c1, c2) (2D: (c0, c1, 0)), the quotients taken
// through float reciprocals: exact for i < 2^22, since the relative error of
// (i + 0.5) * RN(1 / n), at most 2^-23, stays below the 0.5 / n that
// separates (i + 0.5) / n from an integer.
__device__ __forceinline__ void cell_coords(const PGeom& g, int dim, int i, int& c0, int& c1, int& c2) {
  if (dim == 3) {
    const int t = (int)(((float)i + 0.5f) * g.r2);
    c2 = i - t * g.n2;
    c0 = (int)(((float)t + 0.5f) * g.r1);
    c1 = t - c0 * g.n1;
  } else {
    c2 = 0;
    c0 = (int)(((float)i + 0.5f) * g.r1);
    c1 = i - c0 * g.n1;
  }
}

// j-th cell of colour `phase` (rows of the last axis, every other cell);
// exact small-integer division through float reciprocals.
__device__ __forceinline__ bool colour_cell(const PGeom& g, int dim, int j, int phase, int& c0, int& c1, int& c2) {
  const int nl = dim == 3 ? g.n2 : g.n1;
  const int half = (nl + 1) >> 1;
  const int row = (int)(((float)j + 0.5f) / (float)half);
  const int k = j - row * half;
  if (dim == 3) {
    c0 = (int)(((float)row + 0.5f) / (float)g.n1);
    c1 = row - c0 * g.n1;
    c2 = 2 * k + ((phase - c0 - c1) & 1);
    return c2 < g.n2;
  }
  c0 = row;
  c1 = 2 * k + ((phase - c0) & 1);
  c2 = 0;
  return c1 < g.n1;
}

__device__ __forceinline__ int colour_count(const PGeom& g, int dim) {
  const int nl = dim == 3 ? g.n2 : g.n1;
  return (g.n0 * g.n1 * g.n2 / nl) * ((nl + 1) >> 1);
}

// Neighbour sum (mgpcg.py:96-102) at padded index p, masked z.
__device__ __forceinline__ float csum(const float* zm, int p, const PGeom& g, int dim, float ms) {
  float ret = 0.0f;
  ret = __fadd_rn(ret, __fadd_rn(__fmul_rn(ms, zm[p - g.s0]), __fmul_rn(ms, zm[p + g.s0])));
  ret = __fadd_rn(ret, __fadd_rn(__fmul_rn(ms, zm[p - g.s1]), __fmul_rn(ms, zm[p + g.s1])));
  if (dim == 3) ret = __fadd_rn(ret, __fadd_rn(__fmul_rn(ms, zm[p - 1]), __fmul_rn(ms, zm[p + 1])));
  return ret;
}

// The neighbour sum with the stored couplings sx (dim arrays of `total`
// cells each): sum_k Ax[p-s_k][k] z[p-s_k] + Ax[p][k] z[p+s_k].
template <bool STO>
__device__ __forceinline__ float csum_t(const float* zm, const float* sx, int total, int p, const PGeom& g, int dim,
                                        float ms) {
  if constexpr (STO) {
    const float* x0 = sx;
    const float* x1 = sx + total;
    float ret = 0.0f;
    ret = __fadd_rn(ret, __fadd_rn(__fmul_rn(x0[p - g.s0], zm[p - g.s0]), __fmul_rn(x0[p], zm[p + g.s0])));
    ret = __fadd_rn(ret, __fadd_rn(__fmul_rn(x1[p - g.s1], zm[p - g.s1]), __fmul_rn(x1[p], zm[p + g.s1])));
    if (dim == 3) {
      const float* x2 = sx + 2 * total;
      ret = __fadd_rn(ret, __fadd_rn(__fmul_rn(x2[p - 1], zm[p - 1]), __fmul_rn(x2[p], zm[p + 1])));
    }
    return ret;
  } else {
    return csum(zm, p, g, dim, ms);
  }
}

// A half sweep of colour `phase` over the calling thread's own cells of
// level l, listed by padded index (-1: none, or not FLUID): the list form of
// coarse_smooth for a level whose colours have at most 2 * blockDim.x cells.
template <bool STO>
__device__ __forceinline__ void coarse_smooth_list(const CoarseArgs& A, int l, const int (&li)[2], float* zm,
                                                   const float* sr, const float* sa, const float* sx) {
  const PGeom g = pgeom(A, l);
  const float ms = -A.s[l];
  float v[2];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const int p = li[k] >= 0 ? li[k] : g.at(0, 0, 0);
    v[k] = div_pos(__fsub_rn(sr[p], csum_t<STO>(zm, sx, A.total, p, g, A.dim, ms)), sa[p]);
  }
#pragma unroll
  for (int k = 0; k < 2; ++k)
    if (li[k] >= 0) zm[li[k]] = v[k];
}

template <bool STO>
__device__ void coarse_smooth(const CoarseArgs& A, int l, int phase, float* zm, const float* sr, const float* sa,
                              const float* sx) {
  const PGeom g = pgeom(A, l);
  const float ms = -A.s[l];
  const int cnt = colour_count(g, A.dim);
  for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
    int c0, c1, c2;
    if (!colour_cell(g, A.dim, j, phase, c0, c1, c2)) continue;
    const int p = g.at(c0, c1, c2);
    const float a = sa[p];
    if (a == 0.0f) continue;
    zm[p] = div_pos(__fsub_rn(sr[p], csum_t<STO>(zm, sx, A.total, p, g, A.dim, ms)), a);
  }
}

// The coarse V-cycle by the calling block, in `smem` (A.total padded cells
// times 12 bytes, plus the couplings for STO): k_coarse runs it as its own
// launch, the cluster-resident V-cycle (mg_resident.cuh) in its CTA 0.
template <typename ST, bool STO = false>
__device__ __forceinline__ void coarse_vcycle(const CoarseArgs& A, unsigned char* smem) {
  static_assert(!STO || sizeof(ST) == 4, "the stored form runs on float32 grids");
  float* zm = (float*)smem;
  float* sr = zm + A.total;
  float* sa = sr + A.total;
  float* sx = sa + A.total;  // STO: dim arrays
  const float sigma = A.r_f32 ? (float)A.ctl->scale_r : 1.0f;
  const int dim = A.dim;
  const int narr = STO ? 3 + dim : 3;
  // zero everything (the rings stay 0), then load each level's Adiag (and
  // couplings) and level lc's r (FLUID cells) - z starts at 0
  {  // 16-byte stores (the region starts 16-byte aligned), then the tail
    const int nz = narr * A.total, n4 = nz >> 2;
    float4* z4 = reinterpret_cast<float4*>(zm);
    for (int i = threadIdx.x; i < n4; i += blockDim.x) z4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int i = 4 * n4 + threadIdx.x; i < nz; i += blockDim.x) zm[i] = 0.0f;
  }
  __syncthreads();
  for (int l = 0; l < A.nlev; ++l) {
    const PGeom g = pgeom(A, l);
    const int cnt = g.n0 * g.n1 * g.n2;
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
      int c0, c1, c2;
      cell_coords(g, dim, i, c0, c1, c2);
      const int p = g.at(c0, c1, c2);
      const float a = to_f<ST>(((const ST*)A.Ad[l])[i]);
      sa[p] = a;
      if (l == 0 && a != 0.0f) sr[p] = load_r<ST>(A.r0, i, A.r_f32, sigma);
      if constexpr (STO) {
        for (int k = 0; k < dim; ++k) sx[k * A.total + p] = A.Ax[l][k][i];
      }
    }
  }
  __syncthreads();
  const int L = A.nlev;
  // the finest level's cells of each colour, at most 2 per thread: listed once
  // (padded index, -1 for none or not FLUID) for its pre- and post-smoothing
  int li[2][2] = {{-1, -1}, {-1, -1}};
  const bool listed = L > 1 && colour_count(pgeom(A, 0), dim) <= 2 * (int)blockDim.x;
  if (listed) {
    const PGeom g = pgeom(A, 0);
    const int cnt = colour_count(g, dim);
#pragma unroll
    for (int ph = 0; ph < 2; ++ph)
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const int j = threadIdx.x + k * blockDim.x;
        int c0, c1, c2;
        if (j < cnt && colour_cell(g, dim, j, ph, c0, c1, c2)) {
          const int p = g.at(c0, c1, c2);
          if (sa[p] != 0.0f) li[ph][k] = p;
        }
      }
  }
  for (int l = 0; l < L - 1; ++l) {
    for (int i = 0; i < A.pre_post; ++i) {
      if (l == 0 && listed) coarse_smooth_list<STO>(A, 0, li[0], zm, sr, sa, sx);
      else coarse_smooth<STO>(A, l, 0, zm, sr, sa, sx);
      __syncthreads();
      if (l == 0 && listed) coarse_smooth_list<STO>(A, 0, li[1], zm, sr, sa, sx);
      else coarse_smooth<STO>(A, l, 1, zm, sr, sa, sx);
      __syncthreads();
    }
    // restrict: coarse r = rho * sum over FLUID children (lexicographic order);
    // a non-FLUID coarse cell keeps sr = 0, its unmasked z
    const PGeom gf = pgeom(A, l), gc = pgeom(A, l + 1);
    const float ms = -A.s[l];
    const int cnt = gc.n0 * gc.n1 * gc.n2;
    if (dim == 3) {
      // a lane per child: 8 consecutive lanes hold one coarse cell's children
      // (o0, o1, o2 lexicographic), and the first sums their r - A z in that
      // order (blockDim.x is a multiple of 32: every lane of a warp takes the
      // same iterations)
      for (int b = 0; b < 8 * cnt; b += blockDim.x) {
        const int i = b + threadIdx.x;
        const int q = i >> 3, o = i & 7;
        bool use = false;
        float val = 0.0f;
        int pc = -1;
        if (i < 8 * cnt) {
          int c0, c1, c2;
          cell_coords(gc, 3, q, c0, c1, c2);
          pc = gc.at(c0, c1, c2);
          const int p = gf.at(2 * c0 + (o >> 2), 2 * c1 + ((o >> 1) & 1), 2 * c2 + (o & 1));
          const float a = sa[p];
          if (a != 0.0f && sa[pc] != 0.0f) {
            const float Az = __fadd_rn(__fmul_rn(a, zm[p]), csum_t<STO>(zm, sx, A.total, p, gf, dim, ms));
            val = __fsub_rn(sr[p], Az);
            use = true;
          }
        }
        const int lead = (int)(threadIdx.x & 31u) & ~7;
        float acc = 0.0f;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const float vk = __shfl_sync(0xffffffffu, val, lead + k);
          const int uk = __shfl_sync(0xffffffffu, (int)use, lead + k);
          if (uk) acc = __fadd_rn(acc, vk);
        }
        if (o == 0 && pc >= 0 && sa[pc] != 0.0f) sr[pc] = __fmul_rn(A.rho, acc);
      }
      __syncthreads();
      continue;
    }
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
      int c0, c1, c2;
      cell_coords(gc, dim, i, c0, c1, c2);
      const int pc = gc.at(c0, c1, c2);
      if (sa[pc] == 0.0f) continue;
      float acc = 0.0f;
      for (int o0 = 0; o0 < 2; ++o0)
        for (int o1 = 0; o1 < 2; ++o1)
          for (int o2 = 0; o2 < (dim == 3 ? 2 : 1); ++o2) {
            const int p = gf.at(2 * c0 + o0, 2 * c1 + o1, dim == 3 ? 2 * c2 + o2 : 0);
            const float a = sa[p];
            if (a != 0.0f) {
              const float Az = __fadd_rn(__fmul_rn(a, zm[p]), csum_t<STO>(zm, sx, A.total, p, gf, dim, ms));
              acc = __fadd_rn(acc, __fsub_rn(sr[p], Az));
            }
          }
      sr[pc] = __fmul_rn(A.rho, acc);
    }
    __syncthreads();
  }
  // bottom sweeps (mgpcg.py:136-142)
  const int nh = A.bottom / 2;
  {
    const PGeom g = pgeom(A, L - 1);
    const float ms = -A.s[L - 1];
    const int cntb = colour_count(g, dim);
    // participants: kBottomPerThread cells of a colour per thread where that
    // fits, in whole warps; they synchronise among themselves on barrier 1 while the
    // other warps wait at the block barrier below
    int pt = ((cntb + kBottomPerThread - 1) / kBottomPerThread + 31) & ~31;
    if (pt > (int)blockDim.x || (cntb + pt - 1) / pt > kBottomPerThread) pt = blockDim.x;
    if (cntb <= kBottomPerThread * pt) {
      if ((int)threadIdx.x < pt) {
        // each owned cell's padded index, r and 1 / Adiag in registers (and, for
        // STO, its six couplings: constant through the bottom sweeps)
        int gi[2][kBottomPerThread];
        float rr[2][kBottomPerThread];
        double yd[2][kBottomPerThread];  // 1 / Adiag (div_recip64)
        float cx[2][kBottomPerThread][STO ? 6 : 1];
#pragma unroll
        for (int ph = 0; ph < 2; ++ph) {
#pragma unroll
          for (int k = 0; k < kBottomPerThread; ++k) {
            const int j = threadIdx.x + k * pt;
            int c0, c1, c2;
            gi[ph][k] = -1;
            rr[ph][k] = 0.0f;
            yd[ph][k] = 1.0;
#pragma unroll
            for (int e = 0; e < (STO ? 6 : 1); ++e) cx[ph][k][e] = 0.0f;
            if (j < cntb && colour_cell(g, dim, j, ph, c0, c1, c2)) {
              const int p = g.at(c0, c1, c2);
              if (sa[p] != 0.0f) {
                gi[ph][k] = p;
                rr[ph][k] = sr[p];
                yd[ph][k] = 1.0 / (double)sa[p];
                if constexpr (STO) {  // the couplings csum_t reads, in its order
                  cx[ph][k][0] = sx[p - g.s0];
                  cx[ph][k][1] = sx[p];
                  cx[ph][k][2] = sx[A.total + p - g.s1];
                  cx[ph][k][3] = sx[A.total + p];
                  cx[ph][k][4] = dim == 3 ? sx[2 * A.total + p - 1] : 0.0f;
                  cx[ph][k][5] = dim == 3 ? sx[2 * A.total + p] : 0.0f;
                }
              }
            }
          }
        }
        // one half sweep of colour PH (a compile-time constant: the owned
        // cells' registers are named directly, no selects between colours)
        auto half = [&](auto PH) {
          constexpr int ph = decltype(PH)::value;
          float v[kBottomPerThread];
#pragma unroll
          for (int k = 0; k < kBottomPerThread; ++k) {   // all loads first
            const int p = gi[ph][k];
            const int ps = p >= 0 ? p : g.at(0, 0, 0);     // an in-range cell for empty slots
            float sum;
            if constexpr (STO) {  // csum_t with the couplings from registers
              const float* x6 = cx[ph][k];
              sum = __fadd_rn(__fmul_rn(x6[0], zm[ps - g.s0]), __fmul_rn(x6[1], zm[ps + g.s0]));
              sum = __fadd_rn(0.0f, sum);
              sum = __fadd_rn(sum, __fadd_rn(__fmul_rn(x6[2], zm[ps - g.s1]), __fmul_rn(x6[3], zm[ps + g.s1])));
              if (dim == 3) sum = __fadd_rn(sum, __fadd_rn(__fmul_rn(x6[4], zm[ps - 1]), __fmul_rn(x6[5], zm[ps + 1])));
            } else {
              sum = csum_t<STO>(zm, sx, A.total, ps, g, dim, ms);
            }
            v[k] = div_recip64(__fsub_rn(rr[ph][k], sum), yd[ph][k]);
          }
#pragma unroll
          for (int k = 0; k < kBottomPerThread; ++k) {   // then the stores
            const int p = gi[ph][k];
            if (p >= 0) zm[p] = v[k];
          }
          asm volatile("bar.sync 1, %0;" ::"r"(pt) : "memory");
        };
        using C0 = std::integral_constant<int, 0>;
        using C1 = std::integral_constant<int, 1>;
        for (int i = 0; i < nh; ++i) {  // colours 0, 1 (mgpcg.py:136-138)
          half(C0{});
          half(C1{});
        }
        for (int i = 0; i < nh; ++i) {  // then 1, 0 (mgpcg.py:139-141)
          half(C1{});
          half(C0{});
        }
      }
      __syncthreads();
    } else {
      for (int i = 0; i < 2 * nh; ++i) {
        for (int h = 0; h < 2; ++h) {
          coarse_smooth<STO>(A, L - 1, i < nh ? h : 1 - h, zm, sr, sa, sx);
          __syncthreads();
        }
      }
    }
  }
  for (int l = L - 2; l >= 0; --l) {
    // prolongate: every cell += parent's unmasked z (FLUID: zm, else sr)
    const PGeom gf = pgeom(A, l), gc = pgeom(A, l + 1);
    const int cnt = gf.n0 * gf.n1 * gf.n2;
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
      int c0, c1, c2;
      cell_coords(gf, dim, i, c0, c1, c2);
      const int pc = gc.at(c0 >> 1, c1 >> 1, dim == 3 ? c2 >> 1 : 0);
      const float v = __fmul_rn(A.pi, sa[pc] != 0.0f ? zm[pc] : sr[pc]);
      const int p = gf.at(c0, c1, c2);
      if (sa[p] != 0.0f) zm[p] = __fadd_rn(zm[p], v);
      else sr[p] = __fadd_rn(sr[p], v);
    }
    __syncthreads();
    for (int i = 0; i < A.pre_post; ++i) {
      if (l == 0 && listed) coarse_smooth_list<STO>(A, 0, li[1], zm, sr, sa, sx);
      else coarse_smooth<STO>(A, l, 1, zm, sr, sa, sx);
      __syncthreads();
      if (l == 0 && listed) coarse_smooth_list<STO>(A, 0, li[0], zm, sr, sa, sx);
      else coarse_smooth<STO>(A, l, 0, zm, sr, sa, sx);
      __syncthreads();
    }
  }
  const PGeom g0 = pgeom(A, 0);
  const int cnt0 = g0.n0 * g0.n1 * g0.n2;
  for (int i = threadIdx.x; i < cnt0; i += blockDim.x) {
    int c0, c1, c2;
    cell_coords(g0, dim, i, c0, c1, c2);
    const int p = g0.at(c0, c1, c2);
    ((ST*)A.z0)[i] = from_f<ST>(sa[p] != 0.0f ? zm[p] : sr[p]);
  }
}

template <typename ST, bool STO = false>
__global__ void __launch_bounds__(kCoarseThreads) k_coarse(CoarseArgs A) {
  pdl_enter();
  extern __shared__ __align__(16) unsigned char smem[];
  coarse_vcycle<ST, STO>(A, smem);
}

}  // namespace mg
