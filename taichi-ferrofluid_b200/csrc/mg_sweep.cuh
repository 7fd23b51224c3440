// The fused V-cycle kernels for the label-uniform operator (see mg_fused.cuh
// for the design and the scaling of 16-bit grids).
#pragma once
#include "mg_fused.cuh"

namespace mg {

// ---------------------------------------------------------------------------
// k_sweep: streamed, temporally blocked red-black smoothing of one level
// ---------------------------------------------------------------------------
//
// Shared memory holds a ring of W planes; per plane cell: z (float, MASKED:
// 0 on every non-FLUID cell), r (float), Adiag (float), label (int8).
// Because non-FLUID neighbours hold 0, a neighbour term is (-s) * z for every
// neighbour: that is the reference's Ax * z (Ax = -s between two FLUID cells,
// else 0) up to the sign of a zero product, which no later operation can see
// (x + (+-0) == x, and (r - +-0) == r for r != 0; 0 - +-0 == +0).
// Non-FLUID cells are never smoothed; their (unmasked) z is rebuilt for the
// output from the inputs.
//
// The plane after the current one is prefetched into registers while the
// current one is smoothed, so the loads' latency overlaps the half sweeps.
template <int DIM, typename ST, int NS, int TX, int TY, bool PRE, int NT>
__global__ void __launch_bounds__(NT) k_sweep(SweepArgs<ST> A) {
  constexpr int H = PRE ? NS + 1 : NS;            // in-plane halo
  constexpr int RX = TX + 2 * H;
  constexpr int RY = DIM == 3 ? TY + 2 * H : 1;
  constexpr int PL = RX * RY;                     // cells per plane
  constexpr int W = PRE ? NS + 3 : NS + 2;        // ring depth
  constexpr int CX = TX / 2, CY = DIM == 3 ? TY / 2 : 1;
  constexpr int PF = (PL + NT - 1) / NT;          // prefetched cells per thread
  static_assert(CX * CY <= NT, "coarse cells of a tile must not exceed the threads");

  extern __shared__ __align__(16) unsigned char smem[];
  float* sz = (float*)smem;                       // [W][PL]
  float* sr = sz + W * PL;
  float* sa = sr + W * PL;
  int8_t* sl = (int8_t*)(sa + W * PL);

  const FLevel<ST>& F = A.f;
  const int n0 = F.n[0], n1 = F.n[1], n2 = F.n[2];
  const int nx = DIM == 3 ? n2 : n1;             // in-plane fastest extent
  const int ny = DIM == 3 ? n1 : 1;
  const int ntile = A.tiles_x * A.tiles_y;
  const int tile = blockIdx.x % ntile;
  const int chunk_id = blockIdx.x / ntile;
  const int tx0 = (tile % A.tiles_x) * TX;        // interior origin in the plane
  const int ty0 = DIM == 3 ? (tile / A.tiles_x) * TY : 0;
  const int z0 = chunk_id * A.chunk;
  const int z1 = min(z0 + A.chunk, n0);
  const int p_first = z0 - H;
  const int p_last = PRE ? z1 + NS : z1 - 1 + NS;
  const float sigma = A.r_f32 ? (float)A.ctl->scale_r : 1.0f;
  const float ms = -F.s;
  const long long plane_stride = (long long)n1 * n2;
  const int ncx = DIM == 3 ? A.nc[2] : A.nc[1];
  const int ncy = DIM == 3 ? A.nc[1] : 1;

  auto slot = [](int p) { return (p + W * 64) % W; };

  // ---- register prefetch of one plane --------------------------------------
  float fz[PF], fr[PF], fa[PF];
  int8_t fl[PF];
  auto fetch = [&](int p) {
    const bool inside = p >= 0 && p < n0;
#pragma unroll
    for (int k = 0; k < PF; ++k) {
      const int j = threadIdx.x + k * NT;
      fz[k] = 0.0f;
      fr[k] = 0.0f;
      fa[k] = 1.0f;
      fl[k] = SOLID;
      if (j < PL) {
        const int rx = j % RX, ry = j / RX;
        const int gx = tx0 - H + rx, gy = ty0 - (DIM == 3 ? H : 0) + ry;
        if (inside && gx >= 0 && gx < nx && gy >= 0 && gy < ny) {
          const long long gi = (long long)p * plane_stride + (long long)gy * nx + gx;
          fl[k] = F.type[gi];
          fr[k] = load_r<ST>(F.r, gi, A.r_f32, sigma);
          fa[k] = to_f<ST>(F.Ad[gi]);
          if (!PRE) {
            const long long gc = DIM == 3
                ? ((long long)(p >> 1) * A.nc[1] + (gy >> 1)) * A.nc[2] + (gx >> 1)
                : (long long)(p >> 1) * A.nc[1] + (gx >> 1);
            fz[k] = __fadd_rn(to_f<ST>(F.zin[gi]), __fmul_rn(A.pi, to_f<ST>(A.zc[gc])));
          }
        }
      }
    }
  };
  auto store = [&](int p) {
    const int so = slot(p) * PL;
#pragma unroll
    for (int k = 0; k < PF; ++k) {
      const int j = threadIdx.x + k * NT;
      if (j < PL) {
        sl[so + j] = fl[k];
        sr[so + j] = fr[k];
        sa[so + j] = fa[k];
        sz[so + j] = fl[k] == FLUID ? fz[k] : 0.0f;
      }
    }
  };

  // neighbour sum (mgpcg.py:96-102) of cell c of the plane at slot offset sc
  auto nsum = [&](int sb, int sc, int sa_, int c) {
    float ret = 0.0f;
    ret = __fadd_rn(ret, __fadd_rn(__fmul_rn(ms, sz[sb + c]), __fmul_rn(ms, sz[sa_ + c])));
    if (DIM == 3)
      ret = __fadd_rn(ret, __fadd_rn(__fmul_rn(ms, sz[sc + c - RX]), __fmul_rn(ms, sz[sc + c + RX])));
    ret = __fadd_rn(ret, __fadd_rn(__fmul_rn(ms, sz[sc + c - 1]), __fmul_rn(ms, sz[sc + c + 1])));
    return ret;
  };

  float acc = 0.0f;                               // restriction accumulator (PRE)
  const int ct = threadIdx.x;                     // coarse in-plane cell of this thread
  const int ccx = ct % CX, ccy = ct / CX;

  fetch(p_first);
  for (int pl = p_first; pl <= p_last; ++pl) {
    store(pl);
    __syncthreads();
    if (pl < p_last) fetch(pl + 1);  // in flight during the half sweeps

    // ---- half sweeps m = 1..NS on planes pl-m ------------------------------
#pragma unroll
    for (int m = 1; m <= NS; ++m) {
      const int pm = pl - m;
      if (pm - 1 >= p_first && pm >= 0 && pm < n0) {
        const int colour = PRE ? ((m - 1) & 1) : (m & 1);
        const int sc = slot(pm) * PL, sb = slot(pm - 1) * PL, sa_ = slot(pm + 1) * PL;
        constexpr int dummy = 0;
        (void)dummy;
        const int lo = DIM == 3 ? m : 0;           // region rows [lo, RY-lo)
        const int rows = RY - 2 * lo;
        const int cols = RX - 2 * m;
        const int hc = (cols + 1) >> 1;
        // parity of the region origin: global (pm, ty0-H+lo, tx0-H+m)
        const int org = pm + (DIM == 3 ? ty0 - H + lo : 0) + (tx0 - H + m);
        for (int j = threadIdx.x; j < rows * hc; j += NT) {
          const int row = j / hc, k = j - row * hc;
          const int cx = 2 * k + ((colour - org - row) & 1);
          if (cx >= cols) continue;
          const int c = (lo + row) * RX + (m + cx);
          if (sl[sc + c] != FLUID) continue;
          sz[sc + c] = __fdiv_rn(__fsub_rn(sr[sc + c], nsum(sb, sc, sa_, c)), sa[sc + c]);
        }
      }
      __syncthreads();
    }

    // ---- write the finished plane pl-NS --------------------------------------
    const int pw = pl - NS;
    if (pw >= z0 && pw < z1) {
      const int so = slot(pw) * PL;
      for (int j = threadIdx.x; j < TX * (DIM == 3 ? TY : 1); j += NT) {
        const int ix = j % TX, iy = j / TX;
        const int gx = tx0 + ix, gy = ty0 + iy;
        if (gx < nx && gy < ny) {
          const int c = (iy + (DIM == 3 ? H : 0)) * RX + (ix + H);
          const long long gi = (long long)pw * plane_stride + (long long)gy * nx + gx;
          float v = sz[so + c];
          if (!PRE && sl[so + c] != FLUID) {
            // unmasked value of a cell the smoother never touches
            const long long gc = DIM == 3
                ? ((long long)(pw >> 1) * A.nc[1] + (gy >> 1)) * A.nc[2] + (gx >> 1)
                : (long long)(pw >> 1) * A.nc[1] + (gx >> 1);
            v = __fadd_rn(to_f<ST>(F.zin[gi]), __fmul_rn(A.pi, to_f<ST>(A.zc[gc])));
          }
          F.z[gi] = from_f<ST>(v);
        }
      }
    }

    // ---- PRE: residual of plane pl-NS-1 and restriction ------------------------
    if (PRE) {
      const int pr = pl - NS - 1;
      if (pr >= z0 && pr < z1 && ct < CX * CY) {
        const int sc = slot(pr) * PL, sb = slot(pr - 1) * PL, sa_ = slot(pr + 1) * PL;
        if ((pr & 1) == 0) acc = 0.0f;
#pragma unroll
        for (int o1 = 0; o1 < (DIM == 3 ? 2 : 1); ++o1) {
#pragma unroll
          for (int o2 = 0; o2 < 2; ++o2) {
            const int c = (DIM == 3 ? H + 2 * ccy + o1 : 0) * RX + (H + 2 * ccx + o2);
            if (sl[sc + c] == FLUID) {
              const float Az = __fadd_rn(__fmul_rn(sa[sc + c], sz[sc + c]), nsum(sb, sc, sa_, c));
              acc = __fadd_rn(acc, __fsub_rn(sr[sc + c], Az));
            }
          }
        }
        if ((pr & 1) == 1) {
          const int gcx = (tx0 >> 1) + ccx, gcy = (ty0 >> 1) + ccy;
          if (gcx < ncx && gcy < ncy) {
            const long long gc = ((long long)(pr >> 1) * ncy + gcy) * ncx + gcx;
            A.rc[gc] = from_f<ST>(__fmul_rn(A.rho, acc));
            A.zc[gc] = from_f<ST>(0.0f);
          }
        }
      }
    }
    // the next store overwrites the slot of plane pl-W+1 (no longer read)
    __syncthreads();
  }
}

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
