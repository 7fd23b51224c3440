// The streamed smoothing kernels of the fused V-cycle for the label-uniform
// operator (see mg_fused.cuh for the design and the scaling of 16-bit grids).
#pragma once
#include "mg_fused.cuh"

namespace mg {

// ---- 4-wide loads and stores (16 bytes of float32, 8 bytes of 16-bit) -----
template <typename T> __device__ __forceinline__ void ld4(const T* p, float v[4]);
template <> __device__ __forceinline__ void ld4<float>(const float* p, float v[4]) {
  const float4 q = __ldg(reinterpret_cast<const float4*>(p));
  v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
template <> __device__ __forceinline__ void ld4<__half>(const __half* p, float v[4]) {
  const uint2 q = __ldg(reinterpret_cast<const uint2*>(p));
  const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&q.x));
  const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&q.y));
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
template <> __device__ __forceinline__ void ld4<__nv_bfloat16>(const __nv_bfloat16* p, float v[4]) {
  const uint2 q = __ldg(reinterpret_cast<const uint2*>(p));
  const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&q.x));
  const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&q.y));
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
template <typename T> __device__ __forceinline__ void st4(T* p, const float v[4]);
template <> __device__ __forceinline__ void st4<float>(float* p, const float v[4]) {
  *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
template <> __device__ __forceinline__ void st4<__half>(__half* p, const float v[4]) {
  __half2 a = __floats2half2_rn(v[0], v[1]), b = __floats2half2_rn(v[2], v[3]);
  uint2 q;
  q.x = *reinterpret_cast<unsigned*>(&a);
  q.y = *reinterpret_cast<unsigned*>(&b);
  *reinterpret_cast<uint2*>(p) = q;
}
template <> __device__ __forceinline__ void st4<__nv_bfloat16>(__nv_bfloat16* p, const float v[4]) {
  __nv_bfloat162 a = __floats2bfloat162_rn(v[0], v[1]), b = __floats2bfloat162_rn(v[2], v[3]);
  uint2 q;
  q.x = *reinterpret_cast<unsigned*>(&a);
  q.y = *reinterpret_cast<unsigned*>(&b);
  *reinterpret_cast<uint2*>(p) = q;
}

// r of 4 cells: level 0 is the float32 CG residual (times sigma for 16-bit
// grids), coarser levels hold storage-type values.
template <typename ST>
__device__ __forceinline__ void ld4_r(const void* r, long long i, int r_f32, float sigma, float v[4]) {
  if (r_f32) {
    ld4<float>((const float*)r + i, v);
    if constexpr (sizeof(ST) != 4) {
#pragma unroll
      for (int e = 0; e < 4; ++e) v[e] = __fmul_rn(sigma, v[e]);
    }
  } else {
    ld4<ST>((const ST*)r + i, v);
  }
}

// Half sweeps of the whole-domain stored form over the K planes of a step as
// one index space (1) or plane by plane (0); both compute the same values.
// Measured on B200: the stored form's one-step level 32^3 (psi, 128^3) 18.8 +
// 15.3 -> 12.0 + 10.3 us (PRE + POST); the label-uniform kernels are faster
// plane by plane (level 0 PRE 42.7 vs 47.2 us), so they stay so.
#ifndef MG_SWEEP_FLAT
#define MG_SWEEP_FLAT 1
#endif
// When a plane's region holds no more colour cells than the block has
// threads (every tile in use), a half sweep gives each thread one cell per
// plane instead of a pair whose second item is empty: 1 plane by plane, 2
// with the K planes' cells computed before any is stored, 0 the pair loop.
// Measured on B200 (128^3 pressure, level-0 PRE / POST): 39.7 / 43.6 us (1),
// 43.1 / 46.1 (2), 42.8 / 45.3 (0).
#ifndef MG_SWEEP_SINGLE
#define MG_SWEEP_SINGLE 1
#endif

// ---------------------------------------------------------------------------
// k_sweep: streamed, temporally blocked red-black smoothing of one level
// ---------------------------------------------------------------------------
//
// A block owns a (TY x TX) tile of columns and a chunk [z0, z1) of planes
// along axis 0.  Shared memory holds a ring of W planes of the tile plus a
// halo of NS cells (rounded up to 4 along x); per cell z, r and Adiag as float32.  Each step loads K
// planes (4-wide vector loads from registers prefetched during the previous
// step) and applies half sweep m to the planes m behind the newest ones, so
// every half sweep sees its neighbours after the previous half sweep.
//
// Labels never enter the kernel: a cell is FLUID exactly when its Adiag is
// nonzero (the Strategy writes Adiag only on FLUID cells and every FLUID cell
// of a label-uniform level has a nonzero diagonal - mg_plan_prepare checks
// both).  z is stored MASKED (0 on every non-FLUID cell), so a neighbour term
// is (-s) * z for every neighbour: the reference's Ax * z (Ax = -s between two
// FLUID cells, else 0) up to the sign of a zero product, which no later
// operation can see (x + (+-0) == x; r - (+-0) == r for r != 0; 0 - (+-0) == +0).
// Non-FLUID cells are never smoothed; POST writes their (unmasked) output
// value z + pi * z_coarse when it loads them.
//
// PRE starts from z = 0, so its first half sweep is pointwise, z = r / Adiag
// on colour-0 cells (the neighbour sum is +0): it is applied while storing a
// plane, which saves one ring of halo.
//
// STO (whole-domain stored form, float32 only): every cell is FLUID and the
// couplings are the stored Ax of the level, staged in the ring beside z, r
// and Adiag; the neighbour sum is the reference's
//   sum_k Ax[I-e_k][k] z[I-e_k] + Ax[I][k] z[I+e_k]
// with the same operation order, and a neighbour outside the grid is loaded
// as z = 0, Ax = 0 (rule H1).
template <int DIM, typename ST, int NS, int TX, int TY, bool PRE, int NT, int K, bool STO = false>
__device__ __forceinline__ void sweep_body(const SweepArgs<ST>& A, int bid_, int nb_) {
  static_assert(!STO || sizeof(ST) == 4, "the stored form runs on float32 grids");
  // halos: NS cells are needed on each side; along the fastest axis the halo
  // is rounded up to 4 so every 4-wide group starts 16-byte (float) / 8-byte
  // (16-bit) aligned; the XS extra cells are loaded but never smoothed
  constexpr int HY = DIM == 3 ? NS : 0;
  constexpr int HX = (NS + 3) & ~3;
  constexpr int XS = HX - NS;
  constexpr int RX = TX + 2 * HX;
  constexpr int RY = DIM == 3 ? TY + 2 * HY : 1;
  constexpr int PL = RX * RY;                     // cells per plane
  // ring depth; a launch whose single step holds the whole 2-plane chunk and
  // its 2 NS halo planes (K = 2 + 2 NS, chunk 2) needs no ring
  constexpr bool ONE = K == 2 + 2 * NS;
  constexpr int W = ONE ? K : K + NS + 1;
  constexpr int Q = RX / 4;                       // 4-cell groups per row
  constexpr int PL4 = Q * RY;                     // groups per plane
  constexpr int PF = ONE ? 1 : (K * PL4 + NT - 1) / NT;  // prefetched groups per thread
  constexpr int CX = TX / 2, CY = DIM == 3 ? TY / 2 : 1;
  constexpr int D = PRE ? NS - 1 : NS;            // delay of the last half sweep
  static_assert(RX % 4 == 0 && TX % 4 == 0 && HX % 4 == 0, "aligned 4-wide groups");
  static_assert(CX * CY <= NT, "coarse cells of a tile must not exceed the threads");

  extern __shared__ __align__(16) unsigned char smem[];
  float* sz = (float*)smem;                       // [W][PL]
  float* sr = sz + W * PL;
  float* sa = sr + W * PL;
  float* sx0 = sa + W * PL;                       // STO: Ax[0] (plane axis)
  float* sx1 = sx0 + W * PL;                      // STO, 3D: Ax[1] (rows)
  float* sxx = DIM == 3 ? sx1 + W * PL : sx1;     // STO: Ax[dim-1] (fastest axis)
  constexpr int NX = STO ? DIM : 1;               // coefficient arrays loaded per cell
  // 16-bit grids (the mixed form) need no bit-exact float32: the plain
  // neighbour sum as a tree, one FMA and the approximate reciprocal (the
  // column kernel's smooth_cell / residual_cell take the same operations)
  constexpr bool FAST = sizeof(ST) != 4 && !STO;

  const FLevel<ST>& F = A.f;
  const int n0 = F.n[0], n1 = F.n[1], n2 = F.n[2];
  const int nx = DIM == 3 ? n2 : n1;             // in-plane fastest extent (multiple of 4)
  const int ny = DIM == 3 ? n1 : 1;
  const int ntile = A.tiles_x * A.tiles_y;
  const int tile = bid_ % ntile;
  const int chunk_id = bid_ / ntile;
  const int tx0 = (tile % A.tiles_x) * TX;        // interior origin in the plane
  const int ty0 = DIM == 3 ? (tile / A.tiles_x) * TY : 0;
  const int z0 = chunk_id * A.chunk;
  const int z1 = min(z0 + A.chunk, n0);
  const int p_first = z0 - NS;
  const int p_last = z1 + NS - 1;
  const float sigma = A.r_f32 ? (float)A.ctl->scale_r : 1.0f;
  const float ms = -F.s;
  const long long plane_stride = (long long)n1 * n2;
  const int ncx = DIM == 3 ? A.nc[2] : A.nc[1];
  const int ncy = DIM == 3 ? A.nc[1] : 1;

  auto slot = [](int p) { return (p + W * 64) % W; };

  // ---- loading planes ---------------------------------------------------------------
  // group q of the K planes from P: global loads into r[4], a[4], z[4] and
  // (STO) the coefficients x[NX][4]
  auto load_group = [&](int P, int q, float* r, float* a, float* z, float (*x)[4]) {
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      r[e] = 0.0f;
      a[e] = 0.0f;
      z[e] = 0.0f;
#pragma unroll
      for (int k = 0; k < NX; ++k) x[k][e] = 0.0f;
    }
    const int kp = q / PL4, rem = q - kp * PL4;
    const int ry = rem / Q, rx = (rem - ry * Q) * 4;
    const int p = P + kp;
    const int gx = tx0 - HX + rx, gy = ty0 - HY + ry;
    if (p >= 0 && p < n0 && gx >= 0 && gx < nx && gy >= 0 && gy < ny) {
      const long long gi = (long long)p * plane_stride + (long long)gy * nx + gx;
      ld4_r<ST>(F.r, gi, A.r_f32, sigma, r);
      ld4<ST>(F.Ad + gi, a);
      if constexpr (STO) {
#pragma unroll
        for (int k = 0; k < NX; ++k) ld4<float>(F.ax[k] + gi, x[k]);
      }
      if (!PRE) {
        float zi[4];
        ld4<ST>(F.zin + gi, zi);
        const long long gc = DIM == 3
            ? ((long long)(p >> 1) * A.nc[1] + (gy >> 1)) * A.nc[2] + (gx >> 1)
            : (long long)(p >> 1) * A.nc[1] + (gx >> 1);
        const float c0 = to_f<ST>(A.zc[gc]), c1 = to_f<ST>(A.zc[gc + 1]);
        z[0] = __fadd_rn(zi[0], __fmul_rn(A.pi, c0));
        z[1] = __fadd_rn(zi[1], __fmul_rn(A.pi, c0));
        z[2] = __fadd_rn(zi[2], __fmul_rn(A.pi, c1));
        z[3] = __fadd_rn(zi[3], __fmul_rn(A.pi, c1));
      }
    }
  };
  // store group q into shared memory; PRE applies its pointwise first half
  // sweep, POST writes the final value of non-FLUID interior cells it owns
  auto put_group = [&](int P, int q, const float* r, const float* a, const float* z, const float (*x)[4]) {
    const int kp = q / PL4, rem = q - kp * PL4;
    const int ry = rem / Q, rx = (rem - ry * Q) * 4;
    const int p = P + kp;
    const int gx = tx0 - HX + rx, gy = ty0 - HY + ry;
    float zv[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if (PRE) {
        const bool c0 = ((p + gy + gx + e) & 1) == 0;
        zv[e] = (c0 && a[e] != 0.0f) ? (FAST ? __fdividef(r[e], a[e]) : div_pos(r[e], a[e])) : 0.0f;
      } else {
        zv[e] = a[e] != 0.0f ? z[e] : 0.0f;
      }
    }
    const int o = slot(p) * PL + ry * RX + rx;
    *reinterpret_cast<float4*>(sz + o) = make_float4(zv[0], zv[1], zv[2], zv[3]);
    *reinterpret_cast<float4*>(sr + o) = make_float4(r[0], r[1], r[2], r[3]);
    *reinterpret_cast<float4*>(sa + o) = make_float4(a[0], a[1], a[2], a[3]);
    if constexpr (STO) {
      *reinterpret_cast<float4*>(sx0 + o) = make_float4(x[0][0], x[0][1], x[0][2], x[0][3]);
      if (DIM == 3) *reinterpret_cast<float4*>(sx1 + o) = make_float4(x[1][0], x[1][1], x[1][2], x[1][3]);
      *reinterpret_cast<float4*>(sxx + o) =
          make_float4(x[NX - 1][0], x[NX - 1][1], x[NX - 1][2], x[NX - 1][3]);
    }
    if (!PRE && p >= z0 && p < z1 && gx >= tx0 && gx < tx0 + TX && gx < nx &&
        gy >= ty0 && gy < ty0 + (DIM == 3 ? TY : 1) && gy < ny) {
      const long long gi = (long long)p * plane_stride + (long long)gy * nx + gx;
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (a[e] == 0.0f) F.z[gi + e] = from_f<ST>(z[e]);
    }
  };
  // streaming: the next K planes are prefetched into registers during the
  // current step; one step (ONE): loaded straight into shared memory
  float fr[PF][4], fa[PF][4], fz[PF][4], fx[PF][NX][4];
  auto fetch = [&](int P) {
#pragma unroll
    for (int g = 0; g < PF; ++g) {
      const int q = threadIdx.x + g * NT;
      if (q < K * PL4) load_group(P, q, fr[g], fa[g], fz[g], fx[g]);
    }
  };
  auto store = [&](int P) {
    if constexpr (ONE) {
      for (int q = threadIdx.x; q < K * PL4; q += NT) {
        float r[4], a[4], z[4], x[NX][4];
        load_group(P, q, r, a, z, x);
        put_group(P, q, r, a, z, x);
      }
    } else {
#pragma unroll
      for (int g = 0; g < PF; ++g) {
        const int q = threadIdx.x + g * NT;
        if (q < K * PL4) put_group(P, q, fr[g], fa[g], fz[g], fx[g]);
      }
    }
  };

  // neighbour sum (mgpcg.py:96-102) of cell c of the plane at slot offset sc
  auto nsum = [&](int sb, int sc, int sa_, int c) {
    float ret = 0.0f;
    if constexpr (STO) {
      ret = __fadd_rn(ret, __fadd_rn(__fmul_rn(sx0[sb + c], sz[sb + c]), __fmul_rn(sx0[sc + c], sz[sa_ + c])));
      if (DIM == 3)
        ret = __fadd_rn(ret, __fadd_rn(__fmul_rn(sx1[sc + c - RX], sz[sc + c - RX]),
                                       __fmul_rn(sx1[sc + c], sz[sc + c + RX])));
      ret = __fadd_rn(ret, __fadd_rn(__fmul_rn(sxx[sc + c - 1], sz[sc + c - 1]),
                                     __fmul_rn(sxx[sc + c], sz[sc + c + 1])));
    } else {
      ret = __fadd_rn(ret, __fadd_rn(__fmul_rn(ms, sz[sb + c]), __fmul_rn(ms, sz[sa_ + c])));
      if (DIM == 3)
        ret = __fadd_rn(ret, __fadd_rn(__fmul_rn(ms, sz[sc + c - RX]), __fmul_rn(ms, sz[sc + c + RX])));
      ret = __fadd_rn(ret, __fadd_rn(__fmul_rn(ms, sz[sc + c - 1]), __fmul_rn(ms, sz[sc + c + 1])));
    }
    return ret;
  };

  const float spos = F.s;
  auto zsum = [&](int sb, int sc, int sa_, int c) {
    if constexpr (DIM == 3)
      return __fadd_rn(__fadd_rn(__fadd_rn(sz[sb + c], sz[sa_ + c]), __fadd_rn(sz[sc + c - RX], sz[sc + c + RX])),
                       __fadd_rn(sz[sc + c - 1], sz[sc + c + 1]));
    else
      return __fadd_rn(__fadd_rn(sz[sb + c], sz[sa_ + c]), __fadd_rn(sz[sc + c - 1], sz[sc + c + 1]));
  };
  // smooth (mgpcg.py:104-109) of the FLUID cell c with diagonal a and residual r
  auto upd = [&](float r, int sb, int sc, int sa_, int c, float a) -> float {
    if constexpr (FAST) return __fdividef(fmaf(spos, zsum(sb, sc, sa_, c), r), a);
    else return div_pos(__fsub_rn(r, nsum(sb, sc, sa_, c)), a);
  };

  float acc = 0.0f;                               // restriction accumulator (PRE)
  double zr_acc = 0.0;                            // z.r of the cells written (POST, A.zr >= 0)
  const int ct = threadIdx.x;                     // coarse in-plane cell of this thread
  const int ccx = ct % CX, ccy = ct / CX;

  if constexpr (!ONE) fetch(p_first);
  for (int P = p_first; P <= p_last; P += K) {
    store(P);
    __syncthreads();
    if constexpr (!ONE) {
      if (P + K <= p_last) fetch(P + K);  // in flight during the half sweeps
    }

    // ---- half sweeps -------------------------------------------------------
#pragma unroll
    for (int m = PRE ? 2 : 1; m <= NS; ++m) {
      const int shift = PRE ? m - 1 : m;           // planes behind the newest
      const int colour = PRE ? ((m - 1) & 1) : (m & 1);
      const int lo = DIM == 3 ? shift : 0;         // region rows [lo, RY-lo)
      const int rows = RY - 2 * lo;
      const int x0 = XS + shift;                   // region cols [x0, RX-x0)
      const int cols = RX - 2 * x0;
      const int hc = (cols + 1) >> 1;
      if constexpr (STO && MG_SWEEP_FLAT) {
      // the K planes of the step as one index space: two cells per thread and
      // iteration, both computed before either is stored (cells of one colour
      // never read each other, in the same plane or the next), so the K
      // planes' dependent add / divide chains overlap instead of following
      // one another
      {
        const int per = rows * hc;                   // colour cells of one plane's region
        for (int j0 = threadIdx.x; j0 < K * per; j0 += 2 * NT) {
          int cc[2];
          float val[2];
          bool ok[2];
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            // past the end: clamp to the last item and skip it
            const int jj = min(j0 + u * NT, K * per - 1);
            const int kp = jj / per, j = jj - kp * per;
            const int pm = P + kp - shift;
            const int sc = slot(pm) * PL, sb = slot(pm - 1) * PL, sa_ = slot(pm + 1) * PL;
            // parity of the region origin: global (pm, ty0-HY+lo, tx0-HX+x0)
            const int org = pm + (DIM == 3 ? ty0 - HY + lo : 0) + (tx0 - HX + x0);
            const int row = j / hc, k = j - row * hc;
            const int cx = min(2 * k + ((colour - org - row) & 1), cols - 1);
            cc[u] = sc + (lo + row) * RX + (x0 + cx);
            ok[u] = j0 + u * NT < K * per && !(pm - 1 < p_first || pm < 0 || pm >= n0) &&
                    2 * k + ((colour - org - row) & 1) < cols;
            const float a = ok[u] ? sa[cc[u]] : 0.0f;
            ok[u] = ok[u] && a != 0.0f;              // FLUID
            val[u] = ok[u] ? upd(sr[cc[u]], sb, sc, sa_, cc[u] - sc, a) : 0.0f;
          }
#pragma unroll
          for (int u = 0; u < 2; ++u)
            if (ok[u]) sz[cc[u]] = val[u];
        }
      }
      } else if (MG_SWEEP_SINGLE == 2 && rows * hc <= NT) {
      // the colour cells of a plane's region fit the block: one cell per
      // thread and plane (no second, empty item), the K planes' values
      // computed before any is stored (cells of one colour never read each
      // other)
      const int j = min((int)threadIdx.x, rows * hc - 1);
      const int row = j / hc, k = j - row * hc;
      float val[K];
      int cidx[K];
      bool ok[K];
#pragma unroll
      for (int kp = 0; kp < K; ++kp) {
        const int pm = P + kp - shift;
        const int sc = slot(pm) * PL, sb = slot(pm - 1) * PL, sa_ = slot(pm + 1) * PL;
        const int org = pm + (DIM == 3 ? ty0 - HY + lo : 0) + (tx0 - HX + x0);
        const int cxr = 2 * k + ((colour - org - row) & 1);
        const int c = (lo + row) * RX + (x0 + min(cxr, cols - 1));
        cidx[kp] = sc + c;
        ok[kp] = (int)threadIdx.x < rows * hc && cxr < cols && !(pm - 1 < p_first || pm < 0 || pm >= n0);
        const float a = ok[kp] ? sa[sc + c] : 0.0f;
        ok[kp] = ok[kp] && a != 0.0f;              // FLUID
        val[kp] = ok[kp] ? upd(sr[sc + c], sb, sc, sa_, c, a) : 0.0f;
      }
#pragma unroll
      for (int kp = 0; kp < K; ++kp)
        if (ok[kp]) sz[cidx[kp]] = val[kp];
      } else {
#pragma unroll
      for (int kp = 0; kp < K; ++kp) {
        // per-plane values hoisted out of the cell loop (uniform per block)
        const int pm = P + kp - shift;
        if (pm - 1 < p_first || pm < 0 || pm >= n0) continue;
        const int sc = slot(pm) * PL, sb = slot(pm - 1) * PL, sa_ = slot(pm + 1) * PL;
        // parity of the region origin: global (pm, ty0-HY+lo, tx0-HX+x0)
        const int org = pm + (DIM == 3 ? ty0 - HY + lo : 0) + (tx0 - HX + x0);
        if (MG_SWEEP_SINGLE == 1 && rows * hc <= NT) {
          // the colour cells of the region fit the block: one cell per thread
          const int j = threadIdx.x;
          if (j < rows * hc) {
            const int row = j / hc, k = j - row * hc;
            const int cxr = 2 * k + ((colour - org - row) & 1);
            if (cxr < cols) {
              const int c = (lo + row) * RX + (x0 + cxr);
              const float a = sa[sc + c];
              if (a != 0.0f) sz[sc + c] = upd(sr[sc + c], sb, sc, sa_, c, a);
            }
          }
          continue;
        }
        // two cells per thread and iteration, both computed before either is
        // stored: cells of one colour never read each other, and the two
        // dependent add / divide chains overlap
        for (int j0 = threadIdx.x; j0 < rows * hc; j0 += 2 * NT) {
          int cc[2];
          float val[2];
          bool ok[2];
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            // past the end: clamp to the last item (in the region) and skip it
            const int j = min(j0 + u * NT, rows * hc - 1);
            const int row = j / hc, k = j - row * hc;
            const int cx = min(2 * k + ((colour - org - row) & 1), cols - 1);
            cc[u] = (lo + row) * RX + (x0 + cx);
            ok[u] = j0 + u * NT < rows * hc && 2 * k + ((colour - org - row) & 1) < cols;
            const float a = ok[u] ? sa[sc + cc[u]] : 0.0f;
            ok[u] = ok[u] && a != 0.0f;              // FLUID
            val[u] = ok[u] ? upd(sr[sc + cc[u]], sb, sc, sa_, cc[u], a) : 0.0f;
          }
#pragma unroll
          for (int u = 0; u < 2; ++u)
            if (ok[u]) sz[sc + cc[u]] = val[u];
        }
      }
      }
      __syncthreads();
    }

    // ---- write the finished planes ------------------------------------------
#pragma unroll
    for (int kp = 0; kp < K; ++kp) {
      const int pw = P + kp - D;
      if (pw < z0 || pw >= z1) continue;
      const int so = slot(pw) * PL;
      for (int j = threadIdx.x; j < (TX / 4) * (DIM == 3 ? TY : 1); j += NT) {
        const int ix = (j % (TX / 4)) * 4, iy = j / (TX / 4);
        const int gx = tx0 + ix, gy = ty0 + iy;
        if (gx >= nx || gy >= ny) continue;
        const int c = (iy + HY) * RX + (ix + HX);
        const long long gi = (long long)pw * plane_stride + (long long)gy * nx + gx;
        float v[4] = {sz[so + c], sz[so + c + 1], sz[so + c + 2], sz[so + c + 3]};
        if (PRE) {
          st4<ST>(F.z + gi, v);                    // non-FLUID cells hold z = 0
        } else {
#pragma unroll
          for (int e = 0; e < 4; ++e)
            if (sa[so + c + e] != 0.0f) {
              F.z[gi + e] = from_f<ST>(v[e]);
              if (A.zr >= 0) zr_acc += (double)v[e] * (double)sr[so + c + e];
            }
        }
      }
    }

    // ---- PRE: residual of the planes D+1 behind and restriction ----------------
    if (PRE) {
#pragma unroll
      for (int kp = 0; kp < K; ++kp) {
        const int pr = P + kp - NS;
        if (pr < z0 || pr >= z1 || ct >= CX * CY) continue;
        const int sc = slot(pr) * PL, sb = slot(pr - 1) * PL, sa_ = slot(pr + 1) * PL;
        if ((pr & 1) == 0) acc = 0.0f;
#pragma unroll
        for (int o1 = 0; o1 < (DIM == 3 ? 2 : 1); ++o1) {
#pragma unroll
          for (int o2 = 0; o2 < 2; ++o2) {
            const int c = (DIM == 3 ? HY + 2 * ccy + o1 : 0) * RX + (HX + 2 * ccx + o2);
            const float a = sa[sc + c];
            if (a != 0.0f) {
              float res;  // r - A z (mgpcg.py:111-118)
              if constexpr (FAST) {
                res = fmaf(-a, sz[sc + c], fmaf(spos, zsum(sb, sc, sa_, c), sr[sc + c]));
              } else {
                const float Az = __fadd_rn(__fmul_rn(a, sz[sc + c]), nsum(sb, sc, sa_, c));
                res = __fsub_rn(sr[sc + c], Az);
              }
              acc = __fadd_rn(acc, res);
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
    // the next store overwrites the slots of planes that are no longer read
    __syncthreads();
  }
  if constexpr (!PRE) {
    if (A.zr >= 0) {  // the reduction and epilogue of k_zr4 (mgpcg.py:161-166, 197-202)
      __shared__ double sh[32];
      double tot;
      Control* ctl = A.zr_ctl;
      if (last_block_total_at<NT>(zr_acc, A.zr_partials, &ctl->counter[1], sh, &tot, bid_, nb_) &&
          threadIdx.x == 0) {
        if (A.zr == 0) {
          ctl->old_zTr = tot;
          if (ctl->max_iters == 0) ctl->run = 0;
        } else {
          ctl->new_zTr = tot;
          ctl->beta = (float)(tot / (ctl->old_zTr + ctl->eps));
          ctl->old_zTr = tot;
          ctl->iter += 1;
          if (ctl->max_iters != -1 && ctl->iter >= ctl->max_iters) ctl->run = 0;
        }
      }
    }
  }
}

template <int DIM, typename ST, int NS, int TX, int TY, bool PRE, int NT, int K, bool STO = false>
__global__ void __launch_bounds__(NT) k_sweep(SweepArgs<ST> A) {
  pdl_enter();
  sweep_body<DIM, ST, NS, TX, TY, PRE, NT, K, STO>(A, (int)blockIdx.x, (int)gridDim.x);
}

}  // namespace mg
