// The cluster-resident V-cycle: the label-uniform levels [lp, L) of a fused
// plan in ONE launch of ONE thread-block cluster (up to 16 CTAs, one per SM).
// Every CTA holds its brick of each brick level [lp, lb) in shared memory for
// the whole V-cycle; CTA 0 also runs the coarse levels [lb, L) (mg_coarse.cuh)
// in a region of its own.
//
// Why: below the finest levels the streamed kernel (mg_sweep.cuh) is latency-
// bound: each level is its own launches, and each launch recomputes a halo of
// 2 * pre_post cells around every tile for the half sweeps it fuses.  Here a
// CTA owns a brick of the level exactly (no recomputation), and between two
// half sweeps only the one-cell rings of the bricks move, read straight from
// the neighbouring CTAs' shared memory (distributed shared memory) after a
// hardware cluster barrier; nothing of the V-cycle goes through global memory
// between the input r and the output z, except the coarse levels' r and z
// (CTA 0 reads and writes them in the plan's level-lb arrays).  The arithmetic
// per cell is the streamed kernel's (masked z, the reference's neighbour-sum
// order, IEEE division), so the V-cycle's float32 values are the same bit for
// bit.
//
// Shared memory per brick level: zs, the masked z of the brick with its
// one-cell ring ((B0+2)(B1+2)(B2+2) floats; 0 on non-FLUID cells and outside
// the level), rs, B0 B1 B2 floats holding r on FLUID cells and the unmasked z
// on the others (which prolongation carries, mgpcg.py:120-123), and, when
// they fit, the brick's Adiag (else read from global memory, read-only here).
// Adiag tells FLUID cells (nonzero on exactly the FLUID cells of a
// label-uniform level).
//
// Rings and the barrier: whenever a CTA gives a FLUID cell on a face of its
// brick a new z (a half sweep, the prolongation), it also stores the value
// into the ring of the neighbour that reads it (distributed shared memory),
// and one cluster barrier (arrive.release, wait.acquire) then publishes every
// CTA's stores.  During a half sweep of colour c the CTAs store colour-c
// values and read colour 1 - c ring cells only, so stores and reads of a ring
// never meet between two barriers.  A barrier after the initial zeroing keeps
// early stores from being overwritten, and a final one keeps every CTA's
// shared memory alive until its neighbours' last stores.
#pragma once
#include <cooperative_groups.h>

#include "mg_coarse.cuh"

namespace mg {

namespace cgx = cooperative_groups;

#ifndef MG_RESIDENT_THREADS
#define MG_RESIDENT_THREADS 1024
#endif
constexpr int kResThreads = MG_RESIDENT_THREADS;
constexpr int kResMaxCtas = 16;  // non-portable cluster size of B200

struct ResLevel {
  int lb[3];         // log2 of the brick extent per axis
  int n[3];          // extent of the level
  int zoff, roff;    // offsets (floats) of zs and rs in shared memory
  int aoff;          // offset of the brick's Adiag in shared memory, -1: global
  float s;           // kappa * s_l
  const float* Ad;   // Adiag of the level (float32)
};

struct ResArgs {
  int nlev;          // brick levels lp .. lp + nlev - 1 (lp + nlev = lb)
  int nb[3];         // bricks (CTAs) per axis
  int ns;            // half sweeps per smoothing (2 pre_post)
  float rho, pi;
  ResLevel lv[kMaxLevels];
  const float* r0;   // r of level lp
  float* z0;         // z of level lp (written: the unmasked z)
  float* rc;         // r of level lb (written by the last restriction)
  const float* zc;   // z of level lb (written by the coarse phase)
  CoarseArgs coarse; // levels lb .. L-1, run by CTA 0
  int coff;          // offset (floats) of the coarse region in shared memory
  int smem_floats;   // dynamic shared memory, in floats
};

// Brick geometry of one level for the calling CTA.
struct RB {
  int B0, B1, B2, l0, l1, l2;   // extents and their log2
  int o0, o1, o2;               // origin of the brick in the level
  int n0, n1, n2;
  int P1, P2;                   // padded strides: zs index ((c0+1) P1 + c1+1) P2 + c2+1
  float* zs;
  float* rs;
  const float* sa;              // Adiag of the brick in shared memory, or null
  const float* Ad;              // Adiag of the level in global memory
  float ms;                     // -(kappa s_l)
  __device__ __forceinline__ int zp(int c0, int c1, int c2) const { return ((c0 + 1) * P1 + (c1 + 1)) * P2 + c2 + 1; }
  __device__ __forceinline__ int ri(int c0, int c1, int c2) const { return (((c0 << l1) + c1) << l2) + c2; }
  __device__ __forceinline__ int gi(int c0, int c1, int c2) const {
    return ((o0 + c0) * n1 + (o1 + c1)) * n2 + (o2 + c2);
  }
  __device__ __forceinline__ float ad(int c0, int c1, int c2) const {
    return sa ? sa[ri(c0, c1, c2)] : __ldg(Ad + gi(c0, c1, c2));
  }
};

__device__ __forceinline__ RB res_brick(const ResArgs& A, int i, float* sm, int rank) {
  const ResLevel& L = A.lv[i];
  RB b;
  b.l0 = L.lb[0];
  b.l1 = L.lb[1];
  b.l2 = L.lb[2];
  b.B0 = 1 << b.l0;
  b.B1 = 1 << b.l1;
  b.B2 = 1 << b.l2;
  const int bx = rank % A.nb[2];
  const int t = rank / A.nb[2];
  const int by = t % A.nb[1], bz = t / A.nb[1];
  b.o0 = bz << b.l0;
  b.o1 = by << b.l1;
  b.o2 = bx << b.l2;
  b.n0 = L.n[0];
  b.n1 = L.n[1];
  b.n2 = L.n[2];
  b.P1 = b.B1 + 2;
  b.P2 = b.B2 + 2;
  b.zs = sm + L.zoff;
  b.rs = sm + L.roff;
  b.sa = L.aoff >= 0 ? sm + L.aoff : nullptr;
  b.Ad = L.Ad;
  b.ms = -L.s;
  return b;
}

// Neighbour sum (mgpcg.py:96-102) on the masked padded brick, in the
// streamed kernel's order: axis 0, axis 1, axis 2, each (lower + upper).
__device__ __forceinline__ float res_nsum(const RB& b, int p) {
  const float* z = b.zs;
  const int s0 = b.P1 * b.P2, s1 = b.P2;
  float ret = 0.0f;
  ret = __fadd_rn(ret, __fadd_rn(__fmul_rn(b.ms, z[p - s0]), __fmul_rn(b.ms, z[p + s0])));
  ret = __fadd_rn(ret, __fadd_rn(__fmul_rn(b.ms, z[p - s1]), __fmul_rn(b.ms, z[p + s1])));
  ret = __fadd_rn(ret, __fadd_rn(__fmul_rn(b.ms, z[p - 1]), __fmul_rn(b.ms, z[p + 1])));
  return ret;
}

// j-th cell of colour `col` in the brick: rows (c0, c1) of B2/2 cells.
__device__ __forceinline__ void res_colour_cell(const RB& b, int j, int col, int& c0, int& c1, int& c2) {
  const int lh = b.l2 - 1;
  const int row = j >> lh;
  const int k = j - (row << lh);
  c1 = row & (b.B1 - 1);
  c0 = row >> b.l1;
  c2 = 2 * k + ((col - b.o0 - b.o1 - b.o2 - c0 - c1) & 1);
}

// The six neighbouring bricks' zs of a brick level (axis 0 lower, upper, axis
// 1 lower, upper, axis 2 lower, upper) in their shared memory; null where the
// level ends.
struct RNb {
  float* z[6];
};
__device__ __forceinline__ RNb res_nbrs(const RB& b, const ResArgs& A, int rank) {
  cgx::cluster_group cl = cgx::this_cluster();
  const int st1 = A.nb[2], st0 = A.nb[1] * A.nb[2];
  RNb n;
  n.z[0] = b.o0 > 0 ? cl.map_shared_rank(b.zs, rank - st0) : nullptr;
  n.z[1] = b.o0 + b.B0 < b.n0 ? cl.map_shared_rank(b.zs, rank + st0) : nullptr;
  n.z[2] = b.o1 > 0 ? cl.map_shared_rank(b.zs, rank - st1) : nullptr;
  n.z[3] = b.o1 + b.B1 < b.n1 ? cl.map_shared_rank(b.zs, rank + st1) : nullptr;
  n.z[4] = b.o2 > 0 ? cl.map_shared_rank(b.zs, rank - 1) : nullptr;
  n.z[5] = b.o2 + b.B2 < b.n2 ? cl.map_shared_rank(b.zs, rank + 1) : nullptr;
  return n;
}

// v, the new z of brick cell (c0, c1, c2), into the rings of the neighbours
// whose cells are its face neighbours.
__device__ __forceinline__ void res_push(const RB& b, const RNb& n, int c0, int c1, int c2, float v) {
  if (c0 == 0 && n.z[0]) n.z[0][b.zp(b.B0, c1, c2)] = v;
  if (c0 == b.B0 - 1 && n.z[1]) n.z[1][b.zp(-1, c1, c2)] = v;
  if (c1 == 0 && n.z[2]) n.z[2][b.zp(c0, b.B1, c2)] = v;
  if (c1 == b.B1 - 1 && n.z[3]) n.z[3][b.zp(c0, -1, c2)] = v;
  if (c2 == 0 && n.z[4]) n.z[4][b.zp(c0, c1, b.B2)] = v;
  if (c2 == b.B2 - 1 && n.z[5]) n.z[5][b.zp(c0, c1, -1)] = v;
}

// One red-black half sweep (mgpcg.py:104-109) of colour `col` over the brick,
// two cells per thread and iteration, both computed before either is stored;
// face cells also go to the neighbours' rings.
__device__ __forceinline__ void res_smooth(const RB& b, const RNb& n, int col) {
  const int cnt = (b.B0 * b.B1 * b.B2) >> 1;
  if (cnt <= (int)blockDim.x) {  // one cell per thread, no empty second item
    const int j = threadIdx.x;
    if (j < cnt) {
      int c0, c1, c2;
      res_colour_cell(b, j, col, c0, c1, c2);
      const float a = b.ad(c0, c1, c2);
      if (a != 0.0f) {
        const int p = b.zp(c0, c1, c2);
        const float v = div_pos(__fsub_rn(b.rs[b.ri(c0, c1, c2)], res_nsum(b, p)), a);
        b.zs[p] = v;
        res_push(b, n, c0, c1, c2, v);
      }
    }
    return;
  }
  for (int j0 = threadIdx.x; j0 < cnt; j0 += 2 * blockDim.x) {
    int cc[2][3];
    float val[2];
    bool ok[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int j = min(j0 + u * (int)blockDim.x, cnt - 1);
      res_colour_cell(b, j, col, cc[u][0], cc[u][1], cc[u][2]);
      const float a = b.ad(cc[u][0], cc[u][1], cc[u][2]);
      ok[u] = j0 + u * (int)blockDim.x < cnt && a != 0.0f;
      val[u] = ok[u] ? div_pos(__fsub_rn(b.rs[b.ri(cc[u][0], cc[u][1], cc[u][2])],
                                         res_nsum(b, b.zp(cc[u][0], cc[u][1], cc[u][2]))),
                               a)
                     : 0.0f;
    }
#pragma unroll
    for (int u = 0; u < 2; ++u)
      if (ok[u]) {
        b.zs[b.zp(cc[u][0], cc[u][1], cc[u][2])] = val[u];
        res_push(b, n, cc[u][0], cc[u][1], cc[u][2], val[u]);
      }
  }
}

// NT threads a CTA (1024 or 512, chosen by measurement per shape: at 512 a
// thread has 128 registers instead of 64, and handles two cells per colour
// of a 2048-cell brick).
template <int NT>
__global__ void __launch_bounds__(NT, 1) k_resident(ResArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  float* sm = (float*)smem;
  cgx::cluster_group cl = cgx::this_cluster();
  const int rank = (int)cl.block_rank();
  const int nlev = A.nlev;

  for (int i = threadIdx.x; i < A.coff; i += blockDim.x) sm[i] = 0.0f;
  cl.sync();  // every CTA's rings are zero before any neighbour stores into them
  for (int i = 0; i < nlev; ++i) {  // the bricks' Adiag, where it has room
    const RB b = res_brick(A, i, sm, rank);
    if (!b.sa) continue;
    float* sa = sm + A.lv[i].aoff;
    const int cells = b.B0 * b.B1 * b.B2;
#pragma unroll 4
    for (int j = threadIdx.x; j < cells; j += blockDim.x) {
      const int c2 = j & (b.B2 - 1), c1 = (j >> b.l2) & (b.B1 - 1), c0 = j >> (b.l1 + b.l2);
      sa[j] = __ldg(b.Ad + b.gi(c0, c1, c2));
    }
  }
  __syncthreads();

  // ---- pre-smoothing and restriction, finest to coarsest ----------------------
  for (int i = 0; i < nlev; ++i) {
    const RB b = res_brick(A, i, sm, rank);
    const RNb nb = res_nbrs(b, A, rank);
    const int cells = b.B0 * b.B1 * b.B2;
    if (i == 0) {  // r of level lp (FLUID cells; the others hold z = 0)
#pragma unroll 4
      for (int j = threadIdx.x; j < cells; j += blockDim.x) {
        const int c2 = j & (b.B2 - 1), c1 = (j >> b.l2) & (b.B1 - 1), c0 = j >> (b.l1 + b.l2);
        const float r = __ldcg(A.r0 + b.gi(c0, c1, c2));
        b.rs[j] = b.ad(c0, c1, c2) != 0.0f ? r : 0.0f;
      }
      __syncthreads();
    }
    // first half sweep from z = 0: pointwise on colour 0
    for (int j = threadIdx.x; j < (cells >> 1); j += blockDim.x) {
      int c0, c1, c2;
      res_colour_cell(b, j, 0, c0, c1, c2);
      const float a = b.ad(c0, c1, c2);
      if (a != 0.0f) {
        const float v = div_pos(b.rs[b.ri(c0, c1, c2)], a);
        b.zs[b.zp(c0, c1, c2)] = v;
        res_push(b, nb, c0, c1, c2, v);
      }
    }
    for (int m = 2; m <= A.ns; ++m) {
      cl.sync();  // the rings of half sweep m - 1's colour
      res_smooth(b, nb, (m - 1) & 1);
    }
    cl.sync();  // both colours of the rings for the restriction
    // restriction (mgpcg.py:111-118): coarse r = rho * sum over the FLUID
    // children (lexicographic order) of r - A z; a coarse cell of the brick
    // has all 8 children in the brick
    const bool last = i + 1 == nlev;
    RB c;
    if (!last) c = res_brick(A, i + 1, sm, rank);
    const int cl1 = b.l1 - 1, cl2 = b.l2 - 1;
    const int ccells = cells >> 3;
    const int cn1 = b.n1 >> 1, cn2 = b.n2 >> 1;
    for (int j = threadIdx.x; j < ccells; j += blockDim.x) {
      const int q2 = j & ((1 << cl2) - 1), q1 = (j >> cl2) & ((1 << cl1) - 1), q0 = j >> (cl1 + cl2);
      float acc = 0.0f;
#pragma unroll
      for (int o0 = 0; o0 < 2; ++o0)
#pragma unroll
        for (int o1 = 0; o1 < 2; ++o1)
#pragma unroll
          for (int o2 = 0; o2 < 2; ++o2) {
            const int f0 = 2 * q0 + o0, f1 = 2 * q1 + o1, f2 = 2 * q2 + o2;
            const float a = b.ad(f0, f1, f2);
            if (a != 0.0f) {
              const int p = b.zp(f0, f1, f2);
              const float Az = __fadd_rn(__fmul_rn(a, b.zs[p]), res_nsum(b, p));
              acc = __fadd_rn(acc, __fsub_rn(b.rs[b.ri(f0, f1, f2)], Az));
            }
          }
      const float rv = __fmul_rn(A.rho, acc);
      if (last) {
        const int g = (((b.o0 >> 1) + q0) * cn1 + ((b.o1 >> 1) + q1)) * cn2 + ((b.o2 >> 1) + q2);
        __stcg(A.rc + g, rv);
      } else {
        // a non-FLUID coarse cell keeps rs = 0: its unmasked z
        c.rs[j] = c.ad(q0, q1, q2) != 0.0f ? rv : 0.0f;
      }
    }
    __syncthreads();
  }

  // ---- the coarse levels in CTA 0 -------------------------------------------------
  cl.sync();  // level lb's r is complete
  if (rank == 0) coarse_vcycle<float, false>(A.coarse, smem + (size_t)A.coff * 4);
  cl.sync();  // level lb's z is complete

  // ---- prolongation and post-smoothing, coarsest to finest -----------------------
  for (int i = nlev - 1; i >= 0; --i) {
    const RB b = res_brick(A, i, sm, rank);
    const RNb nb = res_nbrs(b, A, rank);
    const int cells = b.B0 * b.B1 * b.B2;
    const bool last = i + 1 == nlev;
    RB c;
    if (!last) c = res_brick(A, i + 1, sm, rank);
    const int cn1 = b.n1 >> 1, cn2 = b.n2 >> 1;
    // prolongation (mgpcg.py:120-123): every cell += the parent's unmasked z
#pragma unroll 4
    for (int j = threadIdx.x; j < cells; j += blockDim.x) {
      const int c2 = j & (b.B2 - 1), c1 = (j >> b.l2) & (b.B1 - 1), c0 = j >> (b.l1 + b.l2);
      const int q0 = c0 >> 1, q1 = c1 >> 1, q2 = c2 >> 1;
      float zc;
      if (last) {
        zc = __ldcg(A.zc + (((b.o0 >> 1) + q0) * cn1 + ((b.o1 >> 1) + q1)) * cn2 + ((b.o2 >> 1) + q2));
      } else {
        const int qr = (((q0 << c.l1) + q1) << c.l2) + q2;
        zc = c.ad(q0, q1, q2) != 0.0f ? c.zs[c.zp(q0, q1, q2)] : c.rs[qr];
      }
      const float v = __fmul_rn(A.pi, zc);
      if (b.ad(c0, c1, c2) != 0.0f) {
        const int p = b.zp(c0, c1, c2);
        const float w = __fadd_rn(b.zs[p], v);
        b.zs[p] = w;
        res_push(b, nb, c0, c1, c2, w);
      } else {
        b.rs[j] = __fadd_rn(b.rs[j], v);
      }
    }
    // post-smoothing: colours 1, 0, 1, 0 ... (mgpcg.py:144-147), each after
    // the rings of the colour smoothed last (both after the prolongation)
    for (int m = 1; m <= A.ns; ++m) {
      cl.sync();
      res_smooth(b, nb, m & 1);
    }
    __syncthreads();
  }

  // ---- z of level lp ---------------------------------------------------------------
  {
    const RB b = res_brick(A, 0, sm, rank);
    const int cells = b.B0 * b.B1 * b.B2;
#pragma unroll 4
    for (int j = threadIdx.x; j < cells; j += blockDim.x) {
      const int c2 = j & (b.B2 - 1), c1 = (j >> b.l2) & (b.B1 - 1), c0 = j >> (b.l1 + b.l2);
      A.z0[b.gi(c0, c1, c2)] = b.ad(c0, c1, c2) != 0.0f ? b.zs[b.zp(c0, c1, c2)] : b.rs[j];
    }
  }
  cl.sync();  // the neighbours' last ring reads are done
}

}  // namespace mg
