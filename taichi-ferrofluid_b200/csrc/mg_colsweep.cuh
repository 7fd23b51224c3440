// Column-register streamed sweeps of the fused V-cycle (label-uniform 3D
// operator): the same smoothing, restriction and prolongation as k_sweep
// (mg_sweep.cuh), with the same float32 operations in the same order, laid
// out for the B200 instead of around a shared-memory ring of every array.
//
// A block owns a (TY x TX) tile of columns plus a halo (NS rows, HX >= NS
// columns rounded up for 16-byte TMA coordinates) and a chunk [z0, z1) of
// planes along axis 0, streamed plane by plane (temporal blocking: half sweep
// m acts on the plane `shift(m)` behind the newest, so it sees its
// neighbours after half sweep m-1, as in mgpcg.py:125-148).
//
// * Thread -> a y-pair of columns (x, rows 2i and 2i+1).  The pair's two cells
//   have opposite colours in every plane, so each half sweep updates exactly
//   one of them: all lanes work.  A plane's active cell is the one whose
//   x + y has the parity of the plane step, the same for every half sweep of
//   a step, so it is fixed per unrolled step (A at even steps, B at odd).
// * Each thread keeps its two columns' z, r and Adiag for the planes in
//   flight in REGISTERS (NS + 2 planes), so the neighbours along axis 0 and
//   the pair's own other cell never touch shared memory; only the three
//   in-plane neighbours (x - 1, x + 1, the row outside the pair) are read from
//   a shared z plane that each thread publishes its updates into.
// * The half sweeps of one step touch disjoint planes and read in-plane
//   neighbours published in the previous step, so a step needs ONE block
//   barrier, not one per half sweep.
// * r, Adiag (and POST's input z) arrive by TMA (cp.async.bulk.tensor, 3D
//   tile loads of the region plane, each block its own) into a ring of NS + 2
//   shared slots, NS + 1 planes ahead of the one being smoothed, completed on
//   one mbarrier per slot.  Out-of-grid boxes are zero-filled, which makes
//   those cells non-FLUID (Adiag 0) with z 0: rule H1 with no bounds checks.
//   Every wait is bounded; a wait that runs out sets Control::wait_timeout
//   and the block leaves the chunk (the solve then reports MG_SOLVE_TIMEOUT).
// * The restriction's 2 x 2 x 2 children sum in the reference oracle's order:
//   the x-partner's two residuals come by warp shuffle (the partner is the
//   adjacent lane), the two planes from consecutive steps.
#pragma once
#include <cuda.h>

#include "mg_fused.cuh"

namespace mg {

// ---- shared-memory barrier and TMA primitives (PTX) ----------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// A wait that gives up after about a second (kWaitCycles SM clocks).
constexpr long long kWaitCycles = 2000000000LL;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > kWaitCycles) return false;
  return true;
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y,
                                            int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
      : "memory");
}

// A shared-memory load the compiler may schedule freely within a plane step
// (no memory clobber).  Its address comes from launder() after the step's
// barrier, so it is never hoisted above that barrier; it is used only for
// cells no thread writes during the step.
__device__ __forceinline__ float lds_free(uint32_t addr) {
  float v;
  asm("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(addr));
  return v;
}
__device__ __forceinline__ uint32_t launder(uint32_t a) {
  asm volatile("" : "+r"(a));
  return a;
}

// ---- shape of one instantiation -------------------------------------------------------
template <typename ST, int NS, int TX, int TY>
struct ColGeom {
  // x halo of the TMA box: NS rounded up so that the box's first column is a
  // multiple of 16 bytes for every array (4 float32 / 8 16-bit cells); the
  // threads cover only NS columns of it (the rest is loaded, never used)
  static constexpr int HB = (sizeof(ST) == 4 && NS <= 4) ? 4 : 8;
  static constexpr int HX = NS;              // x halo of the threads' region
  static constexpr int RXB = TX + 2 * HB;    // box columns (TMA slots)
  static constexpr int RX = TX + 2 * HX;     // region columns (threads)
  static constexpr int RY = TY + 2 * NS;     // region rows (even)
  static constexpr int PLB = RXB * RY;       // cells of a box plane
  static constexpr int PAIRS = RX * (RY / 2);
  static constexpr int NT = PAIRS;
  static constexpr int W = NS + 2;           // planes in registers = TMA ring slots = shared z planes
  // a shared z plane holds the region plus a one-cell border, so every cell's
  // four in-plane neighbours are at fixed offsets (the border feeds only halo
  // cells that are never smoothed)
  static constexpr int ZX = RX + 2, ZY = RY + 2;
  static constexpr int ZPL = (ZX * ZY + 31) / 32 * 32;                     // floats of a shared z plane
  static constexpr int SLOT_R = (PLB * 4 + 127) / 128 * 128;               // r (float32 or ST)
  static constexpr int SLOT_S = (PLB * (int)sizeof(ST) + 127) / 128 * 128;  // Adiag, input z (ST)
  static constexpr int slot_bytes(bool pre) { return SLOT_R + SLOT_S * (pre ? 1 : 2); }
  static constexpr size_t smem(bool pre) {
    return 128 /* alignment */ + 128 /* mbarriers */ + (size_t)W * slot_bytes(pre) + (size_t)W * ZPL * 4;
  }
  static_assert(TX % 8 == 0 && TY % 2 == 0 && NS % 2 == 0, "even pairs, 16-byte TMA rows");
  static_assert(PAIRS % 32 == 0 && (TX * (TY / 2)) % 32 == 0, "whole warps of pairs, interior warps first");
  static_assert(RXB <= 256 && RY <= 256, "TMA box extents");
  static_assert(W <= 16, "mbarriers in 128 bytes");
};

// One red-black update of a label-uniform cell from its six neighbours: the
// two along axis 0, the two along the rows, the two along the fastest axis.
// Exact: the reference's order (mgpcg.py:96-109) in float32, z = (r - sum_k
// (-s) z_nb) / Adiag with six products, the axis pairs summed in turn and an
// IEEE division.  FAST (16-bit grids): z = (r + s * sum z_nb) / Adiag with the
// sum as a tree, one FMA and the approximate reciprocal.
template <bool FAST>
__device__ __forceinline__ float smooth_cell(float ms, float s, float r, float a, float z0m, float z0p, float z1m,
                                             float z1p, float z2m, float z2p) {
  if constexpr (FAST) {
    const float sum = __fadd_rn(__fadd_rn(__fadd_rn(z0m, z0p), __fadd_rn(z1m, z1p)), __fadd_rn(z2m, z2p));
    return __fdividef(fmaf(s, sum, r), a);
  } else {
    // (the reference's sum starts from 0; 0 + x == x up to the sign of a zero)
    float ret = __fadd_rn(__fmul_rn(ms, z0m), __fmul_rn(ms, z0p));
    ret = __fadd_rn(ret, __fadd_rn(__fmul_rn(ms, z1m), __fmul_rn(ms, z1p)));
    ret = __fadd_rn(ret, __fadd_rn(__fmul_rn(ms, z2m), __fmul_rn(ms, z2p)));
    return div_pos(__fsub_rn(r, ret), a);
  }
}

// r - A z of one label-uniform cell (mgpcg.py:111-118), the same two forms.
template <bool FAST>
__device__ __forceinline__ float residual_cell(float ms, float s, float r, float a, float z, float z0m, float z0p,
                                               float z1m, float z1p, float z2m, float z2p) {
  if constexpr (FAST) {
    const float sum = __fadd_rn(__fadd_rn(__fadd_rn(z0m, z0p), __fadd_rn(z1m, z1p)), __fadd_rn(z2m, z2p));
    return fmaf(-a, z, fmaf(s, sum, r));
  } else {
    float ret = __fadd_rn(__fmul_rn(ms, z0m), __fmul_rn(ms, z0p));
    ret = __fadd_rn(ret, __fadd_rn(__fmul_rn(ms, z1m), __fmul_rn(ms, z1p)));
    ret = __fadd_rn(ret, __fadd_rn(__fmul_rn(ms, z2m), __fmul_rn(ms, z2p)));
    return __fsub_rn(r, __fadd_rn(__fmul_rn(a, z), ret));
  }
}

// ---------------------------------------------------------------------------
// k_colsweep: PRE (z = 0, 2 pre_post half sweeps in colour order 0,1,..., then
// the restriction r[l+1] = rho * sum of the children's r - A z and z[l+1] = 0)
// or POST (z += pi * z[l+1][I/2], then half sweeps in colour order 1,0,...),
// with the level-0 POST also summing z.r for the PCG loop (A.zr >= 0).
//
// The step body is written for few instructions per cell: shared-memory
// pointers fixed per thread (the planes at immediate offsets), 32-bit cell
// indices, plane parities known at compile time (chunks start on even
// planes), and one thread that waits for the next plane's loads before the
// step's block barrier.
// ---------------------------------------------------------------------------
//
// colsweep_body is one block's work: block `bid` of the `nb` blocks of a
// level's launch (k_colsweep: the launch itself; k_bt_colsweep: one
// instance's blocks inside a batched launch).
template <typename ST, int NS, int TX, int TY, bool PRE>
__device__ __forceinline__ void colsweep_body(const SweepArgs<ST>& A, Control* flag, const CUtensorMap* tm_r,
                                              const CUtensorMap* tm_ad, const CUtensorMap* tm_zin, int bid,
                                              int nb) {
  using G = ColGeom<ST, NS, TX, TY>;
  constexpr int HX = G::HX, RX = G::RX, W = G::W, NT = G::NT, ZPL = G::ZPL, ZX = G::ZX;
  constexpr int RXB = G::RXB, XOFF = G::HB - G::HX;  // box columns; box column of region column 0
  // the mixed form (16-bit grids) needs no bit-exact float32: a neighbour-sum
  // tree, one FMA and the approximate reciprocal instead of six products,
  // five dependent sums and an IEEE division
  constexpr bool FAST = sizeof(ST) != 4;
  constexpr int SLOT = G::slot_bytes(PRE);
  constexpr int D = PRE ? NS - 1 : NS;  // steps from a plane's load to its final z
  constexpr int NI = TX * (TY / 2), NB = (NS / 2) * RX;

  extern __shared__ __align__(128) unsigned char smem_raw[];
  // 128-byte aligned by pointer arithmetic on the shared array (the compiler
  // keeps shared-space loads and stores)
  unsigned char* smem = smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
  unsigned char* slots = smem + 128;
  float* zs = reinterpret_cast<float*>(slots + W * SLOT);
  __shared__ int abort_flag;

  const FLevel<ST>& F = A.f;
  const int n0 = F.n[0], n1 = F.n[1], n2 = F.n[2];
  // one wave of blocks: tile t is cut into q or q + 1 chunks of nearly equal
  // even length (the first r tiles get q + 1; the host launches
  // ntile <= nb <= ntile * n0 / 2 blocks)
  const int ntile = A.tiles_x * A.tiles_y;
  const int nq = nb / ntile, nr = nb % ntile;
  int tile, cid, nch;
  if (bid < nr * (nq + 1)) {
    tile = bid / (nq + 1);
    cid = bid % (nq + 1);
    nch = nq + 1;
  } else {
    const int b2 = bid - nr * (nq + 1);
    tile = nr + b2 / nq;
    cid = b2 % nq;
    nch = nq;
  }
  const int tx0 = (tile % A.tiles_x) * TX;
  const int ty0 = (tile / A.tiles_x) * TY;
  const int z0 = (cid * n0 / nch) & ~1;  // even
  const int z1 = cid + 1 == nch ? n0 : ((cid + 1) * n0 / nch) & ~1;
  const int p_first = z0 - NS;        // even
  const int p_last = z1 + NS - 1;
  const int ox = tx0 - HX, oy = ty0 - NS;  // region origin (both even)
  const int bx = tx0 - G::HB;               // TMA box origin along x (16-byte aligned)
  const float sigma = A.r_f32 ? (float)A.ctl->scale_r : 1.0f;
  const float ms = -F.s;
  const float s_pos = F.s;
  const int pstride = n1 * n2;  // 32-bit cell indices (the host checks the level's size)
  const int ncx = A.nc[2], cps = A.nc[1] * A.nc[2];
  const bool r32 = sizeof(ST) == 4 || A.r_f32;
  const uint32_t tx_bytes =
      (uint32_t)(G::PLB * ((r32 ? 4 : (int)sizeof(ST)) + (int)sizeof(ST) * (PRE ? 1 : 2)));

  // ---- this thread's pair of columns ----------------------------------------------------
  // Interior first: threads [0, TX * TY / 2) hold the tile's own pairs, one
  // pair row of TX columns per TX threads (whole warps for TX = 32, 64); the
  // halo pairs follow (the top and bottom bands of NS / 2 pair rows, then the
  // left and right bands of HX columns).  A half sweep's active region shrinks
  // towards the tile, so halo warps fall idle as a whole instead of idling
  // lanes inside every warp; the residual runs on the interior warps only.
  const int t = threadIdx.x;
  int rx, pr2;
  if (t < NI) {
    pr2 = NS / 2 + t / TX;
    rx = HX + t % TX;
  } else if (t < NI + NB) {
    pr2 = (t - NI) / RX;
    rx = (t - NI) % RX;
  } else if (t < NI + 2 * NB) {
    pr2 = NS / 2 + TY / 2 + (t - NI - NB) / RX;
    rx = (t - NI - NB) % RX;
  } else {
    const int h = t - NI - 2 * NB;
    pr2 = NS / 2 + h / (2 * HX);
    const int k = h % (2 * HX);
    rx = k < HX ? k : TX + k;
  }
  const bool interior_warp = t < NI;  // warp-uniform
  const int gx = ox + rx, gy0 = oy + 2 * pr2;
  const int odd = rx & 1;                                    // gx parity (ox even)
  const int rowA = 2 * pr2 + odd, rowB = 2 * pr2 + 1 - odd;  // A: x + y even
  const int outA = odd ? rowA + 1 : rowA - 1;                // the row beyond the pair next to A
  const int outB = odd ? rowB - 1 : rowB + 1;
  float* const pA = zs + (rowA + 1) * ZX + rx + 1;  // own cells in shared z plane 0
  float* const pB = zs + (rowB + 1) * ZX + rx + 1;
  const float* const qA = zs + (outA + 1) * ZX + rx + 1;  // the out-of-pair row neighbours
  const float* const qB = zs + (outB + 1) * ZX + rx + 1;
  const uint32_t aPA = smem_addr(pA), aPB = smem_addr(pB), aQA = smem_addr(qA), aQB = smem_addr(qB);
  constexpr uint32_t PLB4 = ZPL * 4;  // bytes between shared z planes
  const int kA = rowA * RXB + rx + XOFF, kB = rowB * RXB + rx + XOFF;  // in a TMA slot
  const int dxr = max(max(HX - rx, rx - (HX + TX - 1)), 0);
  const int ringA = max(dxr, max(max(NS - rowA, rowA - (NS + TY - 1)), 0));
  const int ringB = max(dxr, max(max(NS - rowB, rowB - (NS + TY - 1)), 0));
  // n1 even and gy0 even: the pair's rows are both inside the grid or both outside
  const bool in_grid = gx >= 0 && gx < n2 && gy0 >= 0 && gy0 < n1;
  const bool ownA = in_grid && ringA == 0, ownB = in_grid && ringB == 0;
  const int giA = (oy + rowA) * n2 + gx, giB = (oy + rowB) * n2 + gx;
  // the coarse column of the pair (clamped into the grid: only in-grid cells use it)
  const int cc = (min(max(gy0, 0), n1 - 1) >> 1) * ncx + (min(max(gx, 0), n2 - 1) >> 1);

  float zA[W], zB[W], rA[W], rB[W], aA[W], aB[W];
#pragma unroll
  for (int j = 0; j < W; ++j) {
    zA[j] = 0.0f; zB[j] = 0.0f; rA[j] = 0.0f; rB[j] = 0.0f; aA[j] = 0.0f; aB[j] = 0.0f;
  }
  // POST: the coarse z of the pair's column for the plane pair (p, p + 1), p
  // even, read two steps before its use; planes outside the grid read a
  // clamped plane (their cells are not FLUID and never written)
  auto zc_of = [&](int p) -> float {
    const int h = min(max(p >> 1, 0), (n0 >> 1) - 1);
    return to_f<ST>(A.zc[h * cps + cc]);
  };
  float zc_next = PRE ? 0.0f : zc_of(p_first), zc_cur = 0.0f;
  float acc = 0.0f;      // restriction accumulator (PRE, even-x threads)
  double zr_acc = 0.0;   // z.r of the cells written (POST, A.zr >= 0)

  auto issue = [&](int p, int slot) {  // TMA loads of plane p into a ring slot (thread 0)
    unsigned char* sl = slots + slot * SLOT;
    mbar_expect_tx(&bar[slot], tx_bytes);
    tma_load_3d(sl, tm_r, &bar[slot], bx, oy, p);
    tma_load_3d(sl + G::SLOT_R, tm_ad, &bar[slot], bx, oy, p);
    if (!PRE) tma_load_3d(sl + G::SLOT_R + G::SLOT_S, tm_zin, &bar[slot], bx, oy, p);
  };

  if (t == 0) {
#pragma unroll
    for (int j = 0; j < W; ++j) mbar_init(&bar[j], 1);
    mbar_fence_init();
    abort_flag = 0;
  }
  // the border of every shared z plane (read only for halo cells never smoothed)
  for (int i = t; i < W * ZPL; i += NT) zs[i] = 0.0f;
  __syncthreads();
  int stop_p = p_first;  // the plane whose loads did not complete (abort)
  if (t == 0) {
    for (int k = 0; k < W - 1; ++k)
      if (p_first + k <= p_last) issue(p_first + k, k);
    if (!mbar_wait_bounded(&bar[0], 0u)) abort_flag = 1;
  }
  __syncthreads();

  bool aborted = abort_flag != 0;
  for (int P0 = p_first; P0 <= p_last && !aborted; P0 += W) {
    const int k0 = (P0 - p_first) / W;  // ring pass of this group of W planes
#pragma unroll
    for (int u = 0; u < W; ++u) {
      const int P = P0 + u;
      if (P > p_last) break;
      const int q = P - p_first;
      // this step's in-plane neighbour reads (planes written before the last barrier)
      const uint32_t sPA = launder(aPA), sPB = launder(aPB), sQA = launder(aQA), sQB = launder(aQB);
      // plane P + W - 1 into the slot of plane P - 1 (read before the last barrier)
      if (t == 0 && P + W - 1 <= p_last) issue(P + W - 1, (u + W - 1) % W);

      // ---- plane P (delivered: waited for before the last barrier) into the registers --
      {
        const unsigned char* sl = slots + u * SLOT;
        if (r32) {
          const float* sr = reinterpret_cast<const float*>(sl);
          rA[u] = sizeof(ST) == 4 ? sr[kA] : __fmul_rn(sigma, sr[kA]);
          rB[u] = sizeof(ST) == 4 ? sr[kB] : __fmul_rn(sigma, sr[kB]);
        } else {
          const ST* sr = reinterpret_cast<const ST*>(sl);
          rA[u] = to_f<ST>(sr[kA]);
          rB[u] = to_f<ST>(sr[kB]);
        }
        const ST* sa = reinterpret_cast<const ST*>(sl + G::SLOT_R);
        aA[u] = to_f<ST>(sa[kA]);
        aB[u] = to_f<ST>(sa[kB]);
        if constexpr (PRE) {
          // the first half sweep is pointwise (z = 0 before it): z = r / Adiag on
          // the colour-0 cell, the one active in this step (A: even P)
          if ((u & 1) == 0) {
            zA[u] = aA[u] != 0.0f ? (FAST ? __fdividef(rA[u], aA[u]) : div_pos(rA[u], aA[u])) : 0.0f;
            zB[u] = 0.0f;
          } else {
            zB[u] = aB[u] != 0.0f ? (FAST ? __fdividef(rB[u], aB[u]) : div_pos(rB[u], aB[u])) : 0.0f;
            zA[u] = 0.0f;
          }
        } else {
          if ((u & 1) == 0) {  // the coarse value of planes (P, P + 1); prefetch (P + 2, P + 3)
            zc_cur = zc_next;
            zc_next = zc_of(P + 2);
          }
          const ST* si = reinterpret_cast<const ST*>(sl + G::SLOT_R + G::SLOT_S);
          const float c = __fmul_rn(A.pi, zc_cur);
          const float fa = __fadd_rn(to_f<ST>(si[kA]), c);
          const float fb = __fadd_rn(to_f<ST>(si[kB]), c);
          zA[u] = aA[u] != 0.0f ? fa : 0.0f;
          zB[u] = aB[u] != 0.0f ? fb : 0.0f;
          // an owned non-FLUID cell is never smoothed: its output is this value
          if (P >= z0 && P < z1) {
            const int base = P * pstride;
            if (ownA && aA[u] == 0.0f) F.z[base + giA] = from_f<ST>(fa);
            if (ownB && aB[u] == 0.0f) F.z[base + giB] = from_f<ST>(fb);
          }
        }
        pA[u * ZPL] = zA[u];
        pB[u * ZPL] = zB[u];
      }

      // ---- half sweeps: m on the plane shift(m) behind P ------------------------------
#pragma unroll
      for (int m = PRE ? 2 : 1; m <= NS; ++m) {
        const int s = PRE ? m - 1 : m;      // planes behind P
        const int j = (u - s + 2 * W) % W, jm = (j + W - 1) % W, jp = (j + 1) % W;
        if (q < s + 1) continue;            // the plane below was not loaded
        // cells at ring distance <= NS - s from the tile are needed after this sweep
        // (a branch: most warps of a scene's air or solid skip the division)
        if ((u & 1) == 0) {
          if (ringA <= NS - s && aA[j] != 0.0f) {
            const float v = smooth_cell<FAST>(ms, s_pos, rA[j], aA[j], zA[jm], zA[jp], lds_free(sQA + j * PLB4),
                                              zB[j], lds_free(sPA + j * PLB4 - 4), lds_free(sPA + j * PLB4 + 4));
            zA[j] = v;
            pA[j * ZPL] = v;
          }
        } else {
          if (ringB <= NS - s && aB[j] != 0.0f) {
            const float v = smooth_cell<FAST>(ms, s_pos, rB[j], aB[j], zB[jm], zB[jp], lds_free(sQB + j * PLB4),
                                              zA[j], lds_free(sPB + j * PLB4 - 4), lds_free(sPB + j * PLB4 + 4));
            zB[j] = v;
            pB[j * ZPL] = v;
          }
        }
      }

      // ---- the finished plane P - D ------------------------------------------------------
      {
        const int pw = P - D;
        if (pw >= z0 && pw < z1) {
          const int jw = (u - D + 2 * W) % W;
          const int base = pw * pstride;
          if constexpr (PRE) {  // non-FLUID cells hold z = 0
            if (ownA) F.z[base + giA] = from_f<ST>(zA[jw]);
            if (ownB) F.z[base + giB] = from_f<ST>(zB[jw]);
          } else {
            const bool wa = ownA && aA[jw] != 0.0f, wb = ownB && aB[jw] != 0.0f;
            if (wa) F.z[base + giA] = from_f<ST>(zA[jw]);
            if (wb) F.z[base + giB] = from_f<ST>(zB[jw]);
            if (A.zr >= 0) {
              zr_acc += wa ? (double)zA[jw] * (double)rA[jw] : 0.0;
              zr_acc += wb ? (double)zB[jw] * (double)rB[jw] : 0.0;
            }
          }
        }
      }

      // ---- PRE: residual of plane P - NS and restriction (interior warps) ---------------
      if constexpr (PRE) {
        const int pr = P - NS;  // parity of u (P0 and NS even)
        if (interior_warp && pr >= z0 && pr < z1) {
          const int jr = (u - NS + 2 * W) % W, jrm = (jr + W - 1) % W, jrp = (jr + 1) % W;
          const bool fA = in_grid && aA[jr] != 0.0f, fB = in_grid && aB[jr] != 0.0f;
          float vA = 0.0f, vB = 0.0f;
          if (fA)
            vA = residual_cell<FAST>(ms, s_pos, rA[jr], aA[jr], zA[jr], zA[jrm], zA[jrp], lds_free(sQA + jr * PLB4),
                                     zB[jr], lds_free(sPA + jr * PLB4 - 4), lds_free(sPA + jr * PLB4 + 4));
          if (fB)
            vB = residual_cell<FAST>(ms, s_pos, rB[jr], aB[jr], zB[jr], zB[jrm], zB[jrp], lds_free(sQB + jr * PLB4),
                                     zA[jr], lds_free(sPB + jr * PLB4 - 4), lds_free(sPB + jr * PLB4 + 4));
          // rows y0 (even) and y1 of this column; the x + 1 column is the next lane
          const float v0 = odd ? vB : vA, v1 = odd ? vA : vB;
          const bool f0 = odd ? fB : fA, f1 = odd ? fA : fB;
          const float p0 = __shfl_xor_sync(0xffffffffu, v0, 1);
          const float p1 = __shfl_xor_sync(0xffffffffu, v1, 1);
          const unsigned pf = __shfl_xor_sync(0xffffffffu, (unsigned)f0 | ((unsigned)f1 << 1), 1);
          // children in the order (y0, x0), (y0, x1), (y1, x0), (y1, x1), plane by
          // plane, FLUID children only; even-x lanes keep the sum
          if ((u & 1) == 0) acc = 0.0f;
          acc = f0 ? __fadd_rn(acc, v0) : acc;
          acc = (pf & 1u) ? __fadd_rn(acc, p0) : acc;
          acc = f1 ? __fadd_rn(acc, v1) : acc;
          acc = (pf & 2u) ? __fadd_rn(acc, p1) : acc;
          if ((u & 1) == 1 && !odd && in_grid) {
            const int gc = (pr >> 1) * cps + cc;
            A.rc[gc] = from_f<ST>(__fmul_rn(A.rho, acc));
            A.zc[gc] = from_f<ST>(0.0f);
          }
        }
      }

      // ---- the next plane's loads, then the step's barrier ------------------------------
      if (t == 0 && P + 1 <= p_last) {
        const uint32_t par = (uint32_t)((k0 + (u + 1 == W ? 1 : 0)) & 1);
        if (!mbar_wait_bounded(&bar[(u + 1) % W], par)) abort_flag = 1;
      }
      __syncthreads();
      if (abort_flag) {
        aborted = true;
        stop_p = P + 1;
        break;
      }
    }
  }

  if (aborted && t == 0) {
    // a TMA load did not complete within the bound: flag it, then wait
    // (bounded) for this block's loads still in flight before leaving
    atomicOr(&flag->wait_timeout, 1);
    const int last_issued = min(stop_p + W - 2, p_last);  // issued at step stop_p - 1 (or before the loop)
    for (int p = stop_p; p <= last_issued; ++p) {
      const int k = p - p_first;
      mbar_wait_bounded(&bar[k % W], (uint32_t)((k / W) & 1));
    }
  }
  if constexpr (!PRE) {
    if (A.zr >= 0) {  // the reduction and epilogue of k_zr4 (mgpcg.py:161-166, 197-202)
      __shared__ double sh[32];
      double tot;
      Control* ctl = A.zr_ctl;
      if (last_block_total_at<NT>(zr_acc, A.zr_partials, &ctl->counter[1], sh, &tot, bid, nb) &&
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

template <typename ST, int NS, int TX, int TY, bool PRE, int MINB>
__global__ void __launch_bounds__(ColGeom<ST, NS, TX, TY>::NT, MINB)
    k_colsweep(SweepArgs<ST> A, Control* flag, const __grid_constant__ CUtensorMap tm_r,
               const __grid_constant__ CUtensorMap tm_ad, const __grid_constant__ CUtensorMap tm_zin) {
  pdl_enter();
  colsweep_body<ST, NS, TX, TY, PRE>(A, flag, &tm_r, &tm_ad, &tm_zin, (int)blockIdx.x, (int)gridDim.x);
}

}  // namespace mg
