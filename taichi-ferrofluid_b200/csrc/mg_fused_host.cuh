// Host side of the fused V-cycle: per-level launch shapes, the split between
// streamed levels and the block-resident coarse levels, and the launches.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>

#include "mg_sweep.cuh"
#include "mg_colsweep.cuh"
#include "mg_coarse.cuh"
#include "mg_resident.cuh"

namespace mg {

// Shared memory one block may use (B200: 227 KB per block).
constexpr size_t kSmemLimit = 227 * 1024;
// Padded cells the block-resident coarse V-cycle may hold: 12 bytes each
// (masked z, r / unmasked z, Adiag as float32), under 200 KB.
constexpr int kCoarseMaxCells = 16384;
// The whole-domain stored form adds the dim coupling arrays (24 bytes a cell
// in 3D): 8192 cells, under 200 KB.
constexpr int kCoarseMaxCellsSto = 8192;

// Cells of a level padded by one ring (2D: no padding along the absent axis).
inline long long padded_cells(const Geom& g) {
  return (long long)(g.n[0] + 2) * (g.n[1] + 2) * (g.dim == 3 ? g.n[2] + 2 : 1);
}

struct TileShape {
  int tx, ty, nt, k;  // tile columns (x, y), threads, planes per step
};

// Launch shape of the streamed levels: a tile of ty x tx columns per block,
// k planes per pipeline step.
#ifndef MG_TILE3_K
#define MG_TILE3_K 2
#endif
#ifndef MG_TILE3_TX
#define MG_TILE3_TX 32
#endif
#ifndef MG_TILE3_TY
#define MG_TILE3_TY 16
#endif
#ifndef MG_TILE3_NT
#define MG_TILE3_NT 512
#endif
constexpr TileShape kTile3 = {MG_TILE3_TX, MG_TILE3_TY, MG_TILE3_NT, MG_TILE3_K};
constexpr TileShape kTile2 = {128, 1, 128, 4};
// the whole-domain stored form stages twice the bytes per cell: a smaller
// tile keeps two blocks per SM
constexpr TileShape kTile3S = {32, 8, 256, 2};
inline TileShape tile_for(int dim, bool sto = false) { return sto ? kTile3S : (dim == 3 ? kTile3 : kTile2); }

// z, r, Adiag (and, stored form, the dim couplings) as float32 for a ring of
// k + ns + 1 planes of tile + halo ns (rounded up to 4 along the fastest
// axis, as k_sweep lays it out).  A one-step launch (k = the whole chunk of 2
// planes + 2 ns halo planes) needs no ring: k planes.
inline size_t sweep_smem(int dim, int ns, TileShape t, bool one_step = false, bool sto = false) {
  const int RX = t.tx + 2 * ((ns + 3) & ~3);
  const int RY = dim == 3 ? t.ty + 2 * ns : 1;
  const int W = one_step ? t.k : t.k + ns + 1;
  return (size_t)W * RX * RY * (12 + (sto ? 4 * dim : 0));
}

// Tile shapes of the column-register sweep (k_colsweep) a streamed level may
// run instead of k_sweep: (TX, TY) columns and the blocks per SM its launch
// bounds aim at.  Index 0 is k_sweep.
struct ColShape {
  int tx, ty, minb;
};
constexpr ColShape kColShapes[] = {{0, 0, 0}, {32, 16, 2}, {32, 32, 1}, {64, 16, 1}};
constexpr int kColShapeCount = 4;

struct FusedPlan {
  bool valid = false;
  bool sto = false;                // whole-domain stored form (else label-uniform)
  // per streamed level: run the reference's per-kernel sweeps, restriction and
  // prolongation instead of the streamed kernel (chosen by measurement: on
  // the large levels of the stored form the per-kernel passes are faster)
  bool split[kMaxLevels] = {};
  // per streamed level and direction (bit 0 PRE, bit 1 POST): one plane per
  // pipeline step instead of the tile's two (3D label-uniform float32 only;
  // chosen by measurement)
  unsigned char step1[kMaxLevels] = {};
  // per streamed level: blocks per SM assumed when its grid is sized, beyond
  // those that fit one SM's shared memory (shorter chunks, more blocks; chosen
  // by measurement: 1 extra is faster for the 256^3 level-0 sweeps, slower at
  // 128^3)
  unsigned char grid_extra[kMaxLevels] = {};
  // per streamed level: 0 = k_sweep, k = k_colsweep with kColShapes[k]
  // (chosen by measurement; possible where col_ok holds)
  unsigned char col[kMaxLevels] = {};
  int col_per_sm[kColShapeCount] = {};  // resident blocks of each shape (occupancy)
  int per_sm = 1, num_sms = 148;
  int lc = 0;                      // first level of the block-resident coarse solve
  int dim = 3, ns = 4, storage = 0;
  int chunk[kMaxLevels], tiles_x[kMaxLevels], tiles_y[kMaxLevels], blocks[kMaxLevels];
  TileShape tile;
  CoarseArgs coarse;
  size_t coarse_smem = 0;
  int coarse_threads = 512;
  float kappa = 1.0f, rho = 1.0f, pi = 1.0f;
  float s[kMaxLevels];
  // cluster-resident V-cycle of levels [res_lp, L) (mg_resident.cuh): possible
  // (res_ok) and chosen (res); bricks for [res_lp, res_lb), CTA 0 below
  bool res_ok = false, res = false;
  int res_lp = 0, res_lb = 0, res_blocks = 0;
  size_t res_smem = 0;
  int res_threads = kResThreads;  // k_resident's CTA size (kResThreads or 512)
  ResArgs res_args;
  // z.r of the PCG loop inside the level-0 POST sweep while the plan launches
  // a PCG part (-1: not now; 0 / 1: before / inside the loop)
  int zr_mode = -1;
  Control* zr_ctl = nullptr;
  double* zr_partials = nullptr;
};

// Grid of streamed level l: tiles of the plane times chunks of planes along
// the slowest axis, enough blocks to fill every SM with the blocks that fit
// its shared memory plus `extra` (then a block's chunk is shorter).  Small
// levels are latency-bound: short chunks (more blocks, shorter serial plane
// chains) beat the extra halo planes they load.  The column kernel takes
// exactly that many blocks (no partial last wave) and cuts each tile's planes
// into chunks of nearly equal length itself.
inline void level_grid(FusedPlan* F, const Geom& g, int l, int extra) {
  const int nx = F->dim == 3 ? g.n[2] : g.n[1];
  const int ny = F->dim == 3 ? g.n[1] : 1;
  const int c = F->col[l];
  const int tx = c ? kColShapes[c].tx : F->tile.tx, ty = c ? kColShapes[c].ty : F->tile.ty;
  const int per_sm = c ? (F->col_per_sm[c] > 0 ? F->col_per_sm[c] : 1) : F->per_sm;
  F->tiles_x[l] = (nx + tx - 1) / tx;
  F->tiles_y[l] = F->dim == 3 ? (ny + ty - 1) / ty : 1;
  const long long tiles = (long long)F->tiles_x[l] * F->tiles_y[l];
  const long long target = (long long)(per_sm + extra) * F->num_sms;
  if (c) {
    // k_colsweep: exactly `target` blocks (whole waves), each tile cut into
    // chunks of nearly equal even length (at least 2 planes)
    long long nb = std::min(target, tiles * (g.n[0] / 2));
    nb = std::max(nb, tiles);
    F->blocks[l] = (int)nb;
    F->chunk[l] = (int)((g.n[0] * tiles + nb - 1) / nb);  // the mean chunk
    F->grid_extra[l] = (unsigned char)extra;
    return;
  }
  long long chunk = (long long)g.n[0] * tiles / target;
  if (chunk < 2) chunk = 2;
  chunk &= ~1LL;
  if (chunk > g.n[0]) chunk = g.n[0];
  if (chunk < 2) chunk = 2;
  F->chunk[l] = (int)chunk;
  F->blocks[l] = (int)(tiles * ((g.n[0] + chunk - 1) / chunk));
  F->grid_extra[l] = (unsigned char)extra;
}

// Chooses the launch shapes.  Needs pre_post in 1..3 and either every level
// in label-uniform form, or (the whole-domain stored form: float32 grids, 3D,
// pre_post 1..2) every level whole-domain - every cell FLUID with a nonzero
// diagonal.  Returns false (stored-coefficient kernels) otherwise.
inline bool make_fused_plan(const Level* lv, int L, int dim, int pre_post, int bottom, int storage,
                            const int* op_form, const int* whole, const float* offdiag, int num_sms, FusedPlan* F) {
  F->valid = false;
  F->sto = false;
  F->res_ok = false;
  F->res = false;
  for (int l = 0; l < kMaxLevels; ++l) {
    F->split[l] = false;
    F->step1[l] = 0;
    F->grid_extra[l] = 0;
    F->col[l] = 0;
  }
  bool uniform = true, all_whole = true;
  for (int l = 0; l < L; ++l) {
    uniform = uniform && op_form[l] == 1;
    all_whole = all_whole && whole[l] == 1;
  }
  if (pre_post < 1 || pre_post > 3) return false;
  if (!uniform) {
    if (!(all_whole && storage == MG_STORE_F32 && dim == 3 && pre_post <= 2)) return false;
    F->sto = true;
  }
  F->dim = dim;
  F->ns = 2 * pre_post;
  F->storage = storage;
  F->tile = tile_for(dim, F->sto);
  // first level whose sub-hierarchy fits one block
  const long long cap = F->sto ? kCoarseMaxCellsSto : kCoarseMaxCells;
  long long tot = 0;
  int lc = L;
  for (int l = L - 1; l >= 0; --l) {
    tot += padded_cells(lv[l].g);
    if (tot > cap) break;
    lc = l;
  }
  if (lc == L) return false;  // even the bottom level is too big for one block
  F->lc = lc;
  // scale factors (powers of two): kappa ~ 1/s_0 for 16-bit grids
  F->kappa = 1.0f;
  F->rho = 1.0f;
  F->pi = 1.0f;
  if (storage != MG_STORE_F32) {
    float s0 = 0.0f;
    for (int l = 0; l < L && s0 == 0.0f; ++l) s0 = offdiag[l];
    if (s0 > 0.0f && std::isfinite(s0)) F->kappa = std::ldexp(1.0f, -(int)std::lround(std::log2((double)s0)));
    F->rho = std::ldexp(1.0f, -dim);
    F->pi = std::ldexp(1.0f, dim);
  }
  for (int l = 0; l < L; ++l) F->s[l] = offdiag[l] * F->kappa;
  // streamed levels: the 4-wide groups need the fastest extent to be a
  // multiple of 4 (then a group is wholly inside or wholly outside the grid)
  const size_t smem = sweep_smem(dim, F->ns, F->tile, false, F->sto);
  F->per_sm = (int)(kSmemLimit / (smem + 1024)) < 1 ? 1 : (int)(kSmemLimit / (smem + 1024));
  F->num_sms = num_sms;
  for (int l = 0; l < lc; ++l) {
    const Geom& g = lv[l].g;
    const int nx = dim == 3 ? g.n[2] : g.n[1];
    if (nx % 4 != 0) return false;
    level_grid(F, g, l, 0);
  }
  // block-resident coarse levels
  CoarseArgs& C = F->coarse;
  C.dim = dim;
  C.nlev = L - lc;
  C.pre_post = pre_post;
  C.bottom = bottom;
  int off = 0;
  for (int i = 0; i < C.nlev; ++i) {
    const Geom& g = lv[lc + i].g;
    C.n[i][0] = g.n[0];
    C.n[i][1] = g.n[1];
    C.n[i][2] = g.n[2];
    C.off[i] = off;
    off += (int)padded_cells(g);
    C.s[i] = F->s[lc + i];
    C.Ad[i] = lv[lc + i].Adiag_s;
    for (int k = 0; k < 3; ++k) C.Ax[i][k] = k < dim ? lv[lc + i].Ax[k] : nullptr;
  }
  C.total = off;
  C.r0 = lv[lc].r;
  C.z0 = lv[lc].z;
  C.r_f32 = lc == 0;
  C.rho = F->rho;
  C.pi = F->pi;
  F->coarse_smem = (size_t)off * (12 + (F->sto ? 4 * dim : 0));
  // 1024 threads: the upper coarse levels' phases take 1-2 cells per thread;
  // the bottom level's cells sit in the first threads' registers
  F->coarse_threads = kCoarseThreads;
  F->valid = true;
  return true;
}

// Brick decomposition for the cluster-resident V-cycle (mg_resident.cuh) of a
// label-uniform float32 3D plan: the coarse levels [lb, L) for CTA 0 (the
// bottom level alone when the level above it splits into bricks, else one
// level more, and so on) and the first level lp in [lp_min, lp_max] whose
// levels [lp, lb) halve exactly and split into at most 16 bricks of
// power-of-two extents (at least 2^(lb - lp) a side) that fit one CTA's shared
// memory beside the coarse region; among those, the most bricks, then the
// fewest face cells.  The bricks' Adiag joins them in shared memory when it
// fits.  Fills F->res_* (res_ok); F->res stays as it was.
inline bool make_resident_plan(FusedPlan* F, const Level* lv, int L, int pre_post, int bottom, int lp_min,
                               int lp_max) {
  F->res_ok = false;
  if (!F->valid || F->sto || F->dim != 3 || F->storage != MG_STORE_F32 || L < 2) return false;
  for (int lb = L - 1; lb >= 1; --lb) {
    long long coarse_cells = 0;
    for (int l = lb; l < L; ++l) coarse_cells += padded_cells(lv[l].g);
    const long long coarse_floats = (3 * coarse_cells + 3) / 4 * 4;
    if (coarse_cells > kCoarseMaxCells) break;
    // the levels above the bricks run streamed, and only [0, lc) have
    // streamed launch shapes: the bricks start at lc at the latest
    for (int lp = lp_min; lp < lb && lp <= lp_max && lp <= F->lc; ++lp) {
      const int D = lb - lp;
      const Geom& g = lv[lp].g;
      bool halves = true;
      for (int l = lp + 1; l <= lb; ++l)
        for (int a = 0; a < 3; ++a) halves = halves && ((long long)lv[l].g.n[a] << (l - lp)) == g.n[a];
      if (!halves) continue;
      int emax[3], best[3] = {0, 0, 0};
      for (int a = 0; a < 3; ++a) {
        emax[a] = 0;
        while (((g.n[a] >> emax[a]) & 1) == 0 && emax[a] < 20) ++emax[a];
      }
      long long best_c = 0, best_faces = 0, best_fla = 0;
      for (int e0 = D; e0 <= emax[0]; ++e0)
        for (int e1 = D; e1 <= emax[1]; ++e1)
          for (int e2 = D; e2 <= emax[2]; ++e2) {
            const long long C = (long long)(g.n[0] >> e0) * (g.n[1] >> e1) * (g.n[2] >> e2);
            if (C > kResMaxCtas || C < 1) continue;
            long long fl = 0, fla = 0;  // without / with the bricks' Adiag
            for (int i = 0; i < D; ++i) {
              const long long b0 = 1LL << (e0 - i), b1 = 1LL << (e1 - i), b2 = 1LL << (e2 - i);
              fl += ((b0 + 2) * (b1 + 2) * (b2 + 2) + 3) / 4 * 4 + (b0 * b1 * b2 + 3) / 4 * 4;
              fla += (b0 * b1 * b2 + 3) / 4 * 4;
            }
            fla += fl;
            if ((size_t)(fl + coarse_floats) * 4 + 1024 > kSmemLimit) continue;
            const long long B0 = 1LL << e0, B1 = 1LL << e1, B2 = 1LL << e2;
            const long long faces = 2 * (B1 * B2 + B0 * B2 + B0 * B1);
            if (C > best_c || (C == best_c && faces < best_faces)) {
              best_c = C;
              best_faces = faces;
              best_fla = fla;
              best[0] = e0;
              best[1] = e1;
              best[2] = e2;
            }
          }
      if (best_c == 0) continue;
      ResArgs& R = F->res_args;
      R.nlev = D;
      for (int a = 0; a < 3; ++a) R.nb[a] = g.n[a] >> best[a];
      R.ns = F->ns;
      R.rho = F->rho;
      R.pi = F->pi;
      const bool sad = (size_t)(best_fla + coarse_floats) * 4 + 1024 <= kSmemLimit;
      int off = 0;
      for (int i = 0; i < D; ++i) {
        ResLevel& Q = R.lv[i];
        const Level& lev = lv[lp + i];
        for (int a = 0; a < 3; ++a) {
          Q.lb[a] = best[a] - i;
          Q.n[a] = lev.g.n[a];
        }
        const int b0 = 1 << Q.lb[0], b1 = 1 << Q.lb[1], b2 = 1 << Q.lb[2];
        Q.zoff = off;
        off += ((b0 + 2) * (b1 + 2) * (b2 + 2) + 3) / 4 * 4;
        Q.roff = off;
        off += (b0 * b1 * b2 + 3) / 4 * 4;
        Q.aoff = -1;
        if (sad) {
          Q.aoff = off;
          off += (b0 * b1 * b2 + 3) / 4 * 4;
        }
        Q.s = F->s[lp + i];
        Q.Ad = (const float*)lev.Adiag_s;
      }
      R.r0 = (const float*)lv[lp].r;
      R.z0 = (float*)lv[lp].z;
      R.rc = (float*)lv[lb].r;
      R.zc = (const float*)lv[lb].z;
      // the coarse levels [lb, L) laid out as the coarse block lays them out
      CoarseArgs& C = R.coarse;
      C = F->coarse;
      C.dim = 3;
      C.nlev = L - lb;
      C.pre_post = pre_post;
      C.bottom = bottom;
      int coff = 0;
      for (int i = 0; i < C.nlev; ++i) {
        const Geom& cg = lv[lb + i].g;
        for (int a = 0; a < 3; ++a) C.n[i][a] = cg.n[a];
        C.off[i] = coff;
        coff += (int)padded_cells(cg);
        C.s[i] = F->s[lb + i];
        C.Ad[i] = lv[lb + i].Adiag_s;
        for (int k = 0; k < 3; ++k) C.Ax[i][k] = lv[lb + i].Ax[k];
      }
      C.total = coff;
      C.r0 = lv[lb].r;
      C.z0 = lv[lb].z;
      C.r_f32 = 0;
      C.rho = F->rho;
      C.pi = F->pi;
      R.coff = off;
      R.smem_floats = off + (int)coarse_floats;
      F->res_lp = lp;
      F->res_lb = lb;
      F->res_blocks = (int)best_c;
      F->res_smem = (size_t)R.smem_floats * 4;
      F->res_ok = true;
      return true;
    }
  }
  return false;
}

// One launch of the cluster-resident V-cycle: one cluster of res_blocks CTAs.
inline cudaLaunchConfig_t resident_config(const FusedPlan& F, cudaStream_t s, cudaLaunchAttribute* at) {
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = F.res_blocks;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(F.res_blocks);
  cfg.blockDim = dim3(F.res_threads);
  cfg.dynamicSmemBytes = F.res_smem;
  cfg.stream = s;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cfg;
}

// The instantiation of k_resident for the plan's CTA size.
inline void (*res_kernel(const FusedPlan& F))(ResArgs) {
  return F.res_threads == 512 ? k_resident<512> : k_resident<kResThreads>;
}

inline cudaError_t resident_attributes(const FusedPlan& F) {
  cudaError_t e = cudaFuncSetAttribute(res_kernel(F), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)F.res_smem);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(res_kernel(F), cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  return e;
}

inline cudaError_t launch_resident(const FusedPlan& F, cudaStream_t s) {
  cudaError_t e = resident_attributes(F);
  if (e != cudaSuccess) return e;
  cudaLaunchAttribute at[1];
  const cudaLaunchConfig_t cfg = resident_config(F, s, at);
  return cudaLaunchKernelEx(&cfg, res_kernel(F), F.res_args);
}

template <typename ST, bool PRE>
inline SweepArgs<ST> sweep_args(const FusedPlan& F, const Level* lv, int l, const Control* ctl) {
  SweepArgs<ST> a;
  const Level& f = lv[l];
  const Level& c = lv[l + 1];
  for (int k = 0; k < 3; ++k) {
    a.f.n[k] = f.g.n[k];
    a.nc[k] = c.g.n[k];
  }
  a.f.type = f.type;
  a.f.Ad = (const ST*)f.Adiag_s;
  a.f.r = f.r;
  a.f.z = PRE ? (ST*)f.zt : (ST*)f.z;
  a.f.zin = (const ST*)f.zt;
  a.f.s = F.s[l];
  for (int k = 0; k < 3; ++k) a.f.ax[k] = k < f.g.dim ? f.Ax[k] : nullptr;
  a.rc = (ST*)c.r;
  a.zc = (ST*)c.z;
  a.rho = F.rho;
  a.pi = F.pi;
  a.ctl = ctl;
  a.r_f32 = l == 0;
  a.chunk = F.chunk[l];
  a.tiles_x = F.tiles_x[l];
  a.tiles_y = F.tiles_y[l];
  a.zr = -1;
  a.zr_ctl = nullptr;
  a.zr_partials = nullptr;
  if (!PRE && l == 0 && F.zr_mode >= 0) {
    a.zr = F.zr_mode;
    a.zr_ctl = F.zr_ctl;
    a.zr_partials = F.zr_partials;
  }
  return a;
}

template <int DIM, typename ST, int NS, bool PRE, bool STO = false>
inline cudaError_t launch_sweep_t(const FusedPlan& F, const Level* lv, int l, const Control* ctl, cudaStream_t s) {
  constexpr TileShape T = STO ? kTile3S : (DIM == 3 ? kTile3 : kTile2);
  if constexpr (DIM == 3 && !STO && std::is_same<ST, float>::value && T.k != 1) {
    if (F.chunk[l] > 2 && ((F.step1[l] >> (PRE ? 0 : 1)) & 1)) {
      constexpr TileShape T1 = {T.tx, T.ty, T.nt, 1};
      auto kern = k_sweep<DIM, ST, NS, T1.tx, T1.ty, PRE, T1.nt, T1.k, STO>;
      const size_t smem = sweep_smem(DIM, NS, T1, false, STO);
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      return launch_k(kern, F.blocks[l], T1.nt, smem, s, sweep_args<ST, PRE>(F, lv, l, ctl));
    }
  }
  if (DIM == 3 && F.chunk[l] == 2) {
    // small level: each block's 2 planes + halo planes in ONE pipeline step
    constexpr TileShape T1 = {T.tx, T.ty, T.nt, 2 + 2 * NS};
    auto kern = k_sweep<DIM, ST, NS, T1.tx, T1.ty, PRE, T1.nt, T1.k, STO>;
    const size_t smem = sweep_smem(DIM, NS, T1, true, STO);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return launch_k(kern, F.blocks[l], T1.nt, smem, s, sweep_args<ST, PRE>(F, lv, l, ctl));
  }
  auto kern = k_sweep<DIM, ST, NS, T.tx, T.ty, PRE, T.nt, T.k, STO>;
  constexpr int NT = T.nt;
  const size_t smem = sweep_smem(DIM, NS, T, false, STO);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  return launch_k(kern, F.blocks[l], NT, smem, s, sweep_args<ST, PRE>(F, lv, l, ctl));
}

template <typename ST, bool PRE>
inline cudaError_t launch_sweep_st(const FusedPlan& F, const Level* lv, int l, const Control* ctl, cudaStream_t s) {
  if (F.dim == 3) {
    switch (F.ns) {
      case 2: return launch_sweep_t<3, ST, 2, PRE>(F, lv, l, ctl, s);
      case 4: return launch_sweep_t<3, ST, 4, PRE>(F, lv, l, ctl, s);
      case 6: return launch_sweep_t<3, ST, 6, PRE>(F, lv, l, ctl, s);
    }
  } else {
    switch (F.ns) {
      case 2: return launch_sweep_t<2, ST, 2, PRE>(F, lv, l, ctl, s);
      case 4: return launch_sweep_t<2, ST, 4, PRE>(F, lv, l, ctl, s);
      case 6: return launch_sweep_t<2, ST, 6, PRE>(F, lv, l, ctl, s);
    }
  }
  return cudaErrorInvalidValue;
}

// ---- the column-register sweep (mg_colsweep.cuh) -------------------------------------

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime
// (the library links no driver stub).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
inline EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return (EncodeTiledFn) nullptr;
    }
    return (EncodeTiledFn)p;
  }();
  return fn;
}

// A 3D tiled tensor map over one array of a level (axis 0 slowest), box =
// (bx columns, by rows, 1 plane), zero fill outside the grid.
inline bool tensor_map_3d(CUtensorMap* m, const void* base, int es, const Geom& g, int bx, int by) {
  EncodeTiledFn fn = encode_tiled();
  if (!fn || ((uintptr_t)base & 15) || ((long long)g.n[2] * es) % 16) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)g.n[2], (cuuint64_t)g.n[1], (cuuint64_t)g.n[0]};
  const cuuint64_t strides[2] = {(cuuint64_t)g.n[2] * es, (cuuint64_t)g.n[1] * g.n[2] * es};
  const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
  const cuuint32_t est[3] = {1, 1, 1};
  return fn(m, es == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_UINT16, 3, const_cast<void*>(base),
            dims, strides, box, est, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The column kernel runs streamed level l of a 3D label-uniform plan with
// pre_post 2 whose rows are whole 16-byte units of every array, whose
// extents halve evenly (pairs of rows, pairs of planes) and whose cells have
// 32-bit indices.
inline bool col_ok(const FusedPlan& F, const Level* lv, int l) {
  if (!F.valid || F.sto || F.dim != 3 || F.ns != 4 || l >= F.lc || F.split[l]) return false;
  const Geom& g = lv[l].g;
  const int es = F.storage == MG_STORE_F32 ? 4 : 2;
  return g.n[2] % (16 / es) == 0 && g.n[1] % 2 == 0 && g.n[0] % 2 == 0 &&
         (long long)g.n[0] * g.n[1] * g.n[2] < (1LL << 31) && encode_tiled() != nullptr;
}

template <typename ST, int NS, int TX, int TY, bool PRE, int MINB>
inline cudaError_t launch_col_t(const FusedPlan& F, const Level* lv, int l, const Control* ctl, cudaStream_t s) {
  using G = ColGeom<ST, NS, TX, TY>;
  const Level& f = lv[l];
  CUtensorMap tr, ta, tz;
  std::memset(&tz, 0, sizeof(tz));
  if (!tensor_map_3d(&tr, f.r, l == 0 ? 4 : (int)sizeof(ST), f.g, G::RXB, G::RY) ||
      !tensor_map_3d(&ta, f.Adiag_s, (int)sizeof(ST), f.g, G::RXB, G::RY) ||
      (!PRE && !tensor_map_3d(&tz, f.zt, (int)sizeof(ST), f.g, G::RXB, G::RY)))
    return cudaErrorInvalidValue;
  if (PRE) tz = ta;  // unused by PRE
  auto kern = k_colsweep<ST, NS, TX, TY, PRE, MINB>;
  const size_t smem = G::smem(PRE);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  return launch_k(kern, F.blocks[l], G::NT, smem, s, sweep_args<ST, PRE>(F, lv, l, ctl), const_cast<Control*>(ctl),
                  tr, ta, tz);
}

template <typename ST, bool PRE>
inline cudaError_t launch_col_st(const FusedPlan& F, const Level* lv, int l, const Control* ctl, cudaStream_t s) {
  switch (F.col[l]) {
    case 1: return launch_col_t<ST, 4, 32, 16, PRE, 2>(F, lv, l, ctl, s);
    case 2: return launch_col_t<ST, 4, 32, 32, PRE, 1>(F, lv, l, ctl, s);
    case 3: return launch_col_t<ST, 4, 64, 16, PRE, 1>(F, lv, l, ctl, s);
  }
  return cudaErrorInvalidValue;
}

template <bool PRE>
inline cudaError_t launch_col(const FusedPlan& F, const Level* lv, int l, const Control* ctl, cudaStream_t s) {
  switch (F.storage) {
    case MG_STORE_F32: return launch_col_st<float, PRE>(F, lv, l, ctl, s);
    case MG_STORE_F16: return launch_col_st<__half, PRE>(F, lv, l, ctl, s);
    case MG_STORE_BF16: return launch_col_st<__nv_bfloat16, PRE>(F, lv, l, ctl, s);
  }
  return cudaErrorInvalidValue;
}

// Resident blocks per SM of column shape c (the smaller of PRE and POST).
template <typename ST, int TX, int TY, int MINB>
inline int col_occupancy_t(int num_sms) {
  using G = ColGeom<ST, 4, TX, TY>;
  int a = 0, b = 0;
  auto kp = k_colsweep<ST, 4, TX, TY, true, MINB>;
  auto kq = k_colsweep<ST, 4, TX, TY, false, MINB>;
  if (cudaFuncSetAttribute(kp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::smem(true)) != cudaSuccess ||
      cudaFuncSetAttribute(kq, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::smem(false)) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, kp, G::NT, G::smem(true)) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kq, G::NT, G::smem(false)) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  (void)num_sms;
  return a < b ? a : b;
}

template <typename ST>
inline int col_occupancy_st(int c, int num_sms) {
  switch (c) {
    case 1: return col_occupancy_t<ST, 32, 16, 2>(num_sms);
    case 2: return col_occupancy_t<ST, 32, 32, 1>(num_sms);
    case 3: return col_occupancy_t<ST, 64, 16, 1>(num_sms);
  }
  return 0;
}

inline int col_occupancy(const FusedPlan& F, int c) {
  switch (F.storage) {
    case MG_STORE_F32: return col_occupancy_st<float>(c, F.num_sms);
    case MG_STORE_F16: return col_occupancy_st<__half>(c, F.num_sms);
    case MG_STORE_BF16: return col_occupancy_st<__nv_bfloat16>(c, F.num_sms);
  }
  return 0;
}

template <bool PRE>
inline cudaError_t launch_sweep(const FusedPlan& F, const Level* lv, int l, const Control* ctl, cudaStream_t s) {
  if (F.col[l]) return launch_col<PRE>(F, lv, l, ctl, s);
  if (F.sto) {
    switch (F.ns) {
      case 2: return launch_sweep_t<3, float, 2, PRE, true>(F, lv, l, ctl, s);
      case 4: return launch_sweep_t<3, float, 4, PRE, true>(F, lv, l, ctl, s);
    }
    return cudaErrorInvalidValue;
  }
  switch (F.storage) {
    case MG_STORE_F32: return launch_sweep_st<float, PRE>(F, lv, l, ctl, s);
    case MG_STORE_F16: return launch_sweep_st<__half, PRE>(F, lv, l, ctl, s);
    case MG_STORE_BF16: return launch_sweep_st<__nv_bfloat16, PRE>(F, lv, l, ctl, s);
  }
  return cudaErrorInvalidValue;
}

template <typename ST, bool STO = false>
inline cudaError_t launch_coarse_st(const FusedPlan& F, const Control* ctl, cudaStream_t s) {
  CoarseArgs a = F.coarse;
  a.ctl = ctl;
  auto kern = k_coarse<ST, STO>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)F.coarse_smem);
  if (e != cudaSuccess) return e;
  return launch_k(kern, 1, F.coarse_threads, F.coarse_smem, s, a);
}

inline cudaError_t launch_coarse(const FusedPlan& F, const Control* ctl, cudaStream_t s) {
  if (F.sto) return launch_coarse_st<float, true>(F, ctl, s);
  switch (F.storage) {
    case MG_STORE_F32: return launch_coarse_st<float>(F, ctl, s);
    case MG_STORE_F16: return launch_coarse_st<__half>(F, ctl, s);
    case MG_STORE_BF16: return launch_coarse_st<__nv_bfloat16>(F, ctl, s);
  }
  return cudaErrorInvalidValue;
}

// The V-cycle (mgpcg.py:125-148) of a fused plan is composed in mg_plan.cu:
// per streamed level the streamed kernel or (split) the per-kernel passes,
// then the coarse block.

}  // namespace mg
