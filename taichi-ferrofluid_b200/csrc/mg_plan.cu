// Plan, workspace layout, CUDA-graph PCG solve and the C ABI of the B200
// MGPCG library (include/mgpcg_b200.h).
//
// Ownership: the caller allocates one device workspace of
// mg_plan_workspace_bytes() bytes; every solver field (mgpcg.py:21-44) lives at
// a fixed 256-byte aligned offset in it.  This file allocates host memory only
// (the plan, a pinned parameter block) plus the CUDA graph objects.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <utility>
#include <vector>

#include "mg_common.cuh"
#include "mg_kernels.cuh"
#include "mg_pcg.cuh"
#include "mg_fused_host.cuh"
#include "mg_batch.cuh"
#include "mg_strategies.cuh"
#include "mg_levelset.cuh"
#include "mg_advect.cuh"

using namespace mg;

// Blocks per SM of the reduction kernels' grids (a whole number of waves at
// their register counts).
#ifndef MG_RED_BLOCKS_PER_SM
#define MG_RED_BLOCKS_PER_SM 4
#endif

namespace {

thread_local char g_err[512] = "";

int set_err(const char* what, cudaError_t e) {
  snprintf(g_err, sizeof(g_err), "%s: %s", what, cudaGetErrorString(e));
  return MG_E_CUDA;
}
int bad(const char* what) {
  snprintf(g_err, sizeof(g_err), "bad argument: %s", what);
  return MG_E_BADARG;
}

#define CK(call)                                   \
  do {                                             \
    cudaError_t e_ = (call);                       \
    if (e_ != cudaSuccess) return set_err(#call, e_); \
  } while (0)

#define CKL(what)                                  \
  do {                                             \
    cudaError_t e_ = cudaGetLastError();           \
    if (e_ != cudaSuccess) return set_err(what, e_); \
  } while (0)

constexpr int kFields = 9;
constexpr int kFieldAdiagS = 9;  // internal: storage copy of Adiag
constexpr int kFieldZT = 10;     // internal: second z buffer of the fused V-cycle
constexpr int kFieldXH = 11;     // internal: FP64 x of the mixed form (refresh plans)
constexpr int kFieldCount = 12;

struct Loc {
  int64_t off = -1, bytes = 0;
};

int64_t align256(int64_t v) { return (v + 255) & ~int64_t(255); }

int elem_bytes(int storage) { return storage == MG_STORE_F32 ? 4 : 2; }

}  // namespace

struct mg_plan {
  mg_plan_desc_t d;
  int L;
  Geom geom[kMaxLevels];
  Loc loc[kFieldCount][kMaxLevels][3];
  int64_t off_partials, off_ctl, ws_bytes;
  char* base = nullptr;
  Level lv[kMaxLevels];
  Control* ctl = nullptr;
  double* partials = nullptr;
  int red_blocks = 0;
  int ew_blocks[kMaxLevels];
  int op_form[kMaxLevels];
  int whole[kMaxLevels];     // level is whole-domain: every cell FLUID, Adiag != 0
  float offdiag[kMaxLevels];
  bool prepared = false;
  FusedPlan fp;
  int has_cond = 1;          // the graph body ends by setting the while condition
  uint64_t graph_sig = 0;
  // graph state
  cudaStream_t cap = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaGraphConditionalHandle cond = 0;
  char* base_of_graph = nullptr;
  // pinned parameter / stats staging
  Control* host_ctl = nullptr;
  int device = -1;
  int num_sms = 148;
};

namespace {

int64_t level_cells(const mg_plan* P, int l) { return P->geom[l].count; }

void layout(mg_plan* P) {
  int64_t off = 0;
  auto put = [&](int f, int l, int comp, int64_t bytes) {
    P->loc[f][l][comp].off = off;
    P->loc[f][l][comp].bytes = bytes;
    off = align256(off + bytes);
  };
  const int es = elem_bytes(P->d.storage);
  const int dim = P->d.dim;
  for (int l = 0; l < P->L; ++l) {
    int64_t n = level_cells(P, l);
    put(MG_FIELD_TYPE, l, 0, n);
    put(MG_FIELD_ADIAG, l, 0, n * 4);
    // the dim components back to back, so Ax[l] is one (dim, *shape) array
    put(MG_FIELD_AX, l, 0, dim * n * 4);
    for (int k = 0; k < dim; ++k) {
      P->loc[MG_FIELD_AX][l][k].off = P->loc[MG_FIELD_AX][l][0].off + k * n * 4;
      P->loc[MG_FIELD_AX][l][k].bytes = n * 4;
    }
    put(MG_FIELD_R, l, 0, n * (l == 0 ? 4 : es));
    put(MG_FIELD_Z, l, 0, n * es);
    if (P->d.storage != MG_STORE_F32) put(kFieldAdiagS, l, 0, n * es);
    else P->loc[kFieldAdiagS][l][0] = P->loc[MG_FIELD_ADIAG][l][0];
    put(kFieldZT, l, 0, n * es);
  }
  int64_t n0 = level_cells(P, 0);
  put(MG_FIELD_B, 0, 0, n0 * 4);
  put(MG_FIELD_X, 0, 0, n0 * 4);
  put(MG_FIELD_P, 0, 0, n0 * 4);
  put(MG_FIELD_AP, 0, 0, n0 * 4);
  if (P->d.refresh_every > 0) put(kFieldXH, 0, 0, n0 * 8);
  P->off_partials = off;
  off = align256(off + sizeof(double) * kMaxPartials);
  P->off_ctl = off;
  off = align256(off + sizeof(Control));
  P->ws_bytes = off;
}

void bind_views(mg_plan* P) {
  char* B = P->base;
  for (int l = 0; l < P->L; ++l) {
    Level& v = P->lv[l];
    v.g = P->geom[l];
    v.type = (int8_t*)(B + P->loc[MG_FIELD_TYPE][l][0].off);
    v.Adiag = (float*)(B + P->loc[MG_FIELD_ADIAG][l][0].off);
    for (int k = 0; k < 3; ++k)
      v.Ax[k] = k < P->d.dim ? (float*)(B + P->loc[MG_FIELD_AX][l][k].off) : nullptr;
    v.r = B + P->loc[MG_FIELD_R][l][0].off;
    v.z = B + P->loc[MG_FIELD_Z][l][0].off;
    v.Adiag_s = B + P->loc[kFieldAdiagS][l][0].off;
    v.zt = B + P->loc[kFieldZT][l][0].off;
  }
  P->partials = (double*)(B + P->off_partials);
  P->ctl = (Control*)(B + P->off_ctl);
}

inline cudaStream_t S(void* s) { return (cudaStream_t)s; }

float* fptr(mg_plan* P, int f) { return (float*)(P->base + P->loc[f][0][0].off); }
// The mixed form's FP64 x (refresh plans), else null.
double* xhptr(mg_plan* P) {
  return P->d.refresh_every > 0 ? (double*)(P->base + P->loc[kFieldXH][0][0].off) : nullptr;
}

int grid_for(const mg_plan* P, int64_t n, int threads = 256) {
  int64_t b = (n + threads - 1) / threads;
  int64_t cap = (int64_t)P->num_sms * 16;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

// ---- launch sequences (shared by the direct calls and graph capture) -------

constexpr int64_t kBottomBlockCells = 1 << 16;

int launch_smooth(mg_plan* P, int l, int phase, cudaStream_t s) {
  if (P->whole[l] && P->d.dim == 3 && P->geom[l].n[2] % 4 == 0) {  // every cell FLUID: 4-cell groups
    CK(launch_k(k_smooth_w4, grid_for(P, level_cells(P, l) / 4), 256, 0, s, P->lv[l], phase));
    return MG_OK;
  }
  int64_t n = level_cells(P, l) / 2 + level_cells(P, l) / (P->d.dim == 3 ? P->geom[l].n[2] : P->geom[l].n[1]);
  CK(launch_k(k_smooth, grid_for(P, n), 256, 0, s, P->lv[l], phase));
  return MG_OK;
}

// Level l+1 is level l halved exactly, 3D, level l's fastest extent a
// multiple of 4 (the 4-cell-group restriction and prolongation).
bool halves_by4(const mg_plan* P, int l) {
  if (P->d.dim != 3 || P->geom[l].n[2] % 4 != 0) return false;
  for (int a = 0; a < 3; ++a)
    if (P->geom[l].n[a] != 2 * P->geom[l + 1].n[a]) return false;
  return true;
}

int launch_restrict(mg_plan* P, int l, cudaStream_t s) {
  if (P->whole[l] && halves_by4(P, l)) {
    CK(launch_k(k_restrict_w4, grid_for(P, level_cells(P, l + 1) / 2), 256, 0, s, P->lv[l], P->lv[l + 1]));
    return MG_OK;
  }
  CK(launch_k(k_restrict, grid_for(P, level_cells(P, l + 1)), 256, 0, s, P->lv[l], P->lv[l + 1]));
  return MG_OK;
}

int launch_prolongate(mg_plan* P, int l, cudaStream_t s) {
  if (halves_by4(P, l)) {
    CK(launch_k(k_prolongate4, grid_for(P, level_cells(P, l) / 4), 256, 0, s, P->lv[l], P->lv[l + 1]));
    return MG_OK;
  }
  CK(launch_k(k_prolongate, grid_for(P, level_cells(P, l)), 256, 0, s, P->lv[l], P->lv[l + 1]));
  return MG_OK;
}

// v_cycle (mgpcg.py:125-148) with the stored-coefficient kernels.
int launch_vcycle_generic(mg_plan* P, cudaStream_t s) {
  const int L = P->L;
  CK(cudaMemsetAsync(P->lv[0].z, 0, level_cells(P, 0) * sizeof(float), s));
  for (int l = 0; l < L - 1; ++l) {
    for (int i = 0; i < P->d.pre_post; ++i) {
      if (int rc = launch_smooth(P, l, 0, s)) return rc;
      if (int rc = launch_smooth(P, l, 1, s)) return rc;
    }
    if (int rc = launch_restrict(P, l, s)) return rc;
  }
  const int nh = P->d.bottom / 2;
  if (level_cells(P, L - 1) <= kBottomBlockCells) {
    if (nh > 0) {
      CK(launch_k(k_bottom, 1, 1024, 0, s, P->lv[L - 1], nh));
    }
  } else {
    for (int i = 0; i < nh; ++i) {
      if (int rc = launch_smooth(P, L - 1, 0, s)) return rc;
      if (int rc = launch_smooth(P, L - 1, 1, s)) return rc;
    }
    for (int i = 0; i < nh; ++i) {
      if (int rc = launch_smooth(P, L - 1, 1, s)) return rc;
      if (int rc = launch_smooth(P, L - 1, 0, s)) return rc;
    }
  }
  for (int l = L - 2; l >= 0; --l) {
    if (int rc = launch_prolongate(P, l, s)) return rc;
    for (int i = 0; i < P->d.pre_post; ++i) {
      if (int rc = launch_smooth(P, l, 1, s)) return rc;
      if (int rc = launch_smooth(P, l, 0, s)) return rc;
    }
  }
  return MG_OK;
}

// Pre-smoothing and restriction of streamed level l of a fused plan (PRE),
// or prolongation and post-smoothing (POST): the streamed kernel, or for a
// split level the per-kernel passes on z[l] in place.  The two forms meet
// only in r[l+1] and z[l+1] (restriction zeroes z[l+1]; the streamed PRE
// writes it 0), so levels of either form mix.
int launch_level(mg_plan* P, int l, bool pre, cudaStream_t s) {
  if (!P->fp.split[l]) {
    cudaError_t e = pre ? launch_sweep<true>(P->fp, P->lv, l, P->ctl, s)
                        : launch_sweep<false>(P->fp, P->lv, l, P->ctl, s);
    return e == cudaSuccess ? MG_OK : set_err("launch_sweep", e);
  }
  if (pre) {
    // pre-smoothing starts from z = 0; on a whole-domain level of 4-cell
    // groups its first half sweep (pointwise) also writes those zeros
    const bool first4 = P->whole[l] && P->d.dim == 3 && P->geom[l].n[2] % 4 == 0;
    if (first4) CK(launch_k(k_smooth_first_w4, grid_for(P, level_cells(P, l) / 4), 256, 0, s, P->lv[l]));
    else if (l == 0) CK(cudaMemsetAsync(P->lv[0].z, 0, level_cells(P, 0) * sizeof(float), s));
    for (int i = 0; i < P->d.pre_post; ++i) {
      if (!(first4 && i == 0))
        if (int rc = launch_smooth(P, l, 0, s)) return rc;
      if (int rc = launch_smooth(P, l, 1, s)) return rc;
    }
    return launch_restrict(P, l, s);
  }
  if (int rc = launch_prolongate(P, l, s)) return rc;
  for (int i = 0; i < P->d.pre_post; ++i) {
    if (int rc = launch_smooth(P, l, 1, s)) return rc;
    if (l == 0 && i + 1 == P->d.pre_post && P->fp.zr_mode >= 0) {  // the last half sweep with z.r
      const int nb = std::min(grid_for(P, level_cells(P, 0) / 4), kMaxPartials / 2);
      CK(launch_k(k_smooth_zr_w4, nb, kRedThreads, 0, s, P->lv[0], 0, P->fp.zr_ctl, P->fp.zr_partials,
                  P->fp.zr_mode));
    } else if (int rc = launch_smooth(P, l, 0, s)) {
      return rc;
    }
  }
  return MG_OK;
}

// One V-cycle of a fused plan: the streamed levels down, the coarse block,
// the streamed levels up.
int launch_vcycle_fused(mg_plan* P, cudaStream_t s) {
  if (P->fp.res) {  // streamed levels above the bricks, then one cluster launch
    for (int l = 0; l < P->fp.res_lp; ++l)
      if (int rc = launch_level(P, l, true, s)) return rc;
    cudaError_t e = launch_resident(P->fp, s);
    if (e != cudaSuccess) return set_err("launch_resident", e);
    for (int l = P->fp.res_lp - 1; l >= 0; --l)
      if (int rc = launch_level(P, l, false, s)) return rc;
    return MG_OK;
  }
  for (int l = 0; l < P->fp.lc; ++l)
    if (int rc = launch_level(P, l, true, s)) return rc;
  cudaError_t e = launch_coarse(P->fp, P->ctl, s);
  if (e != cudaSuccess) return set_err("launch_coarse", e);
  for (int l = P->fp.lc - 1; l >= 0; --l)
    if (int rc = launch_level(P, l, false, s)) return rc;
  return MG_OK;
}

int launch_vcycle(mg_plan* P, cudaStream_t s) {
  if (P->fp.valid) return launch_vcycle_fused(P, s);
  return launch_vcycle_generic(P, s);
}

// ---- autotuner: streamed kernel or per-kernel passes, per level ------------
//
// The streamed kernel trades halo recomputation for memory traffic.  For the
// label-uniform form it wins on every level measured (B200, 128^3 and 256^3);
// for the whole-domain stored form, which stages 24 bytes a cell, the
// per-kernel passes win on the large levels and the streamed kernel on the
// small ones.  So for the stored form each streamed level is timed both ways
// (CUDA events on the plan's stream, one warm-up, kTuneReps timed) the first time a
// shape is prepared, and the faster is kept; the choice is cached per shape
// for the process.  Both variants compute the same float32 values.
std::mutex g_tune_mu;
// timed repetitions of each variant (after one warm-up); with three, the
// choice for levels of ~20 us flipped between runs
constexpr int kTuneReps = 10;
std::map<std::array<int, 7>, uint32_t> g_tune;  // bit l: split level l

int tune_split(mg_plan* P, cudaStream_t s) {
  if (!P->fp.valid || !P->fp.sto) return MG_OK;
  // MGPCG_SPLIT=<bits> replaces the timing (profilers serialise the trial
  // launches and would skew the choice)
  if (const char* ov = std::getenv("MGPCG_SPLIT")) {
    const unsigned long v = std::strtoul(ov, nullptr, 0);
    for (int l = 0; l < P->fp.lc; ++l) P->fp.split[l] = (v >> l) & 1ul;
    return MG_OK;
  }
  const Geom& g = P->geom[0];
  const std::array<int, 7> key = {g.dim, g.n[0], g.n[1], g.n[2], P->L, P->d.pre_post, P->fp.lc};
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) {
      for (int l = 0; l < P->fp.lc; ++l) P->fp.split[l] = (it->second >> l) & 1u;
      return MG_OK;
    }
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CK(cudaEventCreate(&e0));
  cudaError_t ce = cudaEventCreate(&e1);
  if (ce != cudaSuccess) {
    cudaEventDestroy(e0);
    return set_err("cudaEventCreate", ce);
  }
  uint32_t bits = 0;
  int rc = MG_OK;
  for (int l = 0; l < P->fp.lc && rc == MG_OK; ++l) {
    float t[2] = {0.0f, 0.0f};
    for (int mode = 0; mode < 2 && rc == MG_OK; ++mode) {
      P->fp.split[l] = mode == 1;
      for (int rep = 0; rep < 1 + kTuneReps && rc == MG_OK; ++rep) {  // rep 0 warms up
        if (rep == 1) cudaEventRecord(e0, s);
        rc = launch_level(P, l, true, s);
        if (rc == MG_OK) rc = launch_level(P, l, false, s);
      }
      if (rc != MG_OK) break;
      cudaEventRecord(e1, s);
      cudaError_t e = cudaEventSynchronize(e1);
      if (e == cudaSuccess) e = cudaEventElapsedTime(&t[mode], e0, e1);
      if (e != cudaSuccess) rc = set_err("tune_split", e);
    }
    P->fp.split[l] = rc == MG_OK && t[1] < t[0];
    if (P->fp.split[l]) bits |= 1u << l;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != MG_OK) {
    for (int l = 0; l < kMaxLevels; ++l) P->fp.split[l] = false;
    return rc;
  }
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[key] = bits;
  return MG_OK;
}

// Grid and planes per pipeline step of the streamed levels.  The grid of a
// level is sized for the blocks that fit one SM's shared memory plus 0, 1 or
// 2 more (shorter chunks, more blocks); measured on B200, 1 more makes the
// 256^3 level-0 sweeps faster (PRE 225.7 -> 170.2 us, POST 240.5 -> 210.9 us)
// and the 128^3 ones slower (PRE 40.2 -> 44.3 us).  Then, for the 3D
// label-uniform float32 form, one plane per step or the tile's two, per
// direction (a shorter ring; with the grid held fixed two planes won on every
// level measured).  Each pipelined level is timed every way (one warm-up,
// kTuneReps timed) the first time a shape is prepared; the choice is cached
// per shape.  All choices compute the same values.
//
// Each streamed level also runs, where col_ok allows, the column-register
// kernel (k_colsweep) in each tile shape of kColShapes with its grid sized
// for its resident blocks plus 0 or 1 more; the fastest of every variant is
// kept (MGPCG_COL=<bits>, 2 bits a level, pins the kernel).
struct StreamChoice {
  uint32_t step, grid, col;
};
std::map<std::array<int, 7>, StreamChoice> g_tune_stream;

// Forces column shape c (0: k_sweep) on streamed level l; false where the
// level cannot run it.
bool set_col(mg_plan* P, int l, int c) {
  FusedPlan& F = P->fp;
  if (c < 0 || c >= kColShapeCount) return false;
  if (c && !col_ok(F, P->lv, l)) return false;
  if (c && F.col_per_sm[c] == 0) F.col_per_sm[c] = col_occupancy(F, c);
  if (c && F.col_per_sm[c] <= 0) return false;
  F.col[l] = (unsigned char)c;
  return true;
}

void apply_stream_bits(mg_plan* P, uint32_t step, uint32_t grid, uint32_t col) {
  FusedPlan& F = P->fp;
  const bool steps_ok = !F.sto && F.dim == 3 && F.storage == MG_STORE_F32;
  for (int l = 0; l < F.lc; ++l) {
    if (!set_col(P, l, (int)((col >> (2 * l)) & 3u))) F.col[l] = 0;
    level_grid(&F, P->lv[l].g, l, (int)((grid >> (2 * l)) & 3u));
    F.step1[l] = steps_ok && !F.col[l] ? (unsigned char)((step >> (2 * l)) & 3u) : 0;
  }
}

int time_level(mg_plan* P, int l, int dirs, cudaEvent_t e0, cudaEvent_t e1, cudaStream_t s, float* ms) {
  int rc = MG_OK;
  for (int rep = 0; rep < 1 + kTuneReps && rc == MG_OK; ++rep) {  // rep 0 warms up
    if (rep == 1) cudaEventRecord(e0, s);
    if (dirs & 1) rc = launch_level(P, l, true, s);
    if (rc == MG_OK && (dirs & 2)) rc = launch_level(P, l, false, s);
  }
  if (rc != MG_OK) return rc;
  cudaEventRecord(e1, s);
  cudaError_t e = cudaEventSynchronize(e1);
  if (e == cudaSuccess) e = cudaEventElapsedTime(ms, e0, e1);
  return e == cudaSuccess ? MG_OK : set_err("tune_stream", e);
}

int tune_stream(mg_plan* P, cudaStream_t s) {
  FusedPlan& F = P->fp;
  if (!F.valid) return MG_OK;
  const bool steps_ok = !F.sto && F.dim == 3 && F.storage == MG_STORE_F32;
  // MGPCG_STEP1=<bits> / MGPCG_GRID=<bits> replace the timing (profilers
  // serialise the trial launches and would skew the choice)
  const char* ov_step = std::getenv("MGPCG_STEP1");
  const char* ov_grid = std::getenv("MGPCG_GRID");
  const char* ov_col = std::getenv("MGPCG_COL");
  if (ov_step || ov_grid || ov_col) {
    apply_stream_bits(P, ov_step ? (uint32_t)std::strtoul(ov_step, nullptr, 0) : 0u,
                      ov_grid ? (uint32_t)std::strtoul(ov_grid, nullptr, 0) : 0u,
                      ov_col ? (uint32_t)std::strtoul(ov_col, nullptr, 0) : 0u);
    return MG_OK;
  }
  const Geom& g = P->geom[0];
  const std::array<int, 7> key = {g.dim, g.n[0], g.n[1], g.n[2], P->L, P->d.pre_post, F.lc};
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_stream.find(key);
    if (it != g_tune_stream.end()) {
      apply_stream_bits(P, it->second.step, it->second.grid, it->second.col);
      return MG_OK;
    }
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CK(cudaEventCreate(&e0));
  cudaError_t ce = cudaEventCreate(&e1);
  if (ce != cudaSuccess) {
    cudaEventDestroy(e0);
    return set_err("cudaEventCreate", ce);
  }
  uint32_t step = 0, grid = 0, col = 0;
  int rc = MG_OK;
  for (int l = 0; l < F.lc && rc == MG_OK; ++l) {
    F.step1[l] = 0;
    F.col[l] = 0;
    if (F.split[l]) continue;  // per-kernel passes
    level_grid(&F, P->lv[l].g, l, 0);
    const bool one_step = F.chunk[l] <= 2;  // k_sweep's one-step launch
    float best = 0.0f;
    int best_extra = 0, best_col = 0, last_chunk = -1;
    for (int extra = 0; extra <= (one_step ? 0 : 2) && rc == MG_OK; ++extra) {
      level_grid(&F, P->lv[l].g, l, extra);
      if (F.chunk[l] == last_chunk) continue;  // the same grid
      last_chunk = F.chunk[l];
      float t = 0.0f;
      rc = time_level(P, l, 3, e0, e1, s, &t);
      if (rc == MG_OK && (extra == 0 || t < best)) {
        best = t;
        best_extra = extra;
      }
    }
    for (int c = 1; c < kColShapeCount && rc == MG_OK; ++c) {
      if (!set_col(P, l, c)) continue;
      last_chunk = -1;
      for (int extra = 0; extra <= 1 && rc == MG_OK; ++extra) {
        level_grid(&F, P->lv[l].g, l, extra);
        if (F.chunk[l] == last_chunk) continue;
        last_chunk = F.chunk[l];
        float t = 0.0f;
        rc = time_level(P, l, 3, e0, e1, s, &t);
        if (rc == MG_OK && t < best) {
          best = t;
          best_extra = extra;
          best_col = c;
        }
      }
    }
    F.col[l] = (unsigned char)(rc == MG_OK ? best_col : 0);
    level_grid(&F, P->lv[l].g, l, rc == MG_OK ? best_extra : 0);
    grid |= (uint32_t)F.grid_extra[l] << (2 * l);
    col |= (uint32_t)F.col[l] << (2 * l);
    if (!steps_ok || F.chunk[l] <= 2 || F.col[l]) continue;
    for (int dir = 0; dir < 2 && rc == MG_OK; ++dir) {
      float t[2] = {0.0f, 0.0f};
      for (int mode = 0; mode < 2 && rc == MG_OK; ++mode) {
        F.step1[l] = (unsigned char)((F.step1[l] & ~(1u << dir)) | ((unsigned)mode << dir));
        rc = time_level(P, l, 1 << dir, e0, e1, s, &t[mode]);
      }
      const bool one = rc == MG_OK && t[1] < t[0];
      F.step1[l] = (unsigned char)((F.step1[l] & ~(1u << dir)) | ((unsigned)one << dir));
    }
    step |= (uint32_t)F.step1[l] << (2 * l);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != MG_OK) {
    apply_stream_bits(P, 0u, 0u, 0u);
    return rc;
  }
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_stream[key] = {step, grid, col};
  return MG_OK;
}

// The cluster-resident V-cycle against the streamed one: for a label-uniform
// float32 plan whose levels allow bricks, the V-cycle is timed streamed and
// with the cluster starting at each feasible level (CUDA events, one warm-up,
// kTuneReps timed) the first time a shape is prepared, and the fastest kept,
// cached per shape for the process.  All compute the same float32 values.
// MGPCG_RESIDENT=<level> (the cluster from the first feasible level from
// there) or MGPCG_RESIDENT=off replaces the timing, e.g. for profilers, which
// serialise the trial launches.
std::map<std::array<int, 7>, int> g_tune_res;  // -1: streamed; else first brick level, + 256 for 512-thread CTAs

// The cluster plan from the first feasible level in [lp_min, lp_max], checked
// against what the device can hold; false (res_ok = false) when there is none.
bool plan_resident(mg_plan* P, int lp_min, int lp_max, cudaStream_t s) {
  if (!make_resident_plan(&P->fp, P->lv, P->L, P->d.pre_post, P->d.bottom, lp_min, lp_max)) return false;
  // whether the device holds the cluster, asked once per (device, CTAs, bytes, threads)
  static std::map<std::array<int64_t, 4>, bool> fits;
  const std::array<int64_t, 4> key = {P->device, P->fp.res_blocks, (int64_t)P->fp.res_smem, P->fp.res_threads};
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = fits.find(key);
    if (it != fits.end()) {
      P->fp.res_ok = it->second;
      return it->second;
    }
  }
  bool ok = resident_attributes(P->fp) == cudaSuccess;
  if (ok) {
    cudaLaunchAttribute at[1];
    const cudaLaunchConfig_t cfg = resident_config(P->fp, s, at);
    int clusters = 0;
    ok = cudaOccupancyMaxActiveClusters(&clusters, res_kernel(P->fp), &cfg) == cudaSuccess && clusters >= 1;
  }
  if (!ok) cudaGetLastError();
  P->fp.res_ok = ok;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  fits[key] = ok;
  return ok;
}

int tune_resident(mg_plan* P, cudaStream_t s) {
  P->fp.res = false;
  P->fp.res_threads = kResThreads;
  if (!P->fp.valid) return MG_OK;
  if (!plan_resident(P, 0, P->L, s)) return MG_OK;
  const int lp_first = P->fp.res_lp;
  // MGPCG_RES_THREADS=512|1024 pins the cluster's CTA size with MGPCG_RESIDENT
  const char* ov_nt = std::getenv("MGPCG_RES_THREADS");
  if (const char* ov = std::getenv("MGPCG_RESIDENT")) {  // "off" / -1, or a start level
    const long v = std::strcmp(ov, "off") == 0 ? -1 : std::strtol(ov, nullptr, 0);
    if (ov_nt && std::strtol(ov_nt, nullptr, 0) == 512) P->fp.res_threads = 512;
    if (v >= 0 && plan_resident(P, (int)v, P->L, s)) P->fp.res = true;
    else plan_resident(P, lp_first, lp_first, s);
    return MG_OK;
  }
  // the choice: -1 streamed, else the first cluster level + 256 for 512 threads
  auto apply = [&](int choice) {
    P->fp.res_threads = choice >= 256 ? 512 : kResThreads;
    const int lp = choice >= 0 ? (choice & 255) : -1;
    if (lp >= 0 && plan_resident(P, lp, lp, s)) {
      P->fp.res = true;
    } else {
      P->fp.res_threads = kResThreads;
      plan_resident(P, lp_first, lp_first, s);
    }
  };
  const Geom& g = P->geom[0];
  const std::array<int, 7> key = {g.dim, g.n[0], g.n[1], g.n[2], P->L, P->d.pre_post, P->fp.lc};
  int cached = -2;  // -2: not timed yet
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_res.find(key);
    if (it != g_tune_res.end()) cached = it->second;
  }
  if (cached != -2) {  // (plan_resident takes the lock itself)
    apply(cached);
    return MG_OK;
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CK(cudaEventCreate(&e0));
  cudaError_t ce = cudaEventCreate(&e1);
  if (ce != cudaSuccess) {
    cudaEventDestroy(e0);
    return set_err("cudaEventCreate", ce);
  }
  auto time_vcycle = [&](float* ms) -> int {
    int rc = MG_OK;
    for (int rep = 0; rep < 1 + kTuneReps && rc == MG_OK; ++rep) {  // rep 0 warms up
      if (rep == 1) cudaEventRecord(e0, s);
      rc = launch_vcycle_fused(P, s);
    }
    if (rc != MG_OK) return rc;
    cudaEventRecord(e1, s);
    cudaError_t e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(ms, e0, e1);
    return e == cudaSuccess ? MG_OK : set_err("tune_resident", e);
  };
  float best = 0.0f;
  int best_choice = -1;
  int rc = time_vcycle(&best);  // streamed (res = false)
  for (int lp = lp_first; rc == MG_OK && lp < P->L; ++lp) {
    for (int nt : {kResThreads, 512}) {
      if (rc != MG_OK) break;
      P->fp.res_threads = nt;
      if (!plan_resident(P, lp, lp, s)) continue;
      P->fp.res = true;
      float t = 0.0f;
      rc = time_vcycle(&t);
      P->fp.res = false;
      if (rc == MG_OK && t < best) {
        best = t;
        best_choice = lp + (nt == 512 ? 256 : 0);
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != MG_OK) {
    P->fp.res_threads = kResThreads;
    return rc;
  }
  apply(best_choice);
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_res[key] = best_choice;
  return MG_OK;
}

// The level-0 POST sweep can take z.r (k_zr4) over the cells it writes: the
// label-uniform float32 form with level 0 streamed (not split, not inside the
// cluster launch) and a grid within the partials buffer.
bool zr_fusable(const mg_plan* P) {
  const FusedPlan& F = P->fp;
  const bool col = F.valid && !F.sto && P->d.storage == MG_STORE_F32 && F.lc > 0 && !F.split[0] &&
                   !(F.res && F.res_lp == 0) && F.blocks[0] <= kMaxPartials / 2;
  // or: level 0 split into per-kernel passes on a whole-domain float32 level
  // of 4-cell groups, whose last post-smoothing half sweep takes z.r
  // (k_smooth_zr_w4)
  const bool split = F.valid && P->d.storage == MG_STORE_F32 && F.lc > 0 && F.split[0] && P->whole[0] &&
                     !(F.res && F.res_lp == 0) &&
                     P->d.dim == 3 && P->geom[0].n[2] % 4 == 0 && P->geom[0].count % 4 == 0 &&
                     P->d.pre_post >= 1;
  return col || split;
}

template <typename ST>
int launch_zr_p(mg_plan* P, bool prologue, cudaStream_t s, bool zr_done = false) {
  const Level& L0 = P->lv[0];
  float* p = fptr(P, MG_FIELD_P);
  if (sizeof(ST) == 4 && P->geom[0].count % 4 == 0) {  // float32: 4-cell groups
    const int eb = grid_for(P, P->geom[0].count / 4);
    const Control* cc = P->ctl;
    if (prologue) {
      CK(launch_k(k_update_p4, eb, 256, 0, s, L0, p, cc));
      if (!zr_done) CK(launch_k(k_zr4, P->red_blocks, kRedThreads, 0, s, L0, P->ctl, P->partials, 0));
    } else {
      if (!zr_done) CK(launch_k(k_zr4, P->red_blocks, kRedThreads, 0, s, L0, P->ctl, P->partials, 1));
      CK(launch_k(k_update_p4, eb, 256, 0, s, L0, p, cc));
    }
    return MG_OK;
  }
  const Control* cc = P->ctl;
  // the mixed form (true-residual refresh) takes the flexible beta
  const float* Ap = P->d.refresh_every > 0 && P->d.storage != MG_STORE_F32 ? fptr(P, MG_FIELD_AP) : nullptr;
  if (prologue) {
    CK(launch_k(k_update_p<ST>, P->ew_blocks[0], 256, 0, s, L0, p, cc));
    CK(launch_k(k_zr<ST>, P->red_blocks, kRedThreads, 0, s, L0, P->ctl, P->partials, 0, Ap));
  } else {
    CK(launch_k(k_zr<ST>, P->red_blocks, kRedThreads, 0, s, L0, P->ctl, P->partials, 1, Ap));
    CK(launch_k(k_update_p<ST>, P->ew_blocks[0], 256, 0, s, L0, p, cc));
  }
  return MG_OK;
}

int launch_zr_p_any(mg_plan* P, bool prologue, cudaStream_t s, bool zr_done = false) {
  switch (P->d.storage) {
    case MG_STORE_F16: return launch_zr_p<__half>(P, prologue, s);
    case MG_STORE_BF16: return launch_zr_p<__nv_bfloat16>(P, prologue, s);
    default: return launch_zr_p<float>(P, prologue, s, zr_done);
  }
}

// The CG step after z is known: Ap, alpha, x/r update, r.r, the test, and
// (mixed form) the true-residual refresh.  Stages 3 and 4 of mg_launch_stage.
// The fastest axis of level 0 holds whole 4-cell groups (16-byte vectors).
bool x_by4(const mg_plan* P) { return P->geom[0].n[P->d.dim - 1] % 4 == 0; }

int launch_cg_tail(mg_plan* P, cudaStream_t s, int which) {
  const Level& L0 = P->lv[0];
  float* b = fptr(P, MG_FIELD_B);
  float* x = fptr(P, MG_FIELD_X);
  float* p = fptr(P, MG_FIELD_P);
  float* Ap = fptr(P, MG_FIELD_AP);
  const int RB = P->red_blocks;
  const bool refresh = P->d.refresh_every > 0;
  if (which & 1) {
    const float* pc = p;
    if (P->fp.valid && !P->fp.sto && x_by4(P))  // label-uniform level 0, 4-cell groups
      CK(launch_k(k_Ap_alpha_uniform4, RB, kRedThreads, 0, s, L0, pc, Ap, P->offdiag[0], P->ctl, P->partials, 0));
    else if (P->fp.valid && !P->fp.sto)
      CK(launch_k(k_Ap_alpha_uniform, RB, kRedThreads, 0, s, L0, pc, Ap, P->offdiag[0], P->ctl, P->partials, 0));
    else if (x_by4(P))
      CK(launch_k(k_Ap_alpha4, RB, kRedThreads, 0, s, L0, pc, Ap, P->ctl, P->partials, 0));
    else
      CK(launch_k(k_Ap_alpha, RB, kRedThreads, 0, s, L0, pc, Ap, P->ctl, P->partials, 0));
  }
  if (which & 2) {
    const float* pc = p;
    const float* Apc = Ap;
    double* xh = xhptr(P);
    if (P->geom[0].count % 4 == 0)  // 4-cell groups
      CK(launch_k(k_xr4, RB, kRedThreads, 0, s, L0, x, pc, Apc, P->ctl, P->partials, P->cond,
                  refresh ? 0 : P->has_cond, 0, xh));
    else
      CK(launch_k(k_xr, RB, kRedThreads, 0, s, L0, x, pc, Apc, P->ctl, P->partials, P->cond,
                  refresh ? 0 : P->has_cond, 0, xh));
    if (refresh) {
      const float* bc = b;
      const double* xhc = xh;
      CK(launch_k(k_refresh, RB, kRedThreads, 0, s, L0, bc, x, P->ctl, P->partials, P->cond, P->has_cond, xhc));
    }
  }
  return MG_OK;
}

// The PCG loop as launches (mgpcg.py:150-209).  `prologue` selects the part
// before the while node; otherwise the while-node body.
int launch_pcg_part(mg_plan* P, bool prologue, cudaStream_t s) {
  const Level& L0 = P->lv[0];
  float* b = fptr(P, MG_FIELD_B);
  float* x = fptr(P, MG_FIELD_X);
  if (prologue) {
    const float* bc = b;
    CK(launch_k(k_pcg_begin, P->red_blocks, kRedThreads, 0, s, L0, bc, x, P->ctl, P->partials, xhptr(P)));
  }
  const bool fuse = zr_fusable(P);
  P->fp.zr_mode = fuse ? (prologue ? 0 : 1) : -1;
  P->fp.zr_ctl = P->ctl;
  P->fp.zr_partials = P->partials;
  const int rc = launch_vcycle(P, s);
  P->fp.zr_mode = -1;
  if (rc) return rc;
  if (int rc2 = launch_zr_p_any(P, prologue, s, fuse)) return rc2;
  return launch_cg_tail(P, s, 3);
}

// Kernels one launch_pcg_part enqueues (the graph's node count per part).
int count_pcg_part(const mg_plan* P, bool prologue) {
  const int refresh = P->d.refresh_every > 0 ? 1 : 0;
  if (P->fp.valid) {
    int v = 1;  // the coarse block, or the cluster-resident launch
    const int streamed = P->fp.res ? P->fp.res_lp : P->fp.lc;
    for (int l = 0; l < streamed; ++l) v += P->fp.split[l] ? 2 * (2 * P->d.pre_post + 1) : 2;
    return (prologue ? 1 : 0) + v + (zr_fusable(P) ? 3 : 4) + refresh;
  }
  int v = (P->L - 1) * (4 * P->d.pre_post + 2) +
          (P->geom[P->L - 1].count <= kBottomBlockCells ? (P->d.bottom / 2 > 0) : 2 * P->d.bottom);
  return (prologue ? 1 : 0) + v + 2 + 2 + refresh;
}

void destroy_graph(mg_plan* P) {
  if (P->exec) cudaGraphExecDestroy(P->exec);
  if (P->graph) cudaGraphDestroy(P->graph);
  P->exec = nullptr;
  P->graph = nullptr;
  P->base_of_graph = nullptr;
}

// Builds graph = [prologue] -> while(cond) { body }.
int build_graph(mg_plan* P) {
  destroy_graph(P);
  if (!P->cap) CK(cudaStreamCreateWithFlags(&P->cap, cudaStreamNonBlocking));
  CK(cudaGraphCreate(&P->graph, 0));
  CK(cudaGraphConditionalHandleCreate(&P->cond, P->graph, 0, cudaGraphCondAssignDefault));
  CK(cudaStreamBeginCaptureToGraph(P->cap, P->graph, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  int rc = launch_pcg_part(P, true, P->cap);
  if (rc) {
    cudaGraph_t g;
    cudaStreamEndCapture(P->cap, &g);
    return rc;
  }
  cudaStreamCaptureStatus st;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  cudaGraph_t capg;
  CK(cudaStreamGetCaptureInfo(P->cap, &st, nullptr, &capg, &deps, &ndeps));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = P->cond;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cnode;
  CK(cudaGraphAddNode(&cnode, capg, deps, ndeps, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  CK(cudaStreamUpdateCaptureDependencies(P->cap, &cnode, 1, cudaStreamSetCaptureDependencies));
  cudaGraph_t out;
  CK(cudaStreamEndCapture(P->cap, &out));
  CK(cudaStreamBeginCaptureToGraph(P->cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  rc = launch_pcg_part(P, false, P->cap);
  {
    cudaGraph_t g2;
    cudaError_t e = cudaStreamEndCapture(P->cap, &g2);
    if (rc) return rc;
    if (e != cudaSuccess) return set_err("cudaStreamEndCapture(body)", e);
  }
  CK(cudaGraphInstantiate(&P->exec, P->graph, 0));
  P->base_of_graph = P->base;
  return MG_OK;
}

// The graph's prologue and loop body launched from the host (MG_PLAN_DIRECT):
// after each part the host reads Control::run, which the body's last kernel
// sets exactly where the graph's while condition is set.
constexpr int kDirectMaxParts = 1 << 20;

int solve_direct(mg_plan* P, const mg_solve_params_t* prm, cudaStream_t s) {
  k_set_params<<<1, 1, 0, s>>>(P->ctl, *prm, P->d.refresh_every);
  CKL("k_set_params");
  const int saved = P->has_cond;
  P->has_cond = 0;
  int rc = launch_pcg_part(P, true, s);
  for (int part = 0; rc == MG_OK && part < kDirectMaxParts; ++part) {
    cudaError_t e = cudaMemcpyAsync(&P->host_ctl->run, &P->ctl->run, sizeof(P->ctl->run), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      rc = set_err("solve_direct", e);
      break;
    }
    if (!P->host_ctl->run) break;
    rc = launch_pcg_part(P, false, s);
  }
  P->has_cond = saved;
  return rc;
}

}  // namespace

// Lets the library's other translation units record an error message.
void mg_internal_set_error(const char* msg) { snprintf(g_err, sizeof(g_err), "%s", msg); }

static int finish_prepare(mg_plan_t* P, cudaStream_t s, int declared);

// ============================================================================
// C ABI
// ============================================================================
extern "C" {

const char* mg_last_error(void) { return g_err; }
int32_t mg_version(void) { return 10000; }

int mg_plan_create(const mg_plan_desc_t* desc, mg_plan_t** out) {
  if (!desc || !out) return bad("null pointer");
  const mg_plan_desc_t& d = *desc;
  if (d.dim != 2 && d.dim != 3) return bad("dim must be 2 or 3");
  if (d.levels < 1 || d.levels > kMaxLevels) return bad("levels out of range");
  if (d.pre_post < 0 || d.bottom < 0) return bad("negative sweep count");
  if (d.storage < MG_STORE_F32 || d.storage > MG_STORE_BF16) return bad("storage");
  for (int k = 0; k < d.dim; ++k) {
    if (d.res[k] < 2) return bad("res must be >= 2");
    if (d.res[k] % (1 << (d.levels - 1)) != 0) return bad("res must be divisible by 2^(levels-1)");
  }
  if ((long long)d.res[0] * d.res[1] * (d.dim == 3 ? d.res[2] : 1) >= (1LL << 31)) {
    snprintf(g_err, sizeof(g_err), "a level of 2^31 cells or more exceeds the 32-bit cell index of the kernels");
    return MG_E_TOO_BIG;
  }
  mg_plan* P = new (std::nothrow) mg_plan();
  if (!P) return bad("out of host memory");
  P->d = d;
  P->L = d.levels;
  for (int l = 0; l < P->L; ++l) {
    Geom& g = P->geom[l];
    g.dim = d.dim;
    g.n[0] = d.res[0] >> l;
    g.n[1] = d.res[1] >> l;
    g.n[2] = d.dim == 3 ? (d.res[2] >> l) : 1;
    g.count = (long long)g.n[0] * g.n[1] * g.n[2];
    P->op_form[l] = 0;
    P->whole[l] = 0;
  }
  layout(P);
  cudaGetDevice(&P->device);
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, P->device) == cudaSuccess && sms > 0)
    P->num_sms = sms;
  cudaGetLastError();
  int64_t n0 = P->geom[0].count;
  int64_t rb = (n0 + kRedThreads * 8 - 1) / (kRedThreads * 8);
  if (rb > P->num_sms * MG_RED_BLOCKS_PER_SM) rb = P->num_sms * MG_RED_BLOCKS_PER_SM;
  if (rb > kMaxPartials / 2) rb = kMaxPartials / 2;  // two partial regions (b.b and r.r)
  if (rb < 1) rb = 1;
  P->red_blocks = (int)rb;
  for (int l = 0; l < P->L; ++l) P->ew_blocks[l] = grid_for(P, P->geom[l].count);
  *out = P;
  return MG_OK;
}

int mg_plan_destroy(mg_plan_t* P) {
  if (!P) return MG_OK;
  destroy_graph(P);
  if (P->cap) cudaStreamDestroy(P->cap);
  if (P->host_ctl) cudaFreeHost(P->host_ctl);
  delete P;
  return MG_OK;
}

int64_t mg_plan_workspace_bytes(const mg_plan_t* P) { return P ? P->ws_bytes : -1; }

int mg_plan_field(const mg_plan_t* P, int32_t field, int32_t level, int32_t comp, int64_t* offset,
                  int64_t* nbytes) {
  if (!P || !offset || !nbytes) return bad("null pointer");
  if (field < 0 || field >= kFields) return bad("field id");
  if (level < 0 || level >= P->L) return bad("level");
  bool level0_only = field == MG_FIELD_B || field == MG_FIELD_X || field == MG_FIELD_P || field == MG_FIELD_AP;
  if (level0_only && level != 0) return bad("field exists on level 0 only");
  int ncomp = field == MG_FIELD_AX ? P->d.dim : 1;
  if (comp < 0 || comp >= ncomp) return bad("component");
  *offset = P->loc[field][level][comp].off;
  *nbytes = P->loc[field][level][comp].bytes;
  return MG_OK;
}

int mg_plan_bind(mg_plan_t* P, void* ws) {
  if (!P || !ws) return bad("null pointer");
  if (((uintptr_t)ws & 255u) != 0) return bad("workspace must be 256-byte aligned");
  P->base = (char*)ws;
  bind_views(P);
  if (!P->host_ctl) CK(cudaMallocHost(&P->host_ctl, sizeof(Control)));
  return MG_OK;
}

#define NEED_BOUND(P)                        \
  do {                                       \
    if (!(P)) return bad("null plan");       \
    if (!(P)->base) {                        \
      snprintf(g_err, sizeof(g_err), "plan has no workspace"); \
      return MG_E_UNBOUND;                   \
    }                                        \
  } while (0)

int mg_initialize(mg_plan_t* P, void* stream) {
  NEED_BOUND(P);
  // Every field, including the control block (counters, beta).
  CK(cudaMemsetAsync(P->base, 0, P->ws_bytes, S(stream)));
  P->prepared = false;
  return MG_OK;
}

int mg_set_cell_type(mg_plan_t* P, const int32_t* ct, void* stream) {
  NEED_BOUND(P);
  if (!ct) return bad("cell_type");
  k_set_cell_type<<<P->ew_blocks[0], 256, 0, S(stream)>>>(ct, P->lv[0].type, P->geom[0].count);
  CKL("k_set_cell_type");
  P->prepared = false;
  return MG_OK;
}

int mg_init_gridtype(mg_plan_t* P, int32_t level, void* stream) {
  NEED_BOUND(P);
  if (level < 1 || level >= P->L) return bad("level");
  k_init_gridtype<<<P->ew_blocks[level], 256, 0, S(stream)>>>(P->lv[level - 1], P->lv[level]);
  CKL("k_init_gridtype");
  P->prepared = false;
  return MG_OK;
}

int mg_fill_fluid(mg_plan_t* P, void* stream) {
  NEED_BOUND(P);
  for (int l = 0; l < P->L; ++l) CK(cudaMemsetAsync(P->lv[l].type, MG_FLUID, P->geom[l].count, S(stream)));
  P->prepared = false;
  return MG_OK;
}

int mg_build_pressure_b(mg_plan_t* P, const float* v0, const float* v1, const float* v2, const float* phi,
                        float p0, float sA, float sB, int32_t ghost, float clamp, void* stream) {
  NEED_BOUND(P);
  if (!v0 || !v1 || (P->d.dim == 3 && !v2)) return bad("velocity");
  if (ghost && !phi) return bad("phi");
  k_build_pressure_b<<<P->ew_blocks[0], 256, 0, S(stream)>>>(P->lv[0], v0, v1, v2, phi, p0, sA, sB, ghost,
                                                             clamp, fptr(P, MG_FIELD_B));
  CKL("k_build_pressure_b");
  return MG_OK;
}

int mg_build_pressure_A(mg_plan_t* P, int32_t level, const float* phi, float sA, int32_t ghost, float clamp,
                        void* stream) {
  NEED_BOUND(P);
  if (level < 0 || level >= P->L) return bad("level");
  if (ghost && level == 0 && !phi) return bad("phi");
  k_build_pressure_A<<<P->ew_blocks[level], 256, 0, S(stream)>>>(P->lv[level], level, phi, sA, ghost, clamp);
  CKL("k_build_pressure_A");
  P->prepared = false;
  return MG_OK;
}

int mg_build_psi_b(mg_plan_t* P, const float* chi, float H0, float H1, float H2, float dx, int32_t p0,
                   int32_t p1, int32_t p2, void* stream) {
  NEED_BOUND(P);
  if (!chi || !(dx > 0.0f)) return bad("chi / dx");
  k_build_psi_b<<<P->ew_blocks[0], 256, 0, S(stream)>>>(P->lv[0], fptr(P, MG_FIELD_B), chi, H0, H1, H2, dx, p0,
                                                         p1, P->d.dim == 3 ? p2 : 0);
  CKL("k_build_psi_b");
  return MG_OK;
}

int mg_build_psi_A(mg_plan_t* P, const float* chi, float dx, int32_t p0, int32_t p1, int32_t p2, void* stream) {
  NEED_BOUND(P);
  if (!chi || !(dx > 0.0f)) return bad("chi / dx");
  k_build_psi_A<<<P->ew_blocks[0], 256, 0, S(stream)>>>(P->lv[0], chi, dx, p0, p1, P->d.dim == 3 ? p2 : 0);
  CKL("k_build_psi_A");
  P->prepared = false;
  return MG_OK;
}

int mg_build_psi_A_level(mg_plan_t* P, int32_t level, const float* chi_fine, float* chi_level, float dx,
                         int32_t p0, int32_t p1, int32_t p2, void* stream) {
  NEED_BOUND(P);
  if (level < 1 || level >= P->L) return bad("level");
  if (!chi_fine || !chi_level || !(dx > 0.0f)) return bad("chi / dx");
  k_mean_children<<<P->ew_blocks[level], 256, 0, S(stream)>>>(P->geom[level - 1], chi_fine, P->geom[level],
                                                               chi_level);
  CKL("k_mean_children");
  const float dxl = dx * (float)(1 << level);  // exact: a power of two
  k_build_psi_A<<<P->ew_blocks[level], 256, 0, S(stream)>>>(P->lv[level], chi_level, dxl, p0 >> level, p1 >> level,
                                                             P->d.dim == 3 ? (p2 >> level) : 0);
  CKL("k_build_psi_A");
  P->prepared = false;
  return MG_OK;
}

int mg_galerkin_coarsen(mg_plan_t* P, int32_t level, float scale, void* stream) {
  NEED_BOUND(P);
  if (level < 1 || level >= P->L) return bad("level");
  int e2 = 0;
  if (!(scale > 0.0f) || std::frexp(scale, &e2) != 0.5f) return bad("scale must be a power of two");
  k_galerkin<<<P->ew_blocks[level], 256, 0, S(stream)>>>(P->lv[level - 1], P->lv[level], scale);
  CKL("k_galerkin");
  P->prepared = false;
  return MG_OK;
}

int mg_add_rhs(mg_plan_t* P, const float* src, float c, void* stream) {
  NEED_BOUND(P);
  k_add_rhs<<<P->ew_blocks[0], 256, 0, S(stream)>>>(P->lv[0], fptr(P, MG_FIELD_B), src, c);
  CKL("k_add_rhs");
  return MG_OK;
}

// ---- the other Strategies and the pressure-gradient update -----------------

namespace {
ThetaK theta_consts(float eps) {
  ThetaK t;
  t.eps = eps;
  t.two_eps = (float)(2.0 * (double)eps);
  t.pi = (float)3.14159265358979323846;
  t.inv_2pi = (float)(1.0 / (2.0 * 3.14159265358979323846));
  return t;
}
}  // namespace

int mg_apply_pressure(mg_plan_t* P, float* u0, float* u1, float* u2, const float* pressure,
                      const int32_t* cell_type, const float* phi, float scale, float p0, int32_t ghost,
                      float clamp, void* stream) {
  NEED_BOUND(P);
  float* u[3] = {u0, u1, u2};
  for (int k = 0; k < P->d.dim; ++k)
    if (!u[k]) return bad("velocity");
  if (ghost && !phi) return bad("phi");
  const float* pr = pressure ? pressure : fptr(P, MG_FIELD_X);
  for (int k = 0; k < P->d.dim; ++k) {
    k_apply_pressure<<<P->ew_blocks[0], 256, 0, S(stream)>>>(P->lv[0], k, u[k], pr, cell_type, phi, scale, p0,
                                                             ghost, clamp, nullptr, nullptr, nullptr, 0.0f);
    CKL("k_apply_pressure");
  }
  return MG_OK;
}

int mg_apply_magnetic_force(mg_plan_t* P, float* u0, float* u1, float* u2, const float* pressure,
                            const int32_t* cell_type, const float* H0, const float* H1, const float* H2,
                            float scale, float p0, float coef, void* stream) {
  NEED_BOUND(P);
  float* u[3] = {u0, u1, u2};
  for (int k = 0; k < P->d.dim; ++k)
    if (!u[k]) return bad("velocity");
  if (!H0 || !H1 || (P->d.dim == 3 && !H2)) return bad("H");
  const float* pr = pressure ? pressure : fptr(P, MG_FIELD_X);
  for (int k = 0; k < P->d.dim; ++k) {
    k_apply_pressure<<<P->ew_blocks[0], 256, 0, S(stream)>>>(P->lv[0], k, u[k], pr, cell_type, nullptr, scale,
                                                             p0, 0, 0.0f, H0, H1, H2, coef);
    CKL("k_apply_pressure");
  }
  return MG_OK;
}

int mg_level_set_volume(mg_plan_t* P, const float* phi, float eps, double* out, void* stream) {
  NEED_BOUND(P);
  if (!phi || !out || !(eps > 0.0f)) return bad("phi / eps / out");
  k_volume<<<P->red_blocks, kRedThreads, 0, S(stream)>>>(P->geom[0], phi, theta_consts(eps), P->partials,
                                                         &P->ctl->counter[4], out, nullptr);
  CKL("k_volume");
  return MG_OK;
}

int mg_volume_control(mg_plan_t* P, const float* phi, float eps, double* state, void* stream) {
  NEED_BOUND(P);
  if (!phi || !state || !(eps > 0.0f)) return bad("phi / eps / state");
  k_volume<<<P->red_blocks, kRedThreads, 0, S(stream)>>>(P->geom[0], phi, theta_consts(eps), P->partials,
                                                         &P->ctl->counter[4], &state[3], state);
  CKL("k_volume");
  k_add_c<<<P->ew_blocks[0], 256, 0, S(stream)>>>(P->lv[0], fptr(P, MG_FIELD_B), state);
  CKL("k_add_c");
  return MG_OK;
}

int mg_build_magnetic_b(mg_plan_t* P, const float* v0, const float* v1, const float* v2, const float* H0,
                        const float* H1, const float* H2, float p0, float sA, float sB, float coef, void* stream) {
  NEED_BOUND(P);
  if (!v0 || !v1 || (P->d.dim == 3 && !v2)) return bad("velocity");
  if (!H0 || !H1 || (P->d.dim == 3 && !H2)) return bad("H");
  k_build_magnetic_b<<<P->ew_blocks[0], 256, 0, S(stream)>>>(P->lv[0], v0, v1, v2, H0, H1, H2, p0, sA, sB, coef,
                                                             fptr(P, MG_FIELD_B));
  CKL("k_build_magnetic_b");
  return MG_OK;
}

int mg_build_potential_b(mg_plan_t* P, const float* chi, const float* Hx0, const float* Hx1, const float* Hx2,
                         void* stream) {
  NEED_BOUND(P);
  if (!chi || !Hx0 || !Hx1 || (P->d.dim == 3 && !Hx2)) return bad("chi / H_ext");
  const Geom& g = P->geom[0];
  k_build_potential_b<<<P->ew_blocks[0], 256, 0, S(stream)>>>(P->lv[0], fptr(P, MG_FIELD_B), chi, Hx0, Hx1, Hx2,
                                                              g.n[0], g.n[1], g.n[2]);
  CKL("k_build_potential_b");
  return MG_OK;
}

int mg_build_potential_A(mg_plan_t* P, int32_t level, const float* chi, double dx, void* stream) {
  NEED_BOUND(P);
  if (level < 0 || level >= P->L) return bad("level");
  if (!chi || !(dx > 0.0)) return bad("chi / dx");
  const Geom& g = P->geom[0];
  const double dxl = dx * (double)(1 << level);
  k_build_potential_A<<<P->ew_blocks[level], 256, 0, S(stream)>>>(P->lv[level], level, chi, g, (float)dxl,
                                                                  (float)(1.0 / dxl), g.n[0], g.n[1], g.n[2]);
  CKL("k_build_potential_A");
  P->prepared = false;
  return MG_OK;
}

// ---- labels and level set from shapes (no plan: a grid shape suffices) ------

namespace {
int grid_of(int32_t dim, const int32_t* res, Geom* g) {
  if ((dim != 2 && dim != 3) || !res) return bad("dim / res");
  g->dim = dim;
  for (int k = 0; k < 3; ++k) g->n[k] = k < dim ? res[k] : 1;
  for (int k = 0; k < dim; ++k)
    if (g->n[k] < 1) return bad("res");
  g->count = (long long)g->n[0] * g->n[1] * g->n[2];
  return MG_OK;
}
int blocks_of(long long n) {
  long long b = (n + 255) / 256;
  return (int)(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}
}  // namespace

int mg_level_set_shape(int32_t dim, const int32_t* res, float* phi, float dx, int32_t sphere, const float* a,
                       const float* b, int32_t combine, void* stream) {
  Geom g;
  if (int rc = grid_of(dim, res, &g)) return rc;
  if (!phi || !a || !b || !(dx > 0.0f)) return bad("phi / shape / dx");
  float A[3] = {0.0f, 0.0f, 0.0f}, B[3] = {0.0f, 0.0f, 0.0f};
  for (int k = 0; k < dim; ++k) A[k] = a[k];
  if (sphere) B[0] = b[0];
  else
    for (int k = 0; k < dim; ++k) B[k] = b[k];
  k_ls_shape<<<blocks_of(g.count), 256, 0, S(stream)>>>(g, phi, dx, sphere ? 1 : 0, A[0], A[1], A[2], B[0], B[1],
                                                          B[2], combine);
  CKL("k_ls_shape");
  return MG_OK;
}

int mg_apply_markers(int32_t dim, const int32_t* res, int32_t* cell_type, const float* phi, int32_t strict,
                     void* stream) {
  Geom g;
  if (int rc = grid_of(dim, res, &g)) return rc;
  if (!cell_type || !phi) return bad("cell_type / phi");
  k_apply_markers<<<blocks_of(g.count), 256, 0, S(stream)>>>(g, cell_type, phi, strict);
  CKL("k_apply_markers");
  return MG_OK;
}

int mg_init_boundary(int32_t dim, const int32_t* res, int32_t* cell_type, void* stream) {
  Geom g;
  if (int rc = grid_of(dim, res, &g)) return rc;
  if (!cell_type) return bad("cell_type");
  k_init_boundary<<<blocks_of(g.count), 256, 0, S(stream)>>>(g, cell_type);
  CKL("k_init_boundary");
  return MG_OK;
}

// FastSweepingLevelSet.propagate (level_set.py:283-327): repeat rounds of the
// 2 dim sweeps, fastest axis first, forward then backward.
static int fs_propagate(const Geom& g, const float* phi, float* phi_temp, const int32_t* valid, double dx,
                        int repeat_times, cudaStream_t s) {
  const float dx1 = (float)dx, two_dx2 = (float)(2.0 * dx * dx), dx2 = (float)(dx * dx), third = (float)(1.0 / 3.0);
  for (int t = 0; t < repeat_times; ++t)
    for (int axis = g.dim - 1; axis >= 0; --axis)
      for (int dir = 1; dir >= -1; dir -= 2) {
        const long long lines = g.count / g.n[axis];
        const int blocks = (int)((lines + 127) / 128);
        k_fs_sweep<<<blocks, 128, 0, s>>>(g, axis, dir, phi_temp, phi, valid, dx1, two_dx2, dx2, third);
        CKL("k_fs_sweep");
      }
  return MG_OK;
}

int mg_level_set_redistance(int32_t dim, const int32_t* res, float* phi, float* phi_temp, int32_t* valid,
                            double dx, int32_t repeat_times, void* stream) {
  Geom g;
  if (int rc = grid_of(dim, res, &g)) return rc;
  for (int k = 0; k < dim; ++k)
    if (g.n[k] < 2) return bad("every axis needs at least 2 cells");
  if (!phi || !phi_temp || !valid || !(dx > 0.0) || repeat_times < 0) return bad("inputs");
  cudaStream_t s = S(stream);
  k_target_surface<<<blocks_of(g.count), 256, 0, s>>>(g, phi, phi_temp, valid, (float)dx);
  CKL("k_target_surface");
  if (int rc = fs_propagate(g, phi, phi_temp, valid, dx, repeat_times, s)) return rc;
  CK(cudaMemcpyAsync(phi, phi_temp, g.count * sizeof(float), cudaMemcpyDeviceToDevice, s));
  return MG_OK;
}

int mg_level_set_propagate(int32_t dim, const int32_t* res, const float* phi, float* phi_temp, const int32_t* valid,
                           double dx, int32_t repeat_times, void* stream) {
  Geom g;
  if (int rc = grid_of(dim, res, &g)) return rc;
  for (int k = 0; k < dim; ++k)
    if (g.n[k] < 2) return bad("every axis needs at least 2 cells");
  if (!phi || !phi_temp || !valid || !(dx > 0.0) || repeat_times < 0) return bad("inputs");
  return fs_propagate(g, phi, phi_temp, valid, dx, repeat_times, S(stream));
}

int mg_level_set_markers_distance(int32_t dim, const int32_t* res, float* phi, int32_t* valid, const float* markers,
                                  int32_t n_markers, double dx, int32_t repeat_times, void* stream) {
  Geom g;
  if (int rc = grid_of(dim, res, &g)) return rc;
  if (!phi || !valid || (n_markers > 0 && !markers) || n_markers < 0 || !(dx > 0.0) || repeat_times < 0)
    return bad("inputs");
  cudaStream_t s = S(stream);
  const float fdx = (float)dx;
  k_markers_init<<<blocks_of(g.count), 256, 0, s>>>(g, phi, valid);
  CKL("k_markers_init");
  if (n_markers > 0) {
    const int mb = (n_markers + 255) / 256 < 4096 ? (n_markers + 255) / 256 : 4096;
    k_marker_min_d<<<mb, 256, 0, s>>>(g, markers, n_markers, fdx, phi);
    CKL("k_marker_min_d");
    k_marker_owner<<<mb, 256, 0, s>>>(g, markers, n_markers, fdx, phi, valid);
    CKL("k_marker_owner");
  }
  k_marker_valid_fix<<<blocks_of(g.count), 256, 0, s>>>(g, valid);
  CKL("k_marker_valid_fix");
  for (int t = 0; t < repeat_times; ++t)
    for (int axis = dim - 1; axis >= 0; --axis)
      for (int dir = 1; dir >= -1; dir -= 2) {
        const long long lines = g.count / g.n[axis];
        k_marker_sweep<<<(int)((lines + 127) / 128), 128, 0, s>>>(g, axis, dir, markers, fdx, phi, valid);
        CKL("k_marker_sweep");
      }
  return MG_OK;
}

int mg_level_set_target_minus(int32_t dim, const int32_t* res, float* phi, float* phi_temp, int32_t* valid,
                              double dx, void* stream) {
  Geom g;
  if (int rc = grid_of(dim, res, &g)) return rc;
  if (!phi || !phi_temp || !valid || !(dx > 0.0)) return bad("inputs");
  cudaStream_t s = S(stream);
  k_target_minus_a<<<blocks_of(g.count), 256, 0, s>>>(g, phi, valid, (float)(0.99 * dx));
  CKL("k_target_minus_a");
  k_target_minus_b<<<blocks_of(g.count), 256, 0, s>>>(g, phi, phi_temp, valid);
  CKL("k_target_minus_b");
  return MG_OK;
}

int mg_level_set_smooth(int32_t dim, const int32_t* res, float* out, const float* in, void* stream) {
  Geom g;
  if (int rc = grid_of(dim, res, &g)) return rc;
  if (!out || !in || out == in) return bad("inputs (out and in must differ)");
  k_ls_smooth<<<blocks_of(g.count), 256, 0, S(stream)>>>(g, out, in);
  CKL("k_ls_smooth");
  return MG_OK;
}

// ---- advection, extrapolation, gravity, solid boundary (plan-free) --------

int mg_advect_quantity(int32_t dim, const int32_t* res, const float* u0, const float* u1, const float* u2,
                       const float* phi, float* phi_out, float* u0_out, float* u1_out, float* u2_out, float dx,
                       float dt, void* stream) {
  Geom g;
  if (int rc = grid_of(dim, res, &g)) return rc;
  const float* u[3] = {u0, u1, u2};
  float* uo[3] = {u0_out, u1_out, u2_out};
  for (int k = 0; k < dim; ++k)
    if (!u[k] || !uo[k]) return bad("velocity");
  if (phi_out && !phi) return bad("phi");
  if (!(dx > 0.0f)) return bad("dx");
  Vel V;
  for (int k = 0; k < 3; ++k) V.u[k] = k < dim ? u[k] : nullptr;
  if (phi_out) {
    k_advect<<<blocks_of(g.count), 256, 0, S(stream)>>>(g, -1, V, phi, phi_out, dx, dt);
    CKL("k_advect");
  }
  for (int k = 0; k < dim; ++k) {
    const long long nf = g.count / g.n[k] * (g.n[k] + 1);
    k_advect<<<blocks_of(nf), 256, 0, S(stream)>>>(g, k, V, u[k], uo[k], dx, dt);
    CKL("k_advect");
  }
  return MG_OK;
}

int mg_extrapolate_velocity(int32_t dim, const int32_t* res, int32_t k, float* u, float* u_tmp, int32_t* valid,
                            int32_t* valid_tmp, const int32_t* cell_type, int32_t iterations, void* stream) {
  Geom g;
  if (int rc = grid_of(dim, res, &g)) return rc;
  if (k < 0 || k >= dim) return bad("axis");
  if (!u || !u_tmp || !valid || !valid_tmp || !cell_type || iterations < 0) return bad("inputs");
  cudaStream_t s = S(stream);
  const long long nf = g.count / g.n[k] * (g.n[k] + 1);
  k_mark_valid<<<blocks_of(nf), 256, 0, s>>>(g, k, cell_type, valid);
  CKL("k_mark_valid");
  float* a = u;
  float* b = u_tmp;
  int32_t* va = valid;
  int32_t* vb = valid_tmp;
  for (int it = 0; it < iterations; ++it) {
    k_diffuse<<<blocks_of(nf), 256, 0, s>>>(g, k, a, b, va, vb);
    CKL("k_diffuse");
    std::swap(a, b);
    std::swap(va, vb);
  }
  if (a != u) {  // an odd round count ends in the scratch buffers
    CK(cudaMemcpyAsync(u, a, nf * sizeof(float), cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(valid, va, nf * sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
  }
  return MG_OK;
}

int mg_enforce_boundary(int32_t dim, const int32_t* res, float* u0, float* u1, float* u2, const int32_t* cell_type,
                        void* stream) {
  Geom g;
  if (int rc = grid_of(dim, res, &g)) return rc;
  float* u[3] = {u0, u1, u2};
  for (int k = 0; k < dim; ++k)
    if (!u[k]) return bad("velocity");
  if (!cell_type) return bad("cell_type");
  Vel V;
  for (int k = 0; k < 3; ++k) V.u[k] = k < dim ? u[k] : nullptr;
  k_enforce_boundary<<<blocks_of(g.count), 256, 0, S(stream)>>>(g, V, cell_type);
  CKL("k_enforce_boundary");
  return MG_OK;
}

int mg_add_gravity(int32_t dim, const int32_t* res, float* u0, float* u1, float* u2, double g0, double g1, double g2,
                   float dt, void* stream) {
  Geom g;
  if (int rc = grid_of(dim, res, &g)) return rc;
  float* u[3] = {u0, u1, u2};
  const double gv[3] = {g0, g1, g2};
  for (int k = 0; k < dim; ++k) {
    if (gv[k] == 0.0) continue;  // the reference skips zero components (ti.static)
    if (!u[k]) return bad("velocity");
    const long long nf = g.count / g.n[k] * (g.n[k] + 1);
    k_add_gravity<<<blocks_of(nf), 256, 0, S(stream)>>>(g, k, u[k], (float)gv[k], dt);
    CKL("k_add_gravity");
  }
  return MG_OK;
}

int mg_update_susceptibility(mg_plan_t* P, const float* phi, double k, float eps, float* chi, void* stream) {
  NEED_BOUND(P);
  if (!phi || !chi || !(eps > 0.0f)) return bad("phi / chi / eps");
  k_update_chi<<<P->ew_blocks[0], 256, 0, S(stream)>>>(P->geom[0], phi, (float)k, theta_consts(eps), chi);
  CKL("k_update_chi");
  return MG_OK;
}

int mg_update_magnetic_field(mg_plan_t* P, const float* psi, const float* Hext0, const float* Hext1,
                             const float* Hext2, float dx, float* H0, float* H1, float* H2, void* stream) {
  NEED_BOUND(P);
  const float* he[3] = {Hext0, Hext1, Hext2};
  float* h[3] = {H0, H1, H2};
  if (!(dx > 0.0f)) return bad("dx");
  for (int k = 0; k < P->d.dim; ++k)
    if (!he[k] || !h[k]) return bad("H / H_ext");
  const float* ps = psi ? psi : fptr(P, MG_FIELD_X);
  for (int k = 0; k < P->d.dim; ++k) {
    k_update_H<<<P->ew_blocks[0], 256, 0, S(stream)>>>(P->geom[0], k, ps, he[k], dx, h[k]);
    CKL("k_update_H");
  }
  return MG_OK;
}

int mg_calc_surface_normal(mg_plan_t* P, int32_t d, const float* phi, float dx, float* n, void* stream) {
  NEED_BOUND(P);
  if (d < 0 || d >= P->d.dim) return bad("axis");
  if (!phi || !n || !(dx > 0.0f)) return bad("phi / n / dx");
  k_calc_n<<<P->ew_blocks[0], 256, 0, S(stream)>>>(P->geom[0], d, phi, dx, n);
  CKL("k_calc_n");
  return MG_OK;
}

int mg_calc_curvature(mg_plan_t* P, const float* n, float dx, float* kappa, void* stream) {
  NEED_BOUND(P);
  if (!n || !kappa || !(dx > 0.0f)) return bad("n / kappa / dx");
  k_calc_kappa<<<P->ew_blocks[0], 256, 0, S(stream)>>>(P->geom[0], n, dx, kappa);
  CKL("k_calc_kappa");
  return MG_OK;
}

int mg_build_surface_tension_b(mg_plan_t* P, int32_t d, const float* u, const float* phi, const float* n,
                               const float* kappa, double sigma, double dt, double dx, double eps, void* stream) {
  NEED_BOUND(P);
  if (d < 0 || d >= P->d.dim) return bad("axis");
  if (!u || !phi || !n || !kappa || !(dt > 0.0) || !(dx > 0.0) || !(eps > 0.0)) return bad("inputs");
  k_build_st_b<<<P->ew_blocks[0], 256, 0, S(stream)>>>(P->geom[0], d, u, phi, n, kappa, (float)sigma, (float)dt,
                                                       (float)dx, (float)(dx * dx), theta_consts((float)eps),
                                                       fptr(P, MG_FIELD_B));
  CKL("k_build_st_b");
  return MG_OK;
}

int mg_build_surface_tension_A(mg_plan_t* P, int32_t level, int32_t d, const float* phi, double sigma, double dt,
                               double dx, double eps, void* stream) {
  NEED_BOUND(P);
  if (level < 0 || level >= P->L) return bad("level");
  if (d < 0 || d >= P->d.dim) return bad("axis");
  if (!phi || !(dt > 0.0) || !(dx > 0.0) || !(eps > 0.0)) return bad("inputs");
  const double dxl = dx * (double)(1 << level);
  const float scale = (float)(sigma * dt / (dxl * dxl));
  k_build_st_A<<<P->ew_blocks[level], 256, 0, S(stream)>>>(P->lv[level], level, P->geom[0], d, phi,
                                                           (float)(1.0 / dt), scale, theta_consts((float)eps));
  CKL("k_build_st_A");
  P->prepared = false;
  return MG_OK;
}

int mg_plan_prepare(mg_plan_t* P, void* stream) {
  NEED_BOUND(P);
  cudaStream_t s = S(stream);
  // 1. operator form of every level (one synchronisation for all levels)
  const int blocks = P->num_sms * 2 < kMaxPartials / 4 ? P->num_sms * 2 : kMaxPartials / 4;
  for (int l = 0; l < P->L; ++l) {
    const int nb = grid_for(P, P->geom[l].count) < blocks ? grid_for(P, P->geom[l].count) : blocks;
    k_detect_uniform<<<nb, kRedThreads, 0, s>>>(P->lv[l], P->partials, &P->ctl->counter[5], &P->ctl->det[4 * l]);
    CKL("k_detect_uniform");
  }
  double det[4 * kMaxLevels];
  CK(cudaMemcpyAsync(det, P->ctl->det, sizeof(double) * 4 * P->L, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  for (int l = 0; l < P->L; ++l) {
    const double* h = det + 4 * l;
    const bool none = h[0] > h[1];  // no nonzero off-diagonal at all
    const bool uniform = h[2] == 0.0 && (none || (h[0] == h[1] && h[0] < 0.0));
    P->op_form[l] = uniform ? 1 : 0;
    P->offdiag[l] = uniform && !none ? (float)(-h[0]) : 0.0f;
    P->whole[l] = h[3] == 0.0 ? 1 : 0;  // every cell FLUID with a nonzero diagonal
  }
  return finish_prepare(P, s, 0);
}

int mg_plan_prepare_declared(mg_plan_t* P, const float* offdiag, void* stream) {
  NEED_BOUND(P);
  if (!offdiag) return bad("offdiag");
  for (int l = 0; l < P->L; ++l) {
    P->op_form[l] = 1;
    P->offdiag[l] = offdiag[l];
    P->whole[l] = 0;
  }
  return finish_prepare(P, S(stream), 1);
}

int mg_plan_prepare_declared_whole(mg_plan_t* P, void* stream) {
  NEED_BOUND(P);
  for (int l = 0; l < P->L; ++l) {
    P->op_form[l] = 0;
    P->offdiag[l] = 0.0f;
    P->whole[l] = 1;
  }
  return finish_prepare(P, S(stream), 2);
}

}  // extern "C"

// Launch shapes, 16-bit coefficient copies, FLUID count, scale factors and
// (declared forms: 1 label-uniform, 2 whole-domain) the asynchronous
// verification; no host synchronization.
static int finish_prepare(mg_plan_t* P, cudaStream_t s, int declared) {
  // 2. launch shapes of the fused V-cycle
  P->fp.valid = false;
  if (!(P->d.flags & MG_PLAN_STORED))
    make_fused_plan(P->lv, P->L, P->d.dim, P->d.pre_post, P->d.bottom, P->d.storage, P->op_form, P->whole,
                    P->offdiag, P->num_sms, &P->fp);
  if (P->d.storage != MG_STORE_F32 && !P->fp.valid)
    return bad("16-bit storage needs the label-uniform operator on every level and pre_and_post_smoothing 1..3");
  // 3. 16-bit coefficient copies, FLUID count, scale factors
  if (P->d.storage == MG_STORE_F16 || P->d.storage == MG_STORE_BF16) {
    for (int l = 0; l < P->L; ++l) {
      if (P->d.storage == MG_STORE_F16)
        k_store_diag<__half><<<P->ew_blocks[l], 256, 0, s>>>(P->lv[l].Adiag, (__half*)P->lv[l].Adiag_s,
                                                             P->geom[l].count, P->fp.kappa);
      else
        k_store_diag<__nv_bfloat16><<<P->ew_blocks[l], 256, 0, s>>>(
            P->lv[l].Adiag, (__nv_bfloat16*)P->lv[l].Adiag_s, P->geom[l].count, P->fp.kappa);
      CKL("k_store_diag");
    }
  }
  k_count_fluid<<<P->red_blocks, kRedThreads, 0, s>>>(P->lv[0], P->partials, &P->ctl->counter[4],
                                                      &P->ctl->n_fluid);
  CKL("k_count_fluid");
  k_set_kappa<<<1, 1, 0, s>>>(P->ctl, (double)P->fp.kappa);
  CKL("k_set_kappa");
  if (int rc = tune_split(P, s)) return rc;
  if (int rc = tune_stream(P, s)) return rc;
  if (int rc = tune_resident(P, s)) return rc;
  if (declared == 1) {
    for (int l = 0; l < P->L; ++l) {
      k_verify_uniform<<<P->ew_blocks[l], 256, 0, s>>>(P->lv[l], P->offdiag[l], P->ctl);
      CKL("k_verify_uniform");
    }
  } else if (declared == 2) {
    for (int l = 0; l < P->L; ++l) {
      k_verify_whole<<<P->ew_blocks[l], 256, 0, s>>>(P->lv[l], P->ctl);
      CKL("k_verify_whole");
    }
  }
  // 4. the solve graph captured kernel arguments (shapes, s_l, kappa): rebuild
  //    it only when they changed
  uint64_t sig = 1469598103934665603ull;
  auto mix = [&](uint64_t v) { sig = (sig ^ v) * 1099511628211ull; };
  mix(P->fp.valid);
  mix(P->fp.sto);
  mix(P->fp.lc);
  mix(P->fp.res);
  mix(P->fp.res_lp);
  for (int l = 0; l < P->L; ++l) mix(P->fp.split[l]);
  for (int l = 0; l < P->L; ++l) mix(P->fp.step1[l]);
  for (int l = 0; l < P->L; ++l) mix(P->fp.col[l]);
  for (int l = 0; l < P->fp.lc; ++l) mix((uint64_t)P->fp.chunk[l] << 32 | (uint32_t)P->fp.blocks[l]);
  for (int l = 0; l < P->L; ++l) {
    uint32_t bits;
    std::memcpy(&bits, &P->fp.s[l], 4);
    mix(bits);
    mix(P->op_form[l]);
  }
  uint32_t kb;
  std::memcpy(&kb, &P->fp.kappa, 4);
  mix(kb);
  if (sig != P->graph_sig) {
    destroy_graph(P);
    P->graph_sig = sig;
  }
  P->prepared = true;
  return MG_OK;
}

extern "C" {

int mg_plan_split(mg_plan_t* P, int32_t set, uint32_t* bits, int32_t* streamed) {
  if (!P || !bits) return bad("null pointer");
  if (streamed) *streamed = P->fp.valid ? P->fp.lc : 0;
  if (set) {
    if (!P->fp.valid) return bad("the plan has no fused V-cycle");
    if (*bits >> P->fp.lc) return bad("split bits beyond the streamed levels");
    for (int l = 0; l < P->fp.lc; ++l) P->fp.split[l] = (*bits >> l) & 1u;
    destroy_graph(P);
    P->graph_sig = 0;
  }
  uint32_t b = 0;
  for (int l = 0; l < P->fp.lc; ++l)
    if (P->fp.split[l]) b |= 1u << l;
  *bits = b;
  return MG_OK;
}

int mg_plan_steps(mg_plan_t* P, int32_t set, uint32_t* bits) {
  if (!P || !bits) return bad("null pointer");
  if (set) {
    if (!P->fp.valid) return bad("the plan has no fused V-cycle");
    if (*bits >> (2 * P->fp.lc)) return bad("step bits beyond the streamed levels");
    if (*bits && (P->fp.sto || P->fp.dim != 3 || P->fp.storage != MG_STORE_F32))
      return bad("one plane per step needs the 3D label-uniform float32 form");
    for (int l = 0; l < P->fp.lc; ++l) P->fp.step1[l] = (unsigned char)((*bits >> (2 * l)) & 3u);
    destroy_graph(P);
    P->graph_sig = 0;
  }
  uint32_t b = 0;
  for (int l = 0; l < P->fp.lc; ++l) b |= (uint32_t)P->fp.step1[l] << (2 * l);
  *bits = b;
  return MG_OK;
}

int mg_plan_sweep_kernel(mg_plan_t* P, int32_t set, uint32_t* bits) {
  if (!P || !bits) return bad("null pointer");
  if (set) {
    if (!P->fp.valid) return bad("the plan has no fused V-cycle");
    if (*bits >> (2 * P->fp.lc)) return bad("kernel bits beyond the streamed levels");
    unsigned char old[kMaxLevels];
    for (int l = 0; l < P->fp.lc; ++l) old[l] = P->fp.col[l];
    for (int l = 0; l < P->fp.lc; ++l) {
      if (!set_col(P, l, (int)((*bits >> (2 * l)) & 3u))) {
        for (int k = 0; k < P->fp.lc; ++k) P->fp.col[k] = old[k];
        return bad("the column-register sweep cannot run that level");
      }
    }
    for (int l = 0; l < P->fp.lc; ++l) {
      if (P->fp.col[l]) P->fp.step1[l] = 0;
      level_grid(&P->fp, P->lv[l].g, l, P->fp.grid_extra[l]);
    }
    destroy_graph(P);
    P->graph_sig = 0;
  }
  uint32_t b = 0;
  for (int l = 0; l < P->fp.lc; ++l) b |= (uint32_t)P->fp.col[l] << (2 * l);
  *bits = b;
  return MG_OK;
}

int mg_plan_grid(mg_plan_t* P, int32_t set, uint32_t* bits) {
  if (!P || !bits) return bad("null pointer");
  if (set) {
    if (!P->fp.valid) return bad("the plan has no fused V-cycle");
    if (*bits >> (2 * P->fp.lc)) return bad("grid bits beyond the streamed levels");
    for (int l = 0; l < P->fp.lc; ++l) level_grid(&P->fp, P->lv[l].g, l, (int)((*bits >> (2 * l)) & 3u));
    destroy_graph(P);
    P->graph_sig = 0;
  }
  uint32_t b = 0;
  for (int l = 0; l < P->fp.lc; ++l) b |= (uint32_t)P->fp.grid_extra[l] << (2 * l);
  *bits = b;
  return MG_OK;
}

int mg_plan_resident(mg_plan_t* P, int32_t set, int32_t* on, int32_t* first_level) {
  if (!P || !on) return bad("null pointer");
  if (set) {
    if (*on && first_level && *first_level >= 0) {
      if (!P->fp.valid || !plan_resident(P, *first_level, *first_level, nullptr))
        return bad("the plan has no cluster-resident V-cycle from that level");
    }
    if (*on && !(P->fp.valid && P->fp.res_ok)) return bad("the plan has no cluster-resident V-cycle");
    P->fp.res = *on != 0;
    destroy_graph(P);
    P->graph_sig = 0;
  }
  *on = P->fp.valid && P->fp.res ? 1 : 0;
  if (first_level) *first_level = P->fp.valid && P->fp.res_ok ? P->fp.res_lp : -1;
  return MG_OK;
}

int mg_plan_operator_form(const mg_plan_t* P, int32_t level, int32_t* form) {
  if (!P || !form) return bad("null pointer");
  if (level < 0 || level >= P->L) return bad("level");
  *form = P->op_form[level] == 1 ? 1 : (P->fp.valid && P->fp.sto ? 2 : 0);
  return MG_OK;
}

int mg_smooth(mg_plan_t* P, int32_t level, int32_t phase, void* stream) {
  NEED_BOUND(P);
  if (level < 0 || level >= P->L || (phase != 0 && phase != 1)) return bad("level/phase");
  if (P->d.storage != MG_STORE_F32) return bad("per-kernel entry points need f32 storage");
  return launch_smooth(P, level, phase, S(stream));
}

int mg_restrict(mg_plan_t* P, int32_t level, void* stream) {
  NEED_BOUND(P);
  if (level < 0 || level >= P->L - 1) return bad("level");
  if (P->d.storage != MG_STORE_F32) return bad("per-kernel entry points need f32 storage");
  return launch_restrict(P, level, S(stream));
}

int mg_prolongate(mg_plan_t* P, int32_t level, void* stream) {
  NEED_BOUND(P);
  if (level < 0 || level >= P->L - 1) return bad("level");
  if (P->d.storage != MG_STORE_F32) return bad("per-kernel entry points need f32 storage");
  return launch_prolongate(P, level, S(stream));
}

int mg_v_cycle(mg_plan_t* P, void* stream) {
  NEED_BOUND(P);
  if (!P->prepared)
    if (int rc = mg_plan_prepare(P, stream)) return rc;
  return launch_vcycle(P, S(stream));
}

int mg_compute_Ap(mg_plan_t* P, void* stream) {
  NEED_BOUND(P);
  k_compute_Ap<<<P->ew_blocks[0], 256, 0, S(stream)>>>(P->lv[0], fptr(P, MG_FIELD_P), fptr(P, MG_FIELD_AP));
  CKL("k_compute_Ap");
  return MG_OK;
}

int mg_reduce(mg_plan_t* P, int32_t fa, int32_t fb, double* out, void* stream) {
  NEED_BOUND(P);
  auto ok = [](int f) { return f == MG_FIELD_B || f == MG_FIELD_X || f == MG_FIELD_P || f == MG_FIELD_AP ||
                               f == MG_FIELD_R || f == MG_FIELD_Z; };
  if (!ok(fa) || !ok(fb) || !out) return bad("reduce fields");
  if (P->d.storage != MG_STORE_F32 && (fa == MG_FIELD_Z || fb == MG_FIELD_Z)) return bad("z is not f32");
  const float* a = (const float*)(P->base + P->loc[fa][0][0].off);
  const float* b = (const float*)(P->base + P->loc[fb][0][0].off);
  k_dot<<<P->red_blocks, kRedThreads, 0, S(stream)>>>(P->lv[0], a, b, P->ctl, P->partials, 0);
  CKL("k_dot");
  CK(cudaMemcpyAsync(out, &P->ctl->scratch[0], sizeof(double), cudaMemcpyDeviceToHost, S(stream)));
  CK(cudaStreamSynchronize(S(stream)));
  return MG_OK;
}

int mg_pcg_solve_async(mg_plan_t* P, const mg_solve_params_t* prm, void* stream) {
  NEED_BOUND(P);
  if (!prm) return bad("params");
  if (prm->max_iters < -1) return bad("max_iters");
  if (!P->prepared)
    if (int rc = mg_plan_prepare(P, stream)) return rc;
  if (P->d.flags & MG_PLAN_DIRECT) return solve_direct(P, prm, S(stream));
  if (!P->exec || P->base_of_graph != P->base)
    if (int rc = build_graph(P)) return rc;
  // Parameters travel as kernel arguments (copied at launch, so back-to-back
  // asynchronous solves cannot race on a host staging buffer); the previous
  // solve's outputs and beta stay in place (mgpcg.py:44 persists beta).
  k_set_params<<<1, 1, 0, S(stream)>>>(P->ctl, *prm, P->d.refresh_every);
  CKL("k_set_params");
  CK(cudaGraphLaunch(P->exec, S(stream)));
  return MG_OK;
}

int mg_pcg_stats(mg_plan_t* P, mg_solve_stats_t* st, void* stream) {
  NEED_BOUND(P);
  if (!st) return bad("stats");
  CK(cudaMemcpyAsync(P->host_ctl, P->ctl, sizeof(Control), cudaMemcpyDeviceToHost, S(stream)));
  CK(cudaStreamSynchronize(S(stream)));
  st->status = P->host_ctl->status;
  st->iters = P->host_ctl->iter;
  st->rTr0 = P->host_ctl->rTr0;
  st->rTr = P->host_ctl->rTr;
  st->bTb = P->host_ctl->bTb;
  return MG_OK;
}

int mg_plan_launch_counts(mg_plan_t* P, int32_t* prologue, int32_t* body) {
  NEED_BOUND(P);
  if (!prologue || !body) return bad("null pointer");
  if (!P->prepared) return bad("plan not prepared");
  *prologue = count_pcg_part(P, true);
  *body = count_pcg_part(P, false);
  return MG_OK;
}

int mg_launch_stage(mg_plan_t* P, int32_t stage, int32_t level, void* stream) {
  NEED_BOUND(P);
  cudaStream_t s = S(stream);
  if (!P->prepared)
    if (int rc = mg_plan_prepare(P, stream)) return rc;
  const Level& L0 = P->lv[0];
  switch (stage) {
    case 0:
    case 1: {
      if (P->fp.valid) {
        if (level < 0 || level >= P->fp.lc) return bad("level is not a streamed level");
        return launch_level(P, level, stage == 0, s);
      }
      if (level < 0 || level >= P->L - 1) return bad("level");
      if (stage == 0) {
        for (int i = 0; i < P->d.pre_post; ++i) {
          if (int rc = launch_smooth(P, level, 0, s)) return rc;
          if (int rc = launch_smooth(P, level, 1, s)) return rc;
        }
        return launch_restrict(P, level, s);
      }
      if (int rc = launch_prolongate(P, level, s)) return rc;
      for (int i = 0; i < P->d.pre_post; ++i) {
        if (int rc = launch_smooth(P, level, 1, s)) return rc;
        if (int rc = launch_smooth(P, level, 0, s)) return rc;
      }
      return MG_OK;
    }
    case 2: {
      if (!P->fp.valid) return bad("the coarse stage belongs to the fused V-cycle");
      cudaError_t e = launch_coarse(P->fp, P->ctl, s);
      return e == cudaSuccess ? MG_OK : set_err("launch_coarse", e);
    }
    case 3:
      if (P->fp.valid && !P->fp.sto && x_by4(P))
        k_Ap_alpha_uniform4<<<P->red_blocks, kRedThreads, 0, s>>>(L0, fptr(P, MG_FIELD_P), fptr(P, MG_FIELD_AP),
                                                                  P->offdiag[0], P->ctl, P->partials, 1);
      else if (P->fp.valid && !P->fp.sto)
        k_Ap_alpha_uniform<<<P->red_blocks, kRedThreads, 0, s>>>(L0, fptr(P, MG_FIELD_P), fptr(P, MG_FIELD_AP),
                                                                 P->offdiag[0], P->ctl, P->partials, 1);
      else if (x_by4(P))
        k_Ap_alpha4<<<P->red_blocks, kRedThreads, 0, s>>>(L0, fptr(P, MG_FIELD_P), fptr(P, MG_FIELD_AP), P->ctl,
                                                          P->partials, 1);
      else
        k_Ap_alpha<<<P->red_blocks, kRedThreads, 0, s>>>(L0, fptr(P, MG_FIELD_P), fptr(P, MG_FIELD_AP), P->ctl,
                                                         P->partials, 1);
      CKL("k_Ap_alpha");
      return MG_OK;
    case 4:
      if (P->geom[0].count % 4 == 0)
        k_xr4<<<P->red_blocks, kRedThreads, 0, s>>>(L0, fptr(P, MG_FIELD_X), fptr(P, MG_FIELD_P),
                                                    fptr(P, MG_FIELD_AP), P->ctl, P->partials, P->cond, 0, 1,
                                                    xhptr(P));
      else
        k_xr<<<P->red_blocks, kRedThreads, 0, s>>>(L0, fptr(P, MG_FIELD_X), fptr(P, MG_FIELD_P),
                                                   fptr(P, MG_FIELD_AP), P->ctl, P->partials, P->cond, 0, 1,
                                                   xhptr(P));
      CKL("k_xr");
      return MG_OK;
    case 5:
      return launch_vcycle(P, s);
    case 6: {
      if (!P->fp.valid || !P->fp.res_ok) return bad("the plan has no cluster-resident V-cycle");
      cudaError_t e = launch_resident(P->fp, s);
      return e == cudaSuccess ? MG_OK : set_err("launch_resident", e);
    }
  }
  return bad("stage");
}

int mg_pressure_solve_async(mg_plan_t* P, const int32_t* ct, const float* v0, const float* v1, const float* v2,
                            const float* phi, float p0, float sA, float sB, int32_t ghost, float clamp,
                            const mg_solve_params_t* prm, void* stream) {
  NEED_BOUND(P);
  if (!prm) return bad("params");
  if (int rc = mg_pressure_setup_async(P, ct, v0, v1, v2, phi, p0, sA, sB, ghost, clamp, prm->warm_start, stream))
    return rc;
  return mg_pcg_solve_async(P, prm, stream);
}

int mg_pressure_setup_async(mg_plan_t* P, const int32_t* ct, const float* v0, const float* v1, const float* v2,
                            const float* phi, float p0, float sA, float sB, int32_t ghost, float clamp,
                            int32_t warm_start, void* stream) {
  NEED_BOUND(P);
  if (!ct) return bad("cell_type");
  cudaStream_t s = S(stream);
  // initialize() (mgpcg.py:63-77); a warm start keeps x
  if (warm_start) {
    const Loc& lx = P->loc[MG_FIELD_X][0][0];
    CK(cudaMemsetAsync(P->base, 0, lx.off, s));
    const int64_t after = lx.off + lx.bytes;
    CK(cudaMemsetAsync(P->base + after, 0, P->ws_bytes - after, s));
  } else {
    CK(cudaMemsetAsync(P->base, 0, P->ws_bytes, s));
  }
  if (int rc = mg_set_cell_type(P, ct, stream)) return rc;
  if (int rc = mg_build_pressure_b(P, v0, v1, v2, phi, p0, sA, sB, ghost, clamp, stream)) return rc;
  if (int rc = mg_build_pressure_A(P, 0, phi, sA, ghost, clamp, stream)) return rc;
  for (int l = 1; l < P->L; ++l) {
    if (int rc = mg_init_gridtype(P, l, stream)) return rc;
    if (int rc = mg_build_pressure_A(P, l, phi, sA, ghost, clamp, stream)) return rc;
  }
  float od[kMaxLevels];
  for (int l = 0; l < P->L; ++l) od[l] = sA;  // Ax = -scale_A between FLUID cells
  return mg_plan_prepare_declared(P, od, stream);
}

int mg_pcg_solve(mg_plan_t* P, const mg_solve_params_t* prm, mg_solve_stats_t* st, void* stream) {
  if (int rc = mg_pcg_solve_async(P, prm, stream)) return rc;
  return mg_pcg_stats(P, st, stream);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batched solves (mg_batch.cuh): tables of blocks, one launch per V-cycle
// stage and CG step for all instances, one CUDA graph for the whole loop.
// ---------------------------------------------------------------------------
struct mg_batch {
  std::vector<mg_plan*> plans;
  std::vector<uint64_t> sigs;   // each plan's launch signature when the tables were built
  int n = 0, storage = 0;
  bool refresh = false;
  // one sweep launch: instances of one kernel form at one level depth
  struct Group {
    int dim, one, pre, depth, blocks, ninst;
    int col;  // 0: the ring sweep; k: the column kernel with kColShapes[k]
    int64_t tab_off, args_off, maps_off;
  };
  std::vector<Group> groups;
  std::vector<unsigned char> blob;  // every table, laid out as in the workspace
  int64_t off_red = 0, off_ew = 0, off_cg = 0, off_coarse = 0, off_any = 0, ws_bytes = 0;
  int red_total = 0, ew_total = 0, maxlc = 0;
  size_t coarse_smem = 0;
  char* base = nullptr;
  cudaStream_t cap = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaGraphConditionalHandle cond = 0;
};

namespace {

int64_t put_blob(std::vector<unsigned char>& blob, const void* src, size_t bytes) {
  const int64_t off = align256((int64_t)blob.size());
  blob.resize(off + bytes);
  if (bytes) std::memcpy(blob.data() + off, src, bytes);
  return off;
}

// Planes a block of a batched sweep streams at least (measured on B200, the
// 96-instance batch: 58.1 / 55.9 / 55.3 / 57.9 ms for 8 / 16 / 32 / 64 in f32,
// 68.1 / 65.8 / 65.1 / 67.8 ms in f16).  A solve alone sizes
// its grid to fill the GPU by itself, which gives a small level chunks of 2
// planes that recompute 2 NS halo planes each (5x the work at NS = 4); in a
// batch the other instances fill the GPU, so chunks stay long.
#ifndef MG_BATCH_MIN_CHUNK
#define MG_BATCH_MIN_CHUNK 32
#endif

// The fused plan of an instance as the batch runs it: on every streamed level
// the kernel the instance's own plan chose (the column kernel with its tile,
// or the tiled ring kernel with two planes a step), chunks of at least
// MG_BATCH_MIN_CHUNK planes, the coarse block for the levels from lc (no
// cluster launch).  Every grid gives the same values.
FusedPlan batch_plan(const mg_plan* P) {
  FusedPlan F = P->fp;
  F.res = false;
  F.zr_mode = -1;
  int min_chunk = MG_BATCH_MIN_CHUNK;  // MGPCG_BATCH_CHUNK=<planes> overrides (even, >= 2)
  if (const char* ov = std::getenv("MGPCG_BATCH_CHUNK")) min_chunk = std::max(2, (int)std::strtol(ov, nullptr, 0) & ~1);
  for (int l = 0; l < F.lc; ++l) {
    F.step1[l] = 0;
    level_grid(&F, P->lv[l].g, l, F.grid_extra[l]);
    const int n0 = P->lv[l].g.n[0];
    if (F.col[l]) {  // each tile cut into k chunks of at least min_chunk planes
      const int k = std::max(1, n0 / std::max(min_chunk, 2));
      F.blocks[l] = F.tiles_x[l] * F.tiles_y[l] * k;
      F.chunk[l] = n0 / k;
    } else if (F.chunk[l] < min_chunk) {
      F.chunk[l] = std::min(n0, min_chunk);
      F.blocks[l] = F.tiles_x[l] * F.tiles_y[l] * ((n0 + F.chunk[l] - 1) / F.chunk[l]);
    }
  }
  return F;
}

// The column kernel's tensor maps of streamed level l of a plan (r, Adiag,
// the pre-smoothed z; PRE takes the Adiag map in the third place, unused).
template <typename ST, int TX, int TY, bool PRE>
bool col_maps_t(const Level* lv, int l, CUtensorMap* m) {
  using G = ColGeom<ST, 4, TX, TY>;
  const Level& f = lv[l];
  if (!tensor_map_3d(&m[0], f.r, l == 0 ? 4 : (int)sizeof(ST), f.g, G::RXB, G::RY) ||
      !tensor_map_3d(&m[1], f.Adiag_s, (int)sizeof(ST), f.g, G::RXB, G::RY))
    return false;
  if (PRE) {
    m[2] = m[1];
    return true;
  }
  return tensor_map_3d(&m[2], f.zt, (int)sizeof(ST), f.g, G::RXB, G::RY);
}

template <typename ST, bool PRE>
bool col_maps(int c, const Level* lv, int l, CUtensorMap* m) {
  switch (c) {
    case 1: return col_maps_t<ST, 32, 16, PRE>(lv, l, m);
    case 2: return col_maps_t<ST, 32, 32, PRE>(lv, l, m);
    case 3: return col_maps_t<ST, 64, 16, PRE>(lv, l, m);
  }
  return false;
}

template <typename ST, bool PRE>
int batch_sweep_args(mg_batch* B, const std::vector<FusedPlan>& fps, int depth, int dim, int one, int col) {
  std::vector<SweepArgs<ST>> args;
  std::vector<BatchBlock> tab;
  std::vector<CUtensorMap> maps;
  for (int i = 0; i < B->n; ++i) {
    const mg_plan* P = B->plans[i];
    const FusedPlan& F = fps[i];
    if (depth >= F.lc || P->d.dim != dim) continue;
    if (F.col[depth] != col) continue;
    const int is_one = !col && dim == 3 && F.chunk[depth] == 2;
    if (is_one != one) continue;
    const int k = (int)args.size();
    args.push_back(sweep_args<ST, PRE>(F, P->lv, depth, P->ctl));
    if (col) {
      CUtensorMap m[3];
      if (!col_maps<ST, PRE>(col, P->lv, depth, m)) return bad("batch: a column-kernel tensor map");
      maps.insert(maps.end(), m, m + 3);
    }
    for (int b = 0; b < F.blocks[depth]; ++b) tab.push_back({k, b, F.blocks[depth]});
  }
  if (args.empty()) return MG_OK;
  mg_batch::Group g;
  g.dim = dim;
  g.one = one;
  g.pre = PRE;
  g.depth = depth;
  g.col = col;
  g.blocks = (int)tab.size();
  g.ninst = (int)args.size();
  g.args_off = put_blob(B->blob, args.data(), args.size() * sizeof(SweepArgs<ST>));
  g.tab_off = put_blob(B->blob, tab.data(), tab.size() * sizeof(BatchBlock));
  g.maps_off = col ? put_blob(B->blob, maps.data(), maps.size() * sizeof(CUtensorMap)) : 0;
  B->groups.push_back(g);
  return MG_OK;
}

template <typename ST>
int batch_tables(mg_batch* B) {
  std::vector<FusedPlan> fps;
  for (auto* P : B->plans) fps.push_back(batch_plan(P));
  B->maxlc = 0;
  for (auto& F : fps) B->maxlc = std::max(B->maxlc, F.lc);
  // sweeps in V-cycle order: PRE by depth, (coarse), POST by depth upward
  for (int d = 0; d < B->maxlc; ++d)
    for (int dim = 3; dim >= 2; --dim)
      for (int col = 0; col < kColShapeCount; ++col)
        for (int one = 0; one <= (col ? 0 : 1); ++one)
          if (int rc = batch_sweep_args<ST, true>(B, fps, d, dim, one, col)) return rc;
  for (int d = B->maxlc - 1; d >= 0; --d)
    for (int dim = 3; dim >= 2; --dim)
      for (int col = 0; col < kColShapeCount; ++col)
        for (int one = 0; one <= (col ? 0 : 1); ++one)
          if (int rc = batch_sweep_args<ST, false>(B, fps, d, dim, one, col)) return rc;
  std::vector<CoarseArgs> coarse;
  B->coarse_smem = 0;
  for (int i = 0; i < B->n; ++i) {
    CoarseArgs a = fps[i].coarse;
    a.ctl = B->plans[i]->ctl;
    coarse.push_back(a);
    B->coarse_smem = std::max(B->coarse_smem, fps[i].coarse_smem);
  }
  B->off_coarse = put_blob(B->blob, coarse.data(), coarse.size() * sizeof(CoarseArgs));
  std::vector<BatchCg> cg;
  std::vector<BatchBlock> red, ew;
  for (int i = 0; i < B->n; ++i) {
    mg_plan* P = B->plans[i];
    BatchCg c;
    c.L0 = P->lv[0];
    c.b = fptr(P, MG_FIELD_B);
    c.x = fptr(P, MG_FIELD_X);
    c.p = fptr(P, MG_FIELD_P);
    c.Ap = fptr(P, MG_FIELD_AP);
    c.xh = xhptr(P);
    c.ctl = P->ctl;
    c.partials = P->partials;
    c.s0 = P->offdiag[0];
    c.by4 = x_by4(P) ? 1 : 0;
    c.c4 = P->geom[0].count % 4 == 0 ? 1 : 0;
    c.refresh = P->d.refresh_every > 0 ? 1 : 0;
    c.refresh_every = P->d.refresh_every;
    c.flex = c.refresh && P->d.storage != MG_STORE_F32 ? 1 : 0;
    cg.push_back(c);
    for (int b = 0; b < P->red_blocks; ++b) red.push_back({i, b, P->red_blocks});
    for (int b = 0; b < P->ew_blocks[0]; ++b) ew.push_back({i, b, P->ew_blocks[0]});
  }
  B->off_cg = put_blob(B->blob, cg.data(), cg.size() * sizeof(BatchCg));
  B->off_red = put_blob(B->blob, red.data(), red.size() * sizeof(BatchBlock));
  B->off_ew = put_blob(B->blob, ew.data(), ew.size() * sizeof(BatchBlock));
  B->red_total = (int)red.size();
  B->ew_total = (int)ew.size();
  const int zero = 0;
  B->off_any = put_blob(B->blob, &zero, sizeof(int));
  B->ws_bytes = align256((int64_t)B->blob.size());
  return MG_OK;
}

template <typename T>
const T* bptr(const mg_batch* B, int64_t off) { return (const T*)(B->base + off); }

template <typename ST, int TX, int TY, bool PRE, int MINB>
cudaError_t launch_bt_col_t(const mg_batch* B, const mg_batch::Group& g, cudaStream_t s) {
  using G = ColGeom<ST, 4, TX, TY>;
  auto kern = k_bt_colsweep<ST, 4, TX, TY, PRE, MINB>;
  const size_t smem = G::smem(PRE);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  return launch_k(kern, g.blocks, G::NT, smem, s, bptr<BatchBlock>(B, g.tab_off),
                  bptr<SweepArgs<ST>>(B, g.args_off), bptr<CUtensorMap>(B, g.maps_off));
}

template <typename ST, bool PRE>
cudaError_t launch_bt_group(const mg_batch* B, const mg_batch::Group& g, cudaStream_t s) {
  const BatchBlock* tab = bptr<BatchBlock>(B, g.tab_off);
  const SweepArgs<ST>* args = bptr<SweepArgs<ST>>(B, g.args_off);
  constexpr int NS = 4;
  switch (g.col) {  // the column kernel (shapes as launch_col_st)
    case 1: return launch_bt_col_t<ST, 32, 16, PRE, 2>(B, g, s);
    case 2: return launch_bt_col_t<ST, 32, 32, PRE, 1>(B, g, s);
    case 3: return launch_bt_col_t<ST, 64, 16, PRE, 1>(B, g, s);
  }
  if (g.dim == 3) {
    constexpr TileShape T = kTile3;
    if (g.one) {
      constexpr int K = 2 + 2 * NS;
      auto kern = k_bt_sweep<3, ST, NS, T.tx, T.ty, PRE, T.nt, K>;
      const size_t smem = sweep_smem(3, NS, {T.tx, T.ty, T.nt, K}, true, false);
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      return launch_k(kern, g.blocks, T.nt, smem, s, tab, args);
    }
    auto kern = k_bt_sweep<3, ST, NS, T.tx, T.ty, PRE, T.nt, T.k>;
    const size_t smem = sweep_smem(3, NS, T, false, false);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return launch_k(kern, g.blocks, T.nt, smem, s, tab, args);
  }
  constexpr TileShape T = kTile2;
  auto kern = k_bt_sweep<2, ST, NS, T.tx, T.ty, PRE, T.nt, T.k>;
  const size_t smem = sweep_smem(2, NS, T, false, false);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  return launch_k(kern, g.blocks, T.nt, smem, s, tab, args);
}

// One V-cycle of every instance (the stages in the order of the tables).
template <typename ST>
int launch_bt_vcycle(mg_batch* B, cudaStream_t s) {
  bool coarse_done = false;
  for (const auto& g : B->groups) {
    if (!g.pre && !coarse_done) {
      auto kern = k_bt_coarse<ST>;
      CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)B->coarse_smem));
      CK(launch_k(kern, B->n, kCoarseThreads, B->coarse_smem, s, bptr<CoarseArgs>(B, B->off_coarse)));
      coarse_done = true;
    }
    cudaError_t e = g.pre ? launch_bt_group<ST, true>(B, g, s) : launch_bt_group<ST, false>(B, g, s);
    if (e != cudaSuccess) return set_err("k_bt_sweep", e);
  }
  if (!coarse_done) {  // no streamed level in the batch
    auto kern = k_bt_coarse<ST>;
    CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)B->coarse_smem));
    CK(launch_k(kern, B->n, kCoarseThreads, B->coarse_smem, s, bptr<CoarseArgs>(B, B->off_coarse)));
  }
  return MG_OK;
}

// The batch's PCG pass: the prologue (mgpcg.py:157-173) or one loop iteration
// (mgpcg.py:175-209), for every instance.
template <typename ST>
int launch_bt_part(mg_batch* B, bool prologue, cudaStream_t s, int has_cond) {
  const BatchBlock* red = bptr<BatchBlock>(B, B->off_red);
  const BatchBlock* ew = bptr<BatchBlock>(B, B->off_ew);
  const BatchCg* cg = bptr<BatchCg>(B, B->off_cg);
  if (prologue) CK(launch_k(k_bt_begin, B->red_total, kRedThreads, 0, s, red, cg));
  if (int rc = launch_bt_vcycle<ST>(B, s)) return rc;
  if (prologue) {
    CK(launch_k(k_bt_update_p<ST>, B->ew_total, 256, 0, s, ew, cg));
    CK(launch_k(k_bt_zr<ST>, B->red_total, kRedThreads, 0, s, red, cg, 0));
  } else {
    CK(launch_k(k_bt_zr<ST>, B->red_total, kRedThreads, 0, s, red, cg, 1));
    CK(launch_k(k_bt_update_p<ST>, B->ew_total, 256, 0, s, ew, cg));
  }
  CK(launch_k(k_bt_Ap, B->red_total, kRedThreads, 0, s, red, cg));
  CK(launch_k(k_bt_xr, B->red_total, kRedThreads, 0, s, red, cg));
  if (B->refresh) CK(launch_k(k_bt_refresh, B->red_total, kRedThreads, 0, s, red, cg));
  int* any = (int*)(B->base + B->off_any);
  CK(launch_k(k_bt_cond, 1, 256, 0, s, cg, B->n, B->cond, has_cond, any));
  return MG_OK;
}

template <typename ST>
int build_batch_graph(mg_batch* B) {
  if (B->exec) cudaGraphExecDestroy(B->exec);
  if (B->graph) cudaGraphDestroy(B->graph);
  B->exec = nullptr;
  B->graph = nullptr;
  if (!B->cap) CK(cudaStreamCreateWithFlags(&B->cap, cudaStreamNonBlocking));
  CK(cudaGraphCreate(&B->graph, 0));
  CK(cudaGraphConditionalHandleCreate(&B->cond, B->graph, 0, cudaGraphCondAssignDefault));
  CK(cudaStreamBeginCaptureToGraph(B->cap, B->graph, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  int rc = launch_bt_part<ST>(B, true, B->cap, 1);
  if (rc) {
    cudaGraph_t g;
    cudaStreamEndCapture(B->cap, &g);
    return rc;
  }
  cudaStreamCaptureStatus st;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  cudaGraph_t capg;
  CK(cudaStreamGetCaptureInfo(B->cap, &st, nullptr, &capg, &deps, &ndeps));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = B->cond;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cnode;
  CK(cudaGraphAddNode(&cnode, capg, deps, ndeps, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  CK(cudaStreamUpdateCaptureDependencies(B->cap, &cnode, 1, cudaStreamSetCaptureDependencies));
  cudaGraph_t out;
  CK(cudaStreamEndCapture(B->cap, &out));
  CK(cudaStreamBeginCaptureToGraph(B->cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  rc = launch_bt_part<ST>(B, false, B->cap, 1);
  {
    cudaGraph_t g2;
    cudaError_t e = cudaStreamEndCapture(B->cap, &g2);
    if (rc) return rc;
    if (e != cudaSuccess) return set_err("cudaStreamEndCapture(batch body)", e);
  }
  CK(cudaGraphInstantiate(&B->exec, B->graph, 0));
  return MG_OK;
}

int build_batch_graph_any(mg_batch* B) {
  switch (B->storage) {
    case MG_STORE_F16: return build_batch_graph<__half>(B);
    case MG_STORE_BF16: return build_batch_graph<__nv_bfloat16>(B);
    default: return build_batch_graph<float>(B);
  }
}

}  // namespace

extern "C" {

int mg_batch_create(mg_plan_t* const* plans, int32_t n, mg_batch_t** out) {
  if (!plans || !out || n < 1) return bad("mg_batch_create: plans / count / out");
  *out = nullptr;
  mg_batch* B = new (std::nothrow) mg_batch();
  if (!B) return bad("mg_batch_create: out of host memory");
  B->n = n;
  for (int i = 0; i < n; ++i) {
    mg_plan* P = plans[i];
    if (!P || !P->base) {
      delete B;
      return bad("mg_batch_create: every plan must be bound");
    }
    if (!P->prepared || !P->fp.valid || P->fp.sto) {
      delete B;
      snprintf(g_err, sizeof(g_err),
               "bad argument: mg_batch_create: plan %d (%dD %dx%dx%d, %d levels) is not prepared in the "
               "label-uniform fused form (prepared %d, fused %d)", i, P->d.dim, P->geom[0].n[0], P->geom[0].n[1],
               P->geom[0].n[2], P->L, (int)P->prepared, (int)P->fp.valid);
      return MG_E_BADARG;
    }
    if (P->d.pre_post != 2) {
      delete B;
      return bad("mg_batch_create: batched sweeps run pre_and_post_smoothing = 2");
    }
    if (i > 0 && (P->d.storage != plans[0]->d.storage || P->device != plans[0]->device)) {
      delete B;
      return bad("mg_batch_create: every plan must have the same storage type and device");
    }
    B->plans.push_back(P);
    B->sigs.push_back(P->graph_sig);
  }
  B->storage = plans[0]->d.storage;
  B->refresh = plans[0]->d.refresh_every > 0;
  for (auto* P : B->plans) B->refresh = B->refresh || P->d.refresh_every > 0;
  int rc = MG_OK;
  switch (B->storage) {
    case MG_STORE_F16: rc = batch_tables<__half>(B); break;
    case MG_STORE_BF16: rc = batch_tables<__nv_bfloat16>(B); break;
    default: rc = batch_tables<float>(B);
  }
  if (rc != MG_OK) {
    delete B;
    return rc;
  }
  *out = B;
  return MG_OK;
}

void mg_batch_destroy(mg_batch_t* B) {
  if (!B) return;
  if (B->exec) cudaGraphExecDestroy(B->exec);
  if (B->graph) cudaGraphDestroy(B->graph);
  if (B->cap) cudaStreamDestroy(B->cap);
  delete B;
}

int64_t mg_batch_workspace_bytes(const mg_batch_t* B) { return B ? B->ws_bytes : 0; }

int mg_batch_bind(mg_batch_t* B, void* workspace, void* stream) {
  if (!B || !workspace) return bad("mg_batch_bind: null pointer");
  if ((uintptr_t)workspace & 255) return bad("mg_batch_bind: workspace not 256-byte aligned");
  B->base = (char*)workspace;
  CK(cudaMemcpyAsync(B->base, B->blob.data(), B->blob.size(), cudaMemcpyHostToDevice, S(stream)));
  CK(cudaStreamSynchronize(S(stream)));
  return build_batch_graph_any(B);
}

int mg_batch_solve_async(mg_batch_t* B, const mg_solve_params_t* prm, void* stream) {
  if (!B || !prm) return bad("mg_batch_solve_async: null pointer");
  if (!B->base || !B->exec) return bad("mg_batch_solve_async: batch not bound");
  if (prm->max_iters < -1) return bad("max_iters");
  for (int i = 0; i < B->n; ++i)
    if (B->plans[i]->graph_sig != B->sigs[i] || !B->plans[i]->prepared)
      return bad("mg_batch_solve_async: an instance's plan changed shape since mg_batch_create");
  const BatchCg* cg = bptr<BatchCg>(B, B->off_cg);
  k_bt_params<<<(B->n + 127) / 128, 128, 0, S(stream)>>>(cg, B->n, *prm);
  CKL("k_bt_params");
  CK(cudaGraphLaunch(B->exec, S(stream)));
  return MG_OK;
}

int mg_batch_launch_counts(const mg_batch_t* B, int32_t* prologue, int32_t* body) {
  if (!B || !prologue || !body) return bad("null pointer");
  const int v = (int)B->groups.size() + 1;  // sweep groups + the coarse launch
  const int cg = 4 + (B->refresh ? 1 : 0) + 1;  // zr, update_p, Ap, xr, [refresh], cond
  *prologue = 1 + v + cg;
  *body = v + cg;
  return MG_OK;
}

}  // extern "C"
