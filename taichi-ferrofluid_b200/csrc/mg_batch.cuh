// Batched solves: many independent label-uniform pressure solves (uneven 2D
// and 3D grids) advanced together, ONE launch per V-cycle stage and per CG
// step for the whole batch, each launch driven by a table of blocks.
//
// Table entry = (instance, the block's index among that instance's blocks,
// their count).  A block runs exactly the code and the decomposition its
// instance's own launch would run (the same sweep tiles and chunks of planes,
// the same reduction blocks), so the arithmetic of each solve is that of the
// solve alone; only which blocks share a launch changes.  Reductions end in a
// per-instance last block (last_block_total_at over the instance's own
// partials and counter), so every instance takes its own alpha, beta and
// convergence test on the device; an instance that has finished (Control::done)
// makes its blocks return at once.  The loop of the whole batch is one CUDA
// graph while-node whose condition k_bt_cond sets: any instance still running.
#pragma once
#include "mg_sweep.cuh"
#include "mg_colsweep.cuh"
#include "mg_coarse.cuh"
#include "mg_pcg.cuh"

namespace mg {

struct BatchBlock {
  int inst;  // index into the launch's argument table
  int bid;   // block index within that instance's launch
  int nb;    // blocks of that instance's launch
};

// Per-instance arguments of the CG steps.
struct BatchCg {
  Level L0;
  float* b;
  float* x;
  float* p;
  float* Ap;
  double* xh;       // mixed form: FP64 x (else null)
  Control* ctl;
  double* partials;
  float s0;         // coupling magnitude of level 0 (label-uniform)
  int by4;          // the matvec on 4-cell groups (fastest extent a multiple of 4)
  int c4;           // the vector steps on 4-cell groups (cell count a multiple of 4)
  int flex;         // mixed form: flexible beta (z.Ap), 16-bit z
  int refresh;      // true-residual refresh
  int refresh_every;
};

// Parameters of one solve into every instance (k_set_params for each).
__global__ void k_bt_params(const BatchCg* inst, int n, mg_solve_params_t prm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Control* ctl = inst[i].ctl;
  ctl->rel_tol = prm.rel_tol;
  ctl->abs_tol = prm.abs_tol;
  ctl->eps = prm.eps;
  ctl->max_iters = prm.max_iters;
  ctl->warm_start = prm.warm_start;
  ctl->refresh_every = inst[i].refresh_every;
  ctl->done = 0;
}

__global__ void __launch_bounds__(kRedThreads) k_bt_begin(const BatchBlock* tab, const BatchCg* inst) {
  pdl_enter();
  const BatchBlock e = tab[blockIdx.x];
  const BatchCg& I = inst[e.inst];
  pcg_begin_body(e.bid, e.nb, I.L0, I.b, I.x, I.ctl, I.partials, I.xh);
}

// One sweep stage of the V-cycle over every instance's level in the table.
template <int DIM, typename ST, int NS, int TX, int TY, bool PRE, int NT, int K>
__global__ void __launch_bounds__(NT) k_bt_sweep(const BatchBlock* tab, const SweepArgs<ST>* args) {
  pdl_enter();
  const BatchBlock e = tab[blockIdx.x];
  const SweepArgs<ST>& A = args[e.inst];
  if (A.ctl->done) return;
  sweep_body<DIM, ST, NS, TX, TY, PRE, NT, K, false>(A, e.bid, e.nb);
}

// One column-kernel sweep stage (k_colsweep) over every instance in the
// table whose level runs it with this tile: each instance's three tensor maps
// (r, Adiag, the pre-smoothed z) sit at maps[3 * inst] in global memory,
// written by the host before the launch.
template <typename ST, int NS, int TX, int TY, bool PRE, int MINB>
__global__ void __launch_bounds__(ColGeom<ST, NS, TX, TY>::NT, MINB)
    k_bt_colsweep(const BatchBlock* tab, const SweepArgs<ST>* args, const CUtensorMap* maps) {
  pdl_enter();
  const BatchBlock e = tab[blockIdx.x];
  const SweepArgs<ST>& A = args[e.inst];
  if (A.ctl->done) return;
  const CUtensorMap* m = maps + 3 * e.inst;
  if (threadIdx.x == 0)  // the maps are read through the tensor-map proxy
    for (int k = 0; k < 3; ++k)
      asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(m + k) : "memory");
  colsweep_body<ST, NS, TX, TY, PRE>(A, const_cast<Control*>(A.ctl), m, m + 1, m + 2, e.bid, e.nb);
}

// The coarse block of every instance: block i solves instance i's coarse levels.
template <typename ST>
__global__ void __launch_bounds__(kCoarseThreads) k_bt_coarse(const CoarseArgs* args) {
  pdl_enter();
  extern __shared__ __align__(16) unsigned char smem[];
  const CoarseArgs& A = args[blockIdx.x];
  if (A.ctl->done) return;
  coarse_vcycle<ST, false>(A, smem);
}

template <typename ST>
__global__ void __launch_bounds__(kRedThreads) k_bt_zr(const BatchBlock* tab, const BatchCg* inst, int mode) {
  pdl_enter();
  const BatchBlock e = tab[blockIdx.x];
  const BatchCg& I = inst[e.inst];
  if (I.ctl->done) return;
  if (sizeof(ST) == 4 && I.c4) zr4_body(e.bid, e.nb, I.L0, I.ctl, I.partials, mode);
  else zr_body<ST>(e.bid, e.nb, I.L0, I.ctl, I.partials, mode, I.flex ? I.Ap : nullptr);
}

template <typename ST>
__global__ void k_bt_update_p(const BatchBlock* tab, const BatchCg* inst) {
  pdl_enter();
  const BatchBlock e = tab[blockIdx.x];
  const BatchCg& I = inst[e.inst];
  if (I.ctl->done) return;
  if (sizeof(ST) == 4 && I.c4) update_p4_body(e.bid, e.nb, I.L0, I.p, I.ctl);
  else update_p_body<ST>(e.bid, e.nb, I.L0, I.p, I.ctl);
}

__global__ void __launch_bounds__(kRedThreads) k_bt_Ap(const BatchBlock* tab, const BatchCg* inst) {
  pdl_enter();
  const BatchBlock e = tab[blockIdx.x];
  const BatchCg& I = inst[e.inst];
  if (I.ctl->done) return;
  if (I.by4) Ap_alpha_uniform4_body(e.bid, e.nb, I.L0, I.p, I.Ap, I.s0, I.ctl, I.partials, 0);
  else Ap_alpha_uniform_body(e.bid, e.nb, I.L0, I.p, I.Ap, I.s0, I.ctl, I.partials, 0);
}

__global__ void __launch_bounds__(kRedThreads) k_bt_xr(const BatchBlock* tab, const BatchCg* inst) {
  pdl_enter();
  const BatchBlock e = tab[blockIdx.x];
  const BatchCg& I = inst[e.inst];
  if (I.ctl->done) return;
  if (I.c4) xr4_body(e.bid, e.nb, I.L0, I.x, I.p, I.Ap, I.ctl, I.partials, 0, 0, 0, I.xh);
  else xr_body(e.bid, e.nb, I.L0, I.x, I.p, I.Ap, I.ctl, I.partials, 0, 0, 0, I.xh);
}

__global__ void __launch_bounds__(kRedThreads) k_bt_refresh(const BatchBlock* tab, const BatchCg* inst) {
  pdl_enter();
  const BatchBlock e = tab[blockIdx.x];
  const BatchCg& I = inst[e.inst];
  if (I.ctl->done || !I.refresh) return;
  refresh_body(e.bid, e.nb, I.L0, I.b, I.x, I.ctl, I.partials, 0, 0, I.xh);
}

// End of a pass: an instance whose loop has stopped is done; the batch's
// loop runs while any instance is not.
__global__ void k_bt_cond(const BatchCg* inst, int n, cudaGraphConditionalHandle cond, int has_cond, int* any_out) {
  pdl_enter();
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    Control* ctl = inst[i].ctl;
    if (!ctl->done && !ctl->run) ctl->done = 1;
    if (!ctl->done) any = 1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    *any_out = any;
    if (has_cond) cudaGraphSetConditional(cond, any ? 1u : 0u);
  }
}

}  // namespace mg
