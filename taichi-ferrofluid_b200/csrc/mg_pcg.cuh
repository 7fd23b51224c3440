// Device-resident PCG loop kernels (mgpcg.py:150-238).
//
// The reference reads every reduction back to the host (three syncs per
// iteration).  Here each reduction ends in a last-block epilogue that computes
// the scalar step of the loop on the device in FP64 (alpha, beta, the
// convergence test, the iteration counter) and, at the end of an iteration,
// sets the condition of the CUDA graph while node that repeats the body.
#pragma once
#include "mg_common.cuh"

namespace mg {

// Copies one solve's parameters into the control block.
__global__ void k_set_params(Control* ctl, mg_solve_params_t prm, int refresh_every) {
  ctl->rel_tol = prm.rel_tol;
  ctl->abs_tol = prm.abs_tol;
  ctl->eps = prm.eps;
  ctl->max_iters = prm.max_iters;
  ctl->warm_start = prm.warm_start;
  ctl->refresh_every = refresh_every;
}

// r = b (reference), or r = b - A x (warm start); then r.r over FLUID cells.
// Epilogue: rTr0, tol = max(abs_tol, rTr0 * rel_tol) (mgpcg.py:157-164).
__global__ void __launch_bounds__(kRedThreads) k_pcg_begin(Level L, const float* __restrict__ b,
                                                           const float* __restrict__ x, Control* ctl,
                                                           double* partials) {
  __shared__ double sh[32];
  float* r = (float*)L.r;
  const int warm = ctl->warm_start;
  double acc = 0.0, accb = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < L.g.count;
       i += (long long)gridDim.x * blockDim.x) {
    float ri = b[i];
    if (L.type[i] == FLUID) accb += (double)ri * (double)ri;
    if (warm && L.type[i] == FLUID) {
      int c[3];
      L.g.coords(i, c);
      float Ax_ = __fmul_rn(L.Adiag[i], x[i]);
      Ax_ = __fadd_rn(Ax_, nbr_sum_f32(L, x, i, c));
      ri = __fsub_rn(ri, Ax_);
    }
    r[i] = ri;
    if (L.type[i] == FLUID) acc += (double)ri * (double)ri;
  }
  double tot, totb;
  // b.b first (its own counter), then r.r; both blocks orders are fixed
  bool lastb = last_block_total<kRedThreads>(accb, partials + kMaxPartials / 2, &ctl->counter[6], sh, &totb);
  if (lastb && threadIdx.x == 0) ctl->bTb = totb;
  if (last_block_total<kRedThreads>(acc, partials, &ctl->counter[0], sh, &tot) && threadIdx.x == 0) {
    __threadfence();
    const double bb = ((volatile Control*)ctl)->bTb;
    ctl->rTr0 = tot;
    ctl->rTr = tot;
    ctl->tol = fmax(ctl->abs_tol, bb * ctl->rel_tol);
    ctl->iter = 0;
    ctl->status = MG_SOLVE_MAX_ITERS;
    ctl->run = 1;
    ctl->since_refresh = 0;
    if (warm) ctl->beta = 0.0f;  // p is rebuilt from z only
  }
}

// update_p (mgpcg.py:234-238): p = z + beta p on FLUID cells.
__global__ void k_update_p(Level L, float* __restrict__ p, const Control* ctl) {
  const float beta = ctl->beta;
  const float* z = (const float*)L.z;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < L.g.count;
       i += (long long)gridDim.x * blockDim.x)
    if (L.type[i] == FLUID) p[i] = __fadd_rn(z[i], __fmul_rn(beta, p[i]));
}

// reduce(z, r) (mgpcg.py:171, :201) with the scalar epilogue.
//  mode 0 (before the loop): old_zTr = z.r; the loop runs iff max_iters != 0.
//  mode 1 (end of an iteration): beta = new / (old + eps); old = new; iter++;
//          stop at max_iters (mgpcg.py:176, :200-209).
__global__ void __launch_bounds__(kRedThreads) k_zr(Level L, Control* ctl, double* partials, int mode) {
  __shared__ double sh[32];
  const float* z = (const float*)L.z;
  const float* r = (const float*)L.r;
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < L.g.count;
       i += (long long)gridDim.x * blockDim.x)
    if (L.type[i] == FLUID) acc += (double)z[i] * (double)r[i];
  double tot;
  if (last_block_total<kRedThreads>(acc, partials, &ctl->counter[1], sh, &tot) && threadIdx.x == 0) {
    if (mode == 0) {
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

// compute_Ap (mgpcg.py:218-224) + reduce(p, Ap) + alpha = zTr / (pAp + eps).
__global__ void __launch_bounds__(kRedThreads) k_Ap_alpha(Level L, const float* __restrict__ p,
                                                          float* __restrict__ Ap, Control* ctl,
                                                          double* partials) {
  if (!ctl->run) return;
  __shared__ double sh[32];
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < L.g.count;
       i += (long long)gridDim.x * blockDim.x) {
    if (L.type[i] != FLUID) continue;
    int c[3];
    L.g.coords(i, c);
    float v = __fmul_rn(L.Adiag[i], p[i]);
    v = __fadd_rn(v, nbr_sum_f32(L, p, i, c));
    Ap[i] = v;
    acc += (double)p[i] * (double)v;
  }
  double tot;
  if (last_block_total<kRedThreads>(acc, partials, &ctl->counter[2], sh, &tot) && threadIdx.x == 0) {
    ctl->pAp = tot;
    ctl->alpha = (float)(ctl->old_zTr / (tot + ctl->eps));
  }
}

// update_xr (mgpcg.py:226-232) + reduce(r, r) + the convergence test
// (mgpcg.py:188-195).  Sets the while-node condition to ctl->run.
__global__ void __launch_bounds__(kRedThreads) k_xr(Level L, float* __restrict__ x,
                                                    const float* __restrict__ p,
                                                    const float* __restrict__ Ap, Control* ctl,
                                                    double* partials, cudaGraphConditionalHandle cond,
                                                    int has_cond) {
  __shared__ double sh[32];
  if (!ctl->run) {
    if (has_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(cond, 0);
    return;
  }
  const float alpha = ctl->alpha;
  float* r = (float*)L.r;
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < L.g.count;
       i += (long long)gridDim.x * blockDim.x) {
    if (L.type[i] != FLUID) continue;
    x[i] = __fadd_rn(x[i], __fmul_rn(alpha, p[i]));
    float ri = __fsub_rn(r[i], __fmul_rn(alpha, Ap[i]));
    r[i] = ri;
    acc += (double)ri * (double)ri;
  }
  double tot;
  if (last_block_total<kRedThreads>(acc, partials, &ctl->counter[3], sh, &tot) && threadIdx.x == 0) {
    ctl->rTr = tot;
    if (!isfinite(tot)) {
      ctl->status = MG_SOLVE_NONFINITE;
      ctl->run = 0;
    } else if (tot < ctl->tol) {
      ctl->status = MG_SOLVE_CONVERGED;
      ctl->run = 0;
    }
    if (has_cond) cudaGraphSetConditional(cond, ctl->run ? 1u : 0u);
  }
}

// Plain masked dot of two level-0 f32 fields into ctl->scratch[slot]
// (reduce(p, q), mgpcg.py:211-216).
__global__ void __launch_bounds__(kRedThreads) k_dot(Level L, const float* __restrict__ a,
                                                     const float* __restrict__ b, Control* ctl,
                                                     double* partials, int slot) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < L.g.count;
       i += (long long)gridDim.x * blockDim.x)
    if (L.type[i] == FLUID) acc += (double)a[i] * (double)b[i];
  double tot;
  if (last_block_total<kRedThreads>(acc, partials, &ctl->counter[4], sh, &tot) && threadIdx.x == 0)
    ctl->scratch[slot] = tot;
}

// compute_Ap alone (mgpcg.py:218-224).
__global__ void k_compute_Ap(Level L, const float* __restrict__ p, float* __restrict__ Ap) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < L.g.count;
       i += (long long)gridDim.x * blockDim.x) {
    if (L.type[i] != FLUID) continue;
    int c[3];
    L.g.coords(i, c);
    float v = __fmul_rn(L.Adiag[i], p[i]);
    v = __fadd_rn(v, nbr_sum_f32(L, p, i, c));
    Ap[i] = v;
  }
}

}  // namespace mg
