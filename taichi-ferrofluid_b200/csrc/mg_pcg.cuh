// Device-resident PCG loop kernels (mgpcg.py:150-238).
//
// The reference reads every reduction back to the host (three syncs per
// iteration).  Here each reduction ends in a last-block epilogue that computes
// the scalar step of the loop on the device in FP64 (alpha, beta, the
// convergence test, the iteration counter) and, at the end of an iteration,
// sets the condition of the CUDA graph while node that repeats the body.
#pragma once
#include "mg_common.cuh"
#include "mg_kernels.cuh"

namespace mg {

// Coefficient scale after mg_plan_prepare; sigma = 1 until a solve sets it.
__global__ void k_set_kappa(Control* ctl, double kappa) {
  ctl->kappa = kappa;
  ctl->scale_r = 1.0;
  ctl->scale_z = kappa;
  ctl->bad_operator = 0;
}

// k_verify_uniform for a compile-time dim (its per-axis arrays and the level's
// extents indexed by constants, so nothing is kept in local memory).
template <int DIM>
__device__ __forceinline__ void k_verify_uniform_dim(Level L, float s, Control* ctl) {
  int bad = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < L.g.count;
       i += (long long)gridDim.x * blockDim.x) {
    int c[3];
    L.g.coords(i, c);
    const bool fl = L.type[i] == FLUID;
    if (fl && L.Adiag[i] == 0.0f) bad |= 2;
    else if (!fl && L.Adiag[i] != 0.0f) bad |= 1;
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
      const bool coupled = fl && (c[k] + 1 < L.g.n[k]) && L.type[i + L.g.stride(k)] == FLUID;
      if (L.Ax[k][i] != (coupled ? -s : 0.0f)) bad |= 1;
    }
  }
  bad = __reduce_or_sync(0xffffffffu, bad);
  if (bad && (threadIdx.x & 31) == 0) atomicOr(&ctl->bad_operator, bad);
}

// Checks a declared label-uniform level: Adiag != 0 exactly on FLUID cells
// and Ax = -s between two FLUID cells, 0 elsewhere.  Flags a mismatch (bit
// 0), or a FLUID cell with a zero diagonal (bit 1: the reference's smoothing
// divides by zero there, a non-finite solve).
__global__ void k_verify_uniform(Level L, float s, Control* ctl) {
  if (L.g.dim == 3) k_verify_uniform_dim<3>(L, s, ctl);
  else k_verify_uniform_dim<2>(L, s, ctl);
}

// Checks a declared whole-domain level: every cell FLUID (bit 0) with
// Adiag != 0 (bit 1, as k_verify_uniform).
__global__ void k_verify_whole(Level L, Control* ctl) {
  int bad = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < L.g.count;
       i += (long long)gridDim.x * blockDim.x) {
    if (L.type[i] != FLUID) bad |= 1;
    if (L.Adiag[i] == 0.0f) bad |= 2;
  }
  bad = __reduce_or_sync(0xffffffffu, bad);
  if (bad && (threadIdx.x & 31) == 0) atomicOr(&ctl->bad_operator, bad);
}

// Copies one solve's parameters into the control block.
__global__ void k_set_params(Control* ctl, mg_solve_params_t prm, int refresh_every) {
  ctl->rel_tol = prm.rel_tol;
  ctl->abs_tol = prm.abs_tol;
  ctl->eps = prm.eps;
  ctl->max_iters = prm.max_iters;
  ctl->warm_start = prm.warm_start;
  ctl->refresh_every = refresh_every;
}

__device__ void set_scales(Control* ctl, double rTr);

// r = b (reference), or r = b - A x (warm start); then r.r over FLUID cells.
// Epilogue: rTr0, tol = max(abs_tol, rTr0 * rel_tol) (mgpcg.py:157-164).
__device__ __forceinline__ void pcg_begin_body(int bid_, int nb_, Level L, const float* __restrict__ b,
                                                           float* __restrict__ x, Control* ctl,
                                                           double* partials, double* __restrict__ xh) {

  __shared__ double sh[32];
  float* r = (float*)L.r;
  const int warm = ctl->warm_start;
  double acc = 0.0, accb = 0.0;
  for (long long i = (long long)bid_ * blockDim.x + threadIdx.x; i < L.g.count;
       i += (long long)nb_ * blockDim.x) {
    float ri = b[i];
    if (L.type[i] == FLUID) accb += (double)ri * (double)ri;
    if (warm && L.type[i] == FLUID) {
      int c[3];
      L.g.coords(i, c);
      float Ax_ = __fmul_rn(L.Adiag[i], x[i]);
      Ax_ = __fadd_rn(Ax_, nbr_sum_f32(L, x, i, c));
      ri = __fsub_rn(ri, Ax_);
    } else if (warm) {
      // a cell that is no longer FLUID holds no pressure (the reference's x
      // is 0 there); its stale value never enters A x (its couplings are 0)
      x[i] = 0.0f;
    }
    r[i] = ri;
    if (L.type[i] == FLUID) acc += (double)ri * (double)ri;
    // mixed form: the FP64 copy of x that the loop accumulates into
    if (xh) xh[i] = warm && L.type[i] == FLUID ? (double)x[i] : 0.0;
  }
  double tot, totb;
  // b.b first (its own counter), then r.r; both blocks orders are fixed
  bool lastb = last_block_total_at<kRedThreads>(accb, partials + kMaxPartials / 2, &ctl->counter[6], sh, &totb, bid_, nb_);
  if (lastb && threadIdx.x == 0) ctl->bTb = totb;
  if (last_block_total_at<kRedThreads>(acc, partials, &ctl->counter[0], sh, &tot, bid_, nb_) && threadIdx.x == 0) {
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
    if (ctl->bad_operator) {     // the declared operator form did not hold,
      // or a FLUID cell has a zero diagonal (the reference divides by it)
      ctl->status = (ctl->bad_operator & 1) ? MG_SOLVE_BAD_OPERATOR : MG_SOLVE_NONFINITE;
      ctl->run = 0;
    }
    ctl->wait_timeout = 0;
    set_scales(ctl, tot);
  }
}

__global__ void __launch_bounds__(kRedThreads) k_pcg_begin(Level L, const float* __restrict__ b,
                                                           float* __restrict__ x, Control* ctl,
                                                           double* partials, double* __restrict__ xh) {
  pdl_enter();
  pcg_begin_body(blockIdx.x, gridDim.x, L, b, x, ctl, partials, xh);
}

// z of level 0 as float32: 16-bit grids hold z~ = z / scale_z (a power of two).
template <typename ST>
__device__ __forceinline__ float z_true(const ST* z, long long i, float scale_z) {
  if constexpr (sizeof(ST) == 4) return z[i];
  else return __fmul_rn(scale_z, to_f<ST>(z[i]));
}

// The per-V-cycle scale of 16-bit grids: sigma = 2^-round(log2(rms(r))), from
// r.r over the FLUID cells, and scale_z = kappa / sigma.
__device__ void set_scales(Control* ctl, double rTr) {
  double sigma = 1.0;
  if (ctl->n_fluid > 0.0 && rTr > 0.0 && isfinite(rTr)) {
    const double rms = sqrt(rTr / ctl->n_fluid);
    sigma = exp2(-rint(log2(rms)));
  }
  ctl->scale_r = sigma;
  ctl->scale_z = ctl->kappa / sigma;
}

// update_p (mgpcg.py:234-238): p = z + beta p on FLUID cells.
template <typename ST>
__device__ __forceinline__ void update_p_body(int bid_, int nb_, Level L, float* __restrict__ p, const Control* ctl) {

  const float beta = ctl->beta;
  const float sz = (float)ctl->scale_z;
  const ST* z = (const ST*)L.z;
  for (long long i = (long long)bid_ * blockDim.x + threadIdx.x; i < L.g.count;
       i += (long long)nb_ * blockDim.x)
    if (L.type[i] == FLUID) p[i] = __fadd_rn(z_true<ST>(z, i, sz), __fmul_rn(beta, p[i]));
}

template <typename ST>
__global__ void k_update_p(Level L, float* __restrict__ p, const Control* ctl) {
  pdl_enter();
  update_p_body<ST>(blockIdx.x, gridDim.x, L, p, ctl);
}

// reduce(z, r) (mgpcg.py:171, :201) with the scalar epilogue.
//  mode 0 (before the loop): old_zTr = z.r; the loop runs iff max_iters != 0.
//  mode 1 (end of an iteration): beta = new / (old + eps); old = new; iter++;
//          stop at max_iters (mgpcg.py:176, :200-209).
//
// Ap != null (the mixed form): flexible beta, the A-orthogonalisation of the
// new z against the last direction, beta = -z.Ap / p.Ap (Notay's flexible
// CG with one direction kept; equal to the reference's z.r ratio for a fixed
// SPD preconditioner in exact arithmetic).  A V-cycle on 16-bit grids is a
// slightly different operator at every application, for which the
// reference's beta loses conjugacy and stalls.
template <typename ST>
__device__ __forceinline__ void zr_body(int bid_, int nb_, Level L, Control* ctl, double* partials, int mode,
                                                    const float* __restrict__ Ap) {

  __shared__ double sh[32];
  const ST* z = (const ST*)L.z;
  const float* r = (const float*)L.r;
  const float sz = (float)ctl->scale_z;
  const bool flex = Ap != nullptr && mode == 1;
  double acc = 0.0, zap = 0.0;
  for (long long i = (long long)bid_ * blockDim.x + threadIdx.x; i < L.g.count;
       i += (long long)nb_ * blockDim.x)
    if (L.type[i] == FLUID) {
      const double zi = (double)z_true<ST>(z, i, sz);
      acc += zi * (double)r[i];
      if (flex) zap += zi * (double)Ap[i];
    }
  double tot;
  if (flex) {  // z.Ap first (its own counter); the z.r epilogue below reads it
    double tz;
    if (last_block_total_at<kRedThreads>(zap, partials + kMaxPartials / 2, &ctl->counter[5], sh, &tz, bid_, nb_) &&
        threadIdx.x == 0)
      ctl->zAp = tz;
  }
  if (last_block_total_at<kRedThreads>(acc, partials, &ctl->counter[1], sh, &tot, bid_, nb_) && threadIdx.x == 0) {
    if (mode == 0) {
      ctl->old_zTr = tot;
      if (ctl->max_iters == 0) ctl->run = 0;
    } else {
      ctl->new_zTr = tot;
      if (flex) {
        __threadfence();
        const double zap_t = ((volatile Control*)ctl)->zAp;
        ctl->beta = (float)(-zap_t / (ctl->pAp + ctl->eps));
      } else {
        ctl->beta = (float)(tot / (ctl->old_zTr + ctl->eps));
      }
      ctl->old_zTr = tot;
      ctl->iter += 1;
      if (ctl->max_iters != -1 && ctl->iter >= ctl->max_iters) ctl->run = 0;
    }
  }
}

template <typename ST>
__global__ void __launch_bounds__(kRedThreads) k_zr(Level L, Control* ctl, double* partials, int mode,
                                                    const float* __restrict__ Ap = nullptr) {
  pdl_enter();
  zr_body<ST>(blockIdx.x, gridDim.x, L, ctl, partials, mode, Ap);
}

// float32 grids whose cell count is a multiple of 4: the same two kernels
// over 4-cell groups (16-byte loads of z, r, p; 4 labels in one load).
__device__ __forceinline__ bool fluid_lane(uint32_t t4, int e) { return ((t4 >> (8 * e)) & 0xffu) == (uint32_t)FLUID; }

__device__ __forceinline__ void update_p4_body(int bid_, int nb_, Level L, float* __restrict__ p, const Control* ctl) {

  const float beta = ctl->beta;
  const int groups = (int)(L.g.count >> 2);
  for (int q = bid_ * blockDim.x + threadIdx.x; q < groups; q += nb_ * blockDim.x) {
    const uint32_t t4 = __ldg(reinterpret_cast<const uint32_t*>(L.type) + q);
    if (t4 == 0x02020202u || t4 == 0x01010101u) continue;  // no FLUID lane (all SOLID / all AIR)
    const float4 z = __ldg(reinterpret_cast<const float4*>((const float*)L.z) + q);
    float4 pv = reinterpret_cast<float4*>(p)[q];
    const float zv[4] = {z.x, z.y, z.z, z.w};
    float* pp = reinterpret_cast<float*>(&pv);
#pragma unroll
    for (int e = 0; e < 4; ++e)
      if (fluid_lane(t4, e)) pp[e] = __fadd_rn(zv[e], __fmul_rn(beta, pp[e]));
    reinterpret_cast<float4*>(p)[q] = pv;
  }
}

// The last post-smoothing half sweep of level 0 (colour 0, k_smooth_w4) of a
// whole-domain level split into per-kernel passes, fused with the z.r that
// k_zr4 would compute after it (mgpcg.py:161-166, 197-202): every thread has
// its group's four final z values (two it computes, two of the other colour,
// final since the half sweep before) and r, so the sum costs no extra pass;
// the last block runs k_zr4's epilogue.  At most kMaxPartials / 2 blocks.
__global__ void __launch_bounds__(kRedThreads) k_smooth_zr_w4(Level L, int phase, Control* ctl, double* partials,
                                                              int mode) {
  pdl_enter();
  __shared__ double sh[32];
  const int n1 = L.g.n[1], n2 = L.g.n[2];
  const int q2 = n2 >> 2;
  const long long groups = L.g.count >> 2;
  float* z = (float*)L.z;
  double acc = 0.0;
  for (long long q = gtid(); q < groups; q += gstride()) {
    long long row;
    int x, i1, i0;
    group4_coords(q, q2, n1, groups, row, x, i1, i0);
    const int e0 = (phase - i0 - i1 - x) & 1;  // first cell of the colour in the group
    Group4 g;
    load_group4(L, z, i0, i1, x, g);
    float out[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float v = 0.0f;
#pragma unroll
      for (int ee = 0; ee < 2; ++ee) {  // unrolled over both values of e0
        const int e = ee + 2 * h;
        if (ee == e0) v = div_pos(__fsub_rn(g.R[e], group4_nsum(g, e)), g.D[e]);
      }
      out[h] = v;
    }
    const long long idx = row * n2 + x;
    z[idx + e0] = out[0];
    z[idx + e0 + 2] = out[1];
#pragma unroll
    for (int e = 0; e < 4; ++e) {  // every cell FLUID (whole-domain level)
      const float ze = ((e - e0) & 1) ? g.Z[e] : out[e >> 1];
      acc += (double)ze * (double)g.R[e];
    }
  }
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

__global__ void k_update_p4(Level L, float* __restrict__ p, const Control* ctl) {
  pdl_enter();
  update_p4_body(blockIdx.x, gridDim.x, L, p, ctl);
}

__device__ __forceinline__ void zr4_body(int bid_, int nb_, Level L, Control* ctl, double* partials, int mode) {

  __shared__ double sh[32];
  const int groups = (int)(L.g.count >> 2);
  double acc = 0.0;
  for (int q = bid_ * blockDim.x + threadIdx.x; q < groups; q += nb_ * blockDim.x) {
    const uint32_t t4 = __ldg(reinterpret_cast<const uint32_t*>(L.type) + q);
    if (t4 == 0x02020202u || t4 == 0x01010101u) continue;
    const float4 z = __ldg(reinterpret_cast<const float4*>((const float*)L.z) + q);
    const float4 r = __ldg(reinterpret_cast<const float4*>((const float*)L.r) + q);
    if (fluid_lane(t4, 0)) acc += (double)z.x * (double)r.x;
    if (fluid_lane(t4, 1)) acc += (double)z.y * (double)r.y;
    if (fluid_lane(t4, 2)) acc += (double)z.z * (double)r.z;
    if (fluid_lane(t4, 3)) acc += (double)z.w * (double)r.w;
  }
  double tot;
  if (last_block_total_at<kRedThreads>(acc, partials, &ctl->counter[1], sh, &tot, bid_, nb_) && threadIdx.x == 0) {
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

__global__ void __launch_bounds__(kRedThreads) k_zr4(Level L, Control* ctl, double* partials, int mode) {
  pdl_enter();
  zr4_body(blockIdx.x, gridDim.x, L, ctl, partials, mode);
}

// compute_Ap (mgpcg.py:218-224) + reduce(p, Ap) + alpha = zTr / (pAp + eps).
__global__ void __launch_bounds__(kRedThreads) k_Ap_alpha(Level L, const float* __restrict__ p,
                                                          float* __restrict__ Ap, Control* ctl,
                                                          double* partials, int force = 0) {
  pdl_enter();
  if (!ctl->run && !force) return;
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

// Component e (a compile-time constant after unrolling) of a float4, without
// taking its address (which would keep the vector in local memory).
__device__ __forceinline__ float f4at(const float4& v, int e) {
  return e == 0 ? v.x : (e == 1 ? v.y : (e == 2 ? v.z : v.w));
}

// k_Ap_alpha over groups of 4 consecutive cells along the fastest axis (its
// extent a multiple of 4): 16-byte loads of labels, Adiag, p, the stored
// couplings and the neighbour rows; the neighbour sum of nbr_sum_f32 per
// cell in the same order.  Ap written on FLUID cells only.
// Coordinates of the 4-cell groups a grid-stride loop visits, advanced by the
// fixed stride without integer division: cell i = 4q of the level has
// x = i % nx along the fastest axis and t = i / nx = c0 n1 + c1 (2D: c0 = t).
struct GroupWalk {
  int x, c0, c1;     // coordinates of the current group's first cell
  int dx, dc0, dc1;  // the loop's stride in cells, split the same way
  int nx, n1, dim;
  __device__ __forceinline__ GroupWalk(const Geom& g, int q, int stride_groups)
      : GroupWalk(g.dim, g.n[g.dim - 1], g.n[1], q, stride_groups) {}
  // the extents given directly (no runtime index into a Geom, which would
  // keep the kernel parameter in local memory)
  __device__ __forceinline__ GroupWalk(int dim_, int nx_, int n1_, int q, int stride_groups) {
    dim = dim_;
    nx = nx_;
    n1 = n1_;
    const long long i = 4LL * q, di = 4LL * stride_groups;
    const long long t = i / nx, dt = di / nx;
    x = (int)(i % nx);
    dx = (int)(di % nx);
    if (dim == 3) {
      c0 = (int)(t / n1);
      c1 = (int)(t % n1);
      dc0 = (int)(dt / n1);
      dc1 = (int)(dt % n1);
    } else {
      c0 = (int)t;
      c1 = 0;
      dc0 = (int)dt;
      dc1 = 0;
    }
  }
  __device__ __forceinline__ void advance() {
    x += dx;
    int carry = 0;
    if (x >= nx) {
      x -= nx;
      carry = 1;
    }
    if (dim == 3) {
      c1 += dc1 + carry;
      c0 += dc0;
      if (c1 >= n1) {
        c1 -= n1;
        c0 += 1;
      }
    } else {
      c0 += dc0 + carry;
    }
  }
};

// The grid-stride loop of k_Ap_alpha4 for a compile-time dim (the per-axis
// neighbour rows and couplings stay in registers); returns this thread's p.Ap.
template <int DIM>
__device__ __forceinline__ double Ap4_loop(Level L, const float* __restrict__ p, float* __restrict__ Ap) {
  constexpr int dim = DIM;
  const int nx = L.g.n[dim - 1];
  const int groups = (int)(L.g.count >> 2);
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  double acc = 0.0;
  const int q0 = blockIdx.x * blockDim.x + threadIdx.x, S = gridDim.x * blockDim.x;
  GroupWalk w(dim, nx, L.g.n[1], q0, S);
  // the next group's labels are loaded one iteration ahead: the loads of a
  // group wait on one round trip, not two
  const uint32_t* t4p = reinterpret_cast<const uint32_t*>(L.type);
  uint32_t t4n = q0 < groups ? __ldg(t4p + q0) : 0x01010101u;
  for (int q = q0; q < groups; q += S, w.advance()) {
    const int i = q << 2;
    const uint32_t t4 = t4n;
    t4n = q + S < groups ? __ldg(t4p + q + S) : 0x01010101u;
    if (t4 == 0x02020202u || t4 == 0x01010101u) continue;
    const int x = w.x;
    const int c[2] = {w.c0, w.c1};  // coordinates of the slower axes
    const float4 pc = __ldg(reinterpret_cast<const float4*>(p + i));
    const float4 ad = __ldg(reinterpret_cast<const float4*>(L.Adiag + i));
    const float* axx = L.Ax[dim - 1];
    const float4 xc = __ldg(reinterpret_cast<const float4*>(axx + i));
    const float pxl = x > 0 ? __ldg(p + i - 1) : 0.0f, axl = x > 0 ? __ldg(axx + i - 1) : 0.0f;
    const float pxr = x + 4 < nx ? __ldg(p + i + 4) : 0.0f;
    float4 plo[2], phi_[2], alo[2], ahi[2];
    bool has_lo[2], has_hi[2];
#pragma unroll
    for (int k = 0; k < dim - 1; ++k) {
      const int st = k == 0 ? (dim == 3 ? L.g.n[1] * nx : nx) : nx;
      has_lo[k] = c[k] > 0;
      has_hi[k] = c[k] + 1 < L.g.n[k];
      plo[k] = has_lo[k] ? __ldg(reinterpret_cast<const float4*>(p + i - st)) : z4;
      alo[k] = has_lo[k] ? __ldg(reinterpret_cast<const float4*>(L.Ax[k] + i - st)) : z4;
      phi_[k] = has_hi[k] ? __ldg(reinterpret_cast<const float4*>(p + i + st)) : z4;
      ahi[k] = __ldg(reinterpret_cast<const float4*>(L.Ax[k] + i));
    }
    // components through f4at (see Ap_uniform4_loop)
    float out[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if (!fluid_lane(t4, e)) continue;
      float ret = 0.0f;
#pragma unroll
    for (int k = 0; k < dim - 1; ++k) {
        const float lo = has_lo[k] ? __fmul_rn(f4at(alo[k], e), f4at(plo[k], e)) : 0.0f;
        const float hi = has_hi[k] ? __fmul_rn(f4at(ahi[k], e), f4at(phi_[k], e)) : 0.0f;
        ret = __fadd_rn(ret, __fadd_rn(lo, hi));
      }
      const float lo = x + e > 0 ? __fmul_rn(e == 0 ? axl : f4at(xc, e - 1), e == 0 ? pxl : f4at(pc, e - 1)) : 0.0f;
      const float hi = x + e + 1 < nx ? __fmul_rn(f4at(xc, e), e == 3 ? pxr : f4at(pc, e + 1)) : 0.0f;
      ret = __fadd_rn(ret, __fadd_rn(lo, hi));
      const float v = __fadd_rn(__fmul_rn(f4at(ad, e), f4at(pc, e)), ret);
      out[e] = v;
      acc += (double)f4at(pc, e) * (double)v;
    }
    if (t4 == 0x01010101u * (uint32_t)(uint8_t)FLUID) {  // every lane FLUID (the whole-domain form): one 16-byte store
      *reinterpret_cast<float4*>(Ap + i) = make_float4(out[0], out[1], out[2], out[3]);
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (fluid_lane(t4, e)) Ap[i + e] = out[e];
    }
  }
  return acc;
}

__global__ void __launch_bounds__(kRedThreads, 4) k_Ap_alpha4(Level L, const float* __restrict__ p,
                                                           float* __restrict__ Ap, Control* ctl, double* partials,
                                                           int force = 0) {
  pdl_enter();
  if (!ctl->run && !force) return;
  __shared__ double sh[32];
  const double acc = L.g.dim == 3 ? Ap4_loop<3>(L, p, Ap) : Ap4_loop<2>(L, p, Ap);
  double tot;
  if (last_block_total<kRedThreads>(acc, partials, &ctl->counter[2], sh, &tot) && threadIdx.x == 0) {
    ctl->pAp = tot;
    ctl->alpha = (float)(ctl->old_zTr / (tot + ctl->eps));
  }
}

// The same for a label-uniform level 0 (every coupling -s between FLUID
// cells): Ap = Adiag p + sum over in-range neighbours of (-s) p.  p is 0 on
// every non-FLUID cell (update_p writes FLUID cells only), so a neighbour term
// equals the reference's Ax * p up to the sign of a zero product; FLUID is
// Adiag != 0 (checked by mg_plan_prepare).  No Ax arrays, no labels: 12 bytes
// per cell instead of 25, the same values and the same summation order.
__device__ __forceinline__ void Ap_alpha_uniform_body(int bid_, int nb_, Level L, const float* __restrict__ p,
                                                                  float* __restrict__ Ap, float s, Control* ctl,
                                                                  double* partials, int force) {

  if (!ctl->run && !force) return;
  __shared__ double sh[32];
  const float ms = -s;
  double acc = 0.0;
  for (long long i = (long long)bid_ * blockDim.x + threadIdx.x; i < L.g.count;
       i += (long long)nb_ * blockDim.x) {
    const float a = L.Adiag[i];
    if (a == 0.0f) continue;
    int c[3];
    L.g.coords(i, c);
    const float pi = p[i];
    float ret = 0.0f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      if (k >= L.g.dim) break;
      const long long st = L.g.stride(k);
      const float lo = c[k] > 0 ? __fmul_rn(ms, p[i - st]) : 0.0f;
      const float hi = c[k] + 1 < L.g.n[k] ? __fmul_rn(ms, p[i + st]) : 0.0f;
      ret = __fadd_rn(ret, __fadd_rn(lo, hi));
    }
    const float v = __fadd_rn(__fmul_rn(a, pi), ret);
    Ap[i] = v;
    acc += (double)pi * (double)v;
  }
  double tot;
  if (last_block_total_at<kRedThreads>(acc, partials, &ctl->counter[2], sh, &tot, bid_, nb_) && threadIdx.x == 0) {
    ctl->pAp = tot;
    ctl->alpha = (float)(ctl->old_zTr / (tot + ctl->eps));
  }
}

__global__ void __launch_bounds__(kRedThreads) k_Ap_alpha_uniform(Level L, const float* __restrict__ p,
                                                                  float* __restrict__ Ap, float s, Control* ctl,
                                                                  double* partials, int force = 0) {
  pdl_enter();
  Ap_alpha_uniform_body(blockIdx.x, gridDim.x, L, p, Ap, s, ctl, partials, force);
}

// k_Ap_alpha_uniform over groups of 4 consecutive cells along the fastest
// axis (its extent a multiple of 4, as every fused plan has): 16-byte loads of
// Adiag, p and the p rows of the other axes' neighbours, two scalar loads for
// the x neighbours, 32-bit indices, several groups in flight per thread.  The
// same float32 operations per cell in the same axis order; non-FLUID cells
// keep their Ap (written only where Adiag != 0).
// The grid-stride loop of Ap_alpha_uniform4_body for a compile-time dim (the
// per-axis neighbour rows stay in registers); returns this thread's p.Ap.
template <int DIM>
__device__ __forceinline__ double Ap_uniform4_loop(int bid_, int nb_, Level L, const float* __restrict__ p,
                                                   float* __restrict__ Ap, float ms) {
  constexpr int dim = DIM;
  const int nx = L.g.n[dim - 1];
  const int groups = (int)(L.g.count >> 2);
  double acc = 0.0;
  const int q0 = bid_ * blockDim.x + threadIdx.x, S = nb_ * blockDim.x;
  GroupWalk w(dim, nx, L.g.n[1], q0, S);
  // the next group's Adiag is loaded one iteration ahead: a group's p loads
  // wait on one round trip, not two
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  float4 an = q0 < groups ? __ldg(reinterpret_cast<const float4*>(L.Adiag) + q0) : z4;
  for (int q = q0; q < groups; q += S, w.advance()) {
    const int i = q << 2;
    const float4 a = an;
    an = q + S < groups ? __ldg(reinterpret_cast<const float4*>(L.Adiag) + q + S) : z4;
    // a group without a FLUID cell loads nothing more (large AIR regions at
    // sizes beyond L2)
    if (a.x == 0.0f && a.y == 0.0f && a.z == 0.0f && a.w == 0.0f) continue;
    const int x = w.x;
    const int c[2] = {w.c0, w.c1};  // coordinates of the slower axes
    const float4 pc = __ldg(reinterpret_cast<const float4*>(p + i));
    const float pxl = x > 0 ? __ldg(p + i - 1) : 0.0f;
    const float pxr = x + 4 < nx ? __ldg(p + i + 4) : 0.0f;
    float4 lo4[2], hi4[2];
    bool has_lo[2], has_hi[2];
#pragma unroll
    for (int k = 0; k < dim - 1; ++k) {
      const int st = k == 0 ? (dim == 3 ? L.g.n[1] * nx : nx) : nx;
      has_lo[k] = c[k] > 0;
      has_hi[k] = c[k] + 1 < L.g.n[k];
      lo4[k] = has_lo[k] ? __ldg(reinterpret_cast<const float4*>(p + i - st)) : z4;
      hi4[k] = has_hi[k] ? __ldg(reinterpret_cast<const float4*>(p + i + st)) : z4;
    }
    // components through f4at (the neighbours e - 1, e + 1 of the end cells
    // are never selected; an array indexed there would live in local memory)
    float out[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      float ret = 0.0f;
#pragma unroll
      for (int k = 0; k < dim - 1; ++k) {
        const float lo = has_lo[k] ? __fmul_rn(ms, f4at(lo4[k], e)) : 0.0f;
        const float hi = has_hi[k] ? __fmul_rn(ms, f4at(hi4[k], e)) : 0.0f;
        ret = __fadd_rn(ret, __fadd_rn(lo, hi));
      }
      const float pl = e == 0 ? pxl : f4at(pc, e - 1);
      const float pr = e == 3 ? pxr : f4at(pc, e + 1);
      const float lo = x + e > 0 ? __fmul_rn(ms, pl) : 0.0f;
      const float hi = x + e + 1 < nx ? __fmul_rn(ms, pr) : 0.0f;
      ret = __fadd_rn(ret, __fadd_rn(lo, hi));
      const float pe = f4at(pc, e), ae = f4at(a, e);
      out[e] = __fadd_rn(__fmul_rn(ae, pe), ret);
      if (ae != 0.0f) acc += (double)pe * (double)out[e];
    }
    if (a.x != 0.0f && a.y != 0.0f && a.z != 0.0f && a.w != 0.0f) {
      *reinterpret_cast<float4*>(Ap + i) = make_float4(out[0], out[1], out[2], out[3]);
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (f4at(a, e) != 0.0f) Ap[i + e] = out[e];
    }
  }
  return acc;
}

__device__ __forceinline__ void Ap_alpha_uniform4_body(int bid_, int nb_, Level L, const float* __restrict__ p,
                                                                   float* __restrict__ Ap, float s, Control* ctl,
                                                                   double* partials, int force) {

  if (!ctl->run && !force) return;
  __shared__ double sh[32];
  const double acc = L.g.dim == 3 ? Ap_uniform4_loop<3>(bid_, nb_, L, p, Ap, -s)
                                  : Ap_uniform4_loop<2>(bid_, nb_, L, p, Ap, -s);
  double tot;
  if (last_block_total_at<kRedThreads>(acc, partials, &ctl->counter[2], sh, &tot, bid_, nb_) && threadIdx.x == 0) {
    ctl->pAp = tot;
    ctl->alpha = (float)(ctl->old_zTr / (tot + ctl->eps));
  }
}

__global__ void __launch_bounds__(kRedThreads) k_Ap_alpha_uniform4(Level L, const float* __restrict__ p,
                                                                   float* __restrict__ Ap, float s, Control* ctl,
                                                                   double* partials, int force = 0) {
  pdl_enter();
  Ap_alpha_uniform4_body(blockIdx.x, gridDim.x, L, p, Ap, s, ctl, partials, force);
}

// update_xr (mgpcg.py:226-232) + reduce(r, r) + the convergence test
// (mgpcg.py:188-195).  Sets the while-node condition to ctl->run.
__device__ __forceinline__ void xr_body(int bid_, int nb_, Level L, float* __restrict__ x,
                                                    const float* __restrict__ p,
                                                    const float* __restrict__ Ap, Control* ctl,
                                                    double* partials, cudaGraphConditionalHandle cond,
                                                    int has_cond, int force, double* __restrict__ xh) {

  __shared__ double sh[32];
  if (!ctl->run && !force) {
    if (has_cond && bid_ == 0 && threadIdx.x == 0) cudaGraphSetConditional(cond, 0);
    return;
  }
  const float alpha = ctl->alpha;
  float* r = (float*)L.r;
  double acc = 0.0;
  for (long long i = (long long)bid_ * blockDim.x + threadIdx.x; i < L.g.count;
       i += (long long)nb_ * blockDim.x) {
    if (L.type[i] != FLUID) continue;
    if (xh) {  // mixed form: x accumulates in FP64, x (float32) is its rounding
      const double v = xh[i] + (double)alpha * (double)p[i];
      xh[i] = v;
      x[i] = (float)v;
    } else {
      x[i] = __fadd_rn(x[i], __fmul_rn(alpha, p[i]));
    }
    float ri = __fsub_rn(r[i], __fmul_rn(alpha, Ap[i]));
    r[i] = ri;
    acc += (double)ri * (double)ri;
  }
  double tot;
  if (last_block_total_at<kRedThreads>(acc, partials, &ctl->counter[3], sh, &tot, bid_, nb_) && threadIdx.x == 0) {
    ctl->rTr = tot;
    if (!isfinite(tot)) {
      ctl->status = MG_SOLVE_NONFINITE;
      ctl->run = 0;
    } else if (tot < ctl->tol) {
      ctl->status = MG_SOLVE_CONVERGED;
      ctl->run = 0;
    }
    if (ctl->wait_timeout) {  // a sweep gave up waiting for its TMA loads
      ctl->status = MG_SOLVE_TIMEOUT;
      ctl->run = 0;
    }
    ctl->since_refresh += 1;
    set_scales(ctl, tot);
    if (has_cond) cudaGraphSetConditional(cond, ctl->run ? 1u : 0u);
  }
}

__global__ void __launch_bounds__(kRedThreads) k_xr(Level L, float* __restrict__ x,
                                                    const float* __restrict__ p,
                                                    const float* __restrict__ Ap, Control* ctl,
                                                    double* partials, cudaGraphConditionalHandle cond,
                                                    int has_cond, int force = 0, double* __restrict__ xh = nullptr) {
  pdl_enter();
  xr_body(blockIdx.x, gridDim.x, L, x, p, Ap, ctl, partials, cond, has_cond, force, xh);
}

// k_xr on 4-cell groups (one 16-byte vector of x, p, r, Ap and one 32-bit
// word of labels per group; the cell count a multiple of 4): the same
// per-cell arithmetic, r.r summed group by group.
__device__ __forceinline__ void xr4_body(int bid_, int nb_, Level L, float* __restrict__ x,
                                                     const float* __restrict__ p,
                                                     const float* __restrict__ Ap, Control* ctl,
                                                     double* partials, cudaGraphConditionalHandle cond,
                                                     int has_cond, int force, double* __restrict__ xh) {

  __shared__ double sh[32];
  if (!ctl->run && !force) {
    if (has_cond && bid_ == 0 && threadIdx.x == 0) cudaGraphSetConditional(cond, 0);
    return;
  }
  const float alpha = ctl->alpha;
  float* r = (float*)L.r;
  const int groups = (int)(L.g.count >> 2);
  double acc = 0.0;
  const int S = nb_ * blockDim.x;
  // two groups per iteration (q and q + S, the grid-stride order), every load
  // of both issued before either is used: twice the bytes in flight
  for (int q = bid_ * blockDim.x + threadIdx.x; q < groups; q += 2 * S) {
    uint32_t t4[2];
    float4 xv[2], pv[2], rv[2], av[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int qq = q + u * S;
      t4[u] = 0x01010101u;
      if (qq < groups) {
        t4[u] = __ldg(reinterpret_cast<const uint32_t*>(L.type) + qq);
        xv[u] = reinterpret_cast<float4*>(x)[qq];
        pv[u] = __ldg(reinterpret_cast<const float4*>(p) + qq);
        rv[u] = reinterpret_cast<float4*>(r)[qq];
        av[u] = __ldg(reinterpret_cast<const float4*>(Ap) + qq);
      }
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int qq = q + u * S;
      if (t4[u] == 0x02020202u || t4[u] == 0x01010101u) continue;  // no FLUID lane (or past the end)
      float* xs = reinterpret_cast<float*>(&xv[u]);
      float* rs = reinterpret_cast<float*>(&rv[u]);
      const float ps[4] = {pv[u].x, pv[u].y, pv[u].z, pv[u].w}, as[4] = {av[u].x, av[u].y, av[u].z, av[u].w};
      if (xh) {  // mixed form: x accumulates in FP64, x (float32) is its rounding
        double2* xh2 = reinterpret_cast<double2*>(xh) + 2 * qq;
        double2 h0 = xh2[0], h1 = xh2[1];
        double hv[4] = {h0.x, h0.y, h1.x, h1.y};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          if (!fluid_lane(t4[u], e)) continue;
          hv[e] += (double)alpha * (double)ps[e];
          xs[e] = (float)hv[e];
        }
        xh2[0] = make_double2(hv[0], hv[1]);
        xh2[1] = make_double2(hv[2], hv[3]);
      }
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        if (!fluid_lane(t4[u], e)) continue;
        if (!xh) xs[e] = __fadd_rn(xs[e], __fmul_rn(alpha, ps[e]));
        rs[e] = __fsub_rn(rs[e], __fmul_rn(alpha, as[e]));
        acc += (double)rs[e] * (double)rs[e];
      }
      reinterpret_cast<float4*>(x)[qq] = xv[u];
      reinterpret_cast<float4*>(r)[qq] = rv[u];
    }
  }
  double tot;
  if (last_block_total_at<kRedThreads>(acc, partials, &ctl->counter[3], sh, &tot, bid_, nb_) && threadIdx.x == 0) {
    ctl->rTr = tot;
    if (!isfinite(tot)) {
      ctl->status = MG_SOLVE_NONFINITE;
      ctl->run = 0;
    } else if (tot < ctl->tol) {
      ctl->status = MG_SOLVE_CONVERGED;
      ctl->run = 0;
    }
    if (ctl->wait_timeout) {  // a sweep gave up waiting for its TMA loads
      ctl->status = MG_SOLVE_TIMEOUT;
      ctl->run = 0;
    }
    ctl->since_refresh += 1;
    set_scales(ctl, tot);
    if (has_cond) cudaGraphSetConditional(cond, ctl->run ? 1u : 0u);
  }
}

__global__ void __launch_bounds__(kRedThreads) k_xr4(Level L, float* __restrict__ x,
                                                     const float* __restrict__ p,
                                                     const float* __restrict__ Ap, Control* ctl,
                                                     double* partials, cudaGraphConditionalHandle cond,
                                                     int has_cond, int force = 0, double* __restrict__ xh = nullptr) {
  pdl_enter();
  xr4_body(blockIdx.x, gridDim.x, L, x, p, Ap, ctl, partials, cond, has_cond, force, xh);
}

// True-residual refresh (the mixed form's iterative refinement): every
// refresh_every iterations, and whenever the recursive residual claims
// convergence, r = b - A x is recomputed in FP64 arithmetic from the stored
// float32 x, and the convergence test is taken again on it.  The recursive
// residual of the reference never does this (mgpcg.py:226-232).
__device__ __forceinline__ void refresh_body(int bid_, int nb_, Level L, const float* __restrict__ b,
                                                         const float* __restrict__ x, Control* ctl,
                                                         double* partials, cudaGraphConditionalHandle cond,
                                                         int has_cond, const double* __restrict__ xh) {

  __shared__ double sh[32];
  const bool claimed = ctl->status == MG_SOLVE_CONVERGED && !ctl->run;
  const bool due = ctl->run && ctl->refresh_every > 0 && ctl->since_refresh >= ctl->refresh_every;
  if (!(claimed || due)) {
    if (has_cond && bid_ == 0 && threadIdx.x == 0) cudaGraphSetConditional(cond, ctl->run ? 1u : 0u);
    return;
  }
  float* r = (float*)L.r;
  double acc = 0.0;
  for (long long i = (long long)bid_ * blockDim.x + threadIdx.x; i < L.g.count;
       i += (long long)nb_ * blockDim.x) {
    if (L.type[i] != FLUID) continue;
    int c[3];
    L.g.coords(i, c);
    // x in FP64 (the mixed form's accumulated copy) or the float32 x
    auto xv = [&](long long j) { return xh ? xh[j] : (double)x[j]; };
    double ax = (double)L.Adiag[i] * xv(i);
    for (int k = 0; k < L.g.dim; ++k) {
      const long long s = L.g.stride(k);
      if (c[k] > 0) ax += (double)L.Ax[k][i - s] * xv(i - s);
      if (c[k] + 1 < L.g.n[k]) ax += (double)L.Ax[k][i] * xv(i + s);
    }
    const double rr = (double)b[i] - ax;
    r[i] = (float)rr;
    acc += rr * rr;
  }
  double tot;
  if (last_block_total_at<kRedThreads>(acc, partials, &ctl->counter[7], sh, &tot, bid_, nb_) && threadIdx.x == 0) {
    ctl->rTr = tot;
    ctl->since_refresh = 0;
    if (!isfinite(tot)) {
      ctl->status = MG_SOLVE_NONFINITE;
      ctl->run = 0;
    } else if (tot < ctl->tol) {
      ctl->status = MG_SOLVE_CONVERGED;
      ctl->run = 0;
    } else {
      // the recursive residual was too optimistic: keep iterating
      ctl->status = MG_SOLVE_MAX_ITERS;
      ctl->run = ctl->max_iters == -1 || ctl->iter + 1 < ctl->max_iters;
    }
    if (ctl->wait_timeout) {
      ctl->status = MG_SOLVE_TIMEOUT;
      ctl->run = 0;
    }
    set_scales(ctl, tot);
    if (has_cond) cudaGraphSetConditional(cond, ctl->run ? 1u : 0u);
  }
}

__global__ void __launch_bounds__(kRedThreads) k_refresh(Level L, const float* __restrict__ b,
                                                         const float* __restrict__ x, Control* ctl,
                                                         double* partials, cudaGraphConditionalHandle cond,
                                                         int has_cond, const double* __restrict__ xh) {
  pdl_enter();
  refresh_body(blockIdx.x, gridDim.x, L, b, x, ctl, partials, cond, has_cond, xh);
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
