// Shared definitions of the B200 MGPCG library: grid geometry, the per-level
// view passed to kernels, storage-type conversion and reduction helpers.
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "../../include/mgpcg_b200.h"

namespace mg {

constexpr int8_t FLUID = MG_FLUID;
constexpr int8_t AIR = MG_AIR;
constexpr int8_t SOLID = MG_SOLID;

constexpr int kMaxLevels = 12;
constexpr int kRedThreads = 256;      // threads of every reduction kernel
constexpr int kMaxPartials = 2048;    // upper bound on reduction blocks

// Row-major grid geometry, last axis fastest.  A 2D grid is stored as
// (n0, n1, 1) and only axes < dim have neighbours, so one index formula serves
// both dimensionalities: idx = (i0 * n1 + i1) * n2 + i2.
struct Geom {
  int dim;
  int n[3];
  long long count;
  __host__ __device__ inline long long stride(int axis) const {
    return axis == 0 ? (long long)n[1] * n[2] : (axis == 1 ? (long long)n[2] : 1LL);
  }
  __host__ __device__ inline void coords(long long idx, int c[3]) const {
    c[2] = (int)(idx % n[2]);
    long long t = idx / n[2];
    c[1] = (int)(t % n[1]);
    c[0] = (int)(t / n[1]);
  }
  __host__ __device__ inline long long index(int c0, int c1, int c2) const {
    return ((long long)c0 * n[1] + c1) * n[2] + c2;
  }
};

// Device pointers of one multigrid level (all inside the caller's workspace).
struct Level {
  Geom g;
  int8_t* type;     // grid_type[l]
  float* Adiag;     // public f32 coefficients written by the Strategy
  float* Ax[3];     // SoA: Ax[k][idx] = A(idx, idx + e_k)
  void* r;          // level 0: f32 CG residual; coarser: storage type
  void* z;          // storage type
  void* zt;         // storage type: the fused V-cycle's pre-smoothed z
  void* Adiag_s;    // storage-type copy of Adiag (aliases Adiag for f32)
};

// Scalars of the device-resident PCG loop (mgpcg.py:150-209).
struct Control {
  double rTr0, bTb, tol, old_zTr, pAp, rTr, new_zTr;
  double rel_tol, abs_tol, eps;
  float alpha, beta;          // the reference's f32 scalar fields (mgpcg.py:43-44)
  int iter, status, max_iters, run;
  int warm_start, refresh_every, since_refresh;
  int done;                   // a batched solve: this instance has finished (its blocks return)
  double scale_z;             // z (true) = scale_z * z (stored), 16-bit storage only
  double scale_r;             // r (stored, level 0 input of the V-cycle) = scale_r * r
  double kappa;               // coefficient scale of 16-bit grids
  double n_fluid;             // FLUID cells of level 0
  int bad_operator;           // declared operator form: bit 0 wrong, bit 1 a FLUID cell with Adiag 0
  int wait_timeout;           // set when a bounded wait in a kernel ran out
  unsigned int counter[8];    // arrival counters of the last-block reductions
  double scratch[8];          // single-value results of mg_reduce
  double det[4 * 12];         // operator detection per level (k_detect_uniform)
  double zAp;                 // z.Ap of the mixed form's flexible beta
};

// x / a in IEEE float32 for a != 0 (Adiag of a FLUID cell).  A zero dividend
// would take the division's slow path (a subroutine call for the whole warp);
// it is returned as is: x / a bit for bit when a > 0, equal in value (a zero
// of the other sign) when a < 0.
__device__ __forceinline__ float div_pos(float x, float a) {
  const bool z = x == 0.0f;
  const float q = __fdiv_rn(z ? 1.0f : x, a);
  return z ? x : q;
}

// x / a in IEEE float32 (round to nearest even) from yd = 1 / (double)a, for
// a divisor used many times.  The double product x * yd is within 2^-52
// (relative) of x / a, while a quotient of two floats that is not a float
// lies at least 2^-49 (relative) from every float32 rounding boundary (a
// boundary has an odd 25-bit significand, which a 24-bit divisor times it
// cannot bring back to a 24-bit dividend; the same holds for the subnormal
// grid and the overflow threshold), so the product rounds to the correctly
// rounded quotient (rounding twice, first to 53 bits, is innocuous here).
// For a > 0 it is x / a bit for bit, zeros keeping the dividend's sign as in
// div_pos.
__device__ __forceinline__ float div_recip64(float x, double yd) { return __double2float_rn((double)x * yd); }

template <typename T> __device__ __forceinline__ float to_f(T v);
template <> __device__ __forceinline__ float to_f<float>(float v) { return v; }
template <> __device__ __forceinline__ float to_f<__half>(__half v) { return __half2float(v); }
template <> __device__ __forceinline__ float to_f<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }

template <typename T> __device__ __forceinline__ T from_f(float v);
template <> __device__ __forceinline__ float from_f<float>(float v) { return v; }
template <> __device__ __forceinline__ __half from_f<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 from_f<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

// Neighbour sum of mgpcg.py:96-102 in the reference's operation order:
//   ret = 0; for each axis i: ret += (Ax[I-e_i][i] * v[I-e_i] + Ax[I][i] * v[I+e_i])
// An index outside the level contributes 0 (out-of-range rule H1).
__device__ __forceinline__ float nbr_sum_f32(const Level& L, const float* v, long long idx,
                                             const int c[3]) {
  float ret = 0.0f;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    if (i >= L.g.dim) break;
    long long s = L.g.stride(i);
    float lo = 0.0f, hi = 0.0f;
    if (c[i] > 0) lo = __fmul_rn(L.Ax[i][idx - s], v[idx - s]);
    if (c[i] + 1 < L.g.n[i]) hi = __fmul_rn(L.Ax[i][idx], v[idx + s]);
    ret = __fadd_rn(ret, __fadd_rn(lo, hi));
  }
  return ret;
}

// Programmatic dependent launch between the kernels of the PCG loop: each is
// launched with programmatic stream serialisation, so its launch overlaps the
// end of the kernel before it, and it first waits (griddepcontrol.wait; a
// no-op without a programmatic dependency) until that kernel has completed
// and its writes are visible.  Every memory access follows the wait, so the
// overlap changes no result.  An explicit early trigger
// (griddepcontrol.launch_dependents, MG_PDL_TRIGGER=1) lets the next grid's
// CTAs become resident while this one runs; measured on B200 it speeds up
// host-launched V-cycles but slows the graph-launched solve (128^3: 4.84 ->
// 5.07 ms; 256^3: 27.1 -> 29.4 ms), so by default the dependents launch at
// the implicit trigger, this grid's completion (128^3 solve 4.80 ms, V-cycle
// from a host loop 187 -> 173 us).
#ifndef MG_PDL
#define MG_PDL 1
#endif
#ifndef MG_PDL_TRIGGER
#define MG_PDL_TRIGGER 0
#endif
__device__ __forceinline__ void pdl_enter() {
#if MG_PDL
  asm volatile("griddepcontrol.wait;" ::: "memory");
#if MG_PDL_TRIGGER
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
#endif
#endif
}

// Launch with the programmatic-serialisation attribute (see pdl_enter).
template <typename... P, typename... A>
inline cudaError_t launch_k(void (*kern)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, A... args) {
#if MG_PDL
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, args...);
#else
  kern<<<grid, block, smem, s>>>(args...);
  return cudaGetLastError();
#endif
}

// Block-wide FP64 sum; result valid in thread 0.  Fixed tree order.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double t = 0.0;
  if (w == 0) {
    t = lane < NT / 32 ? sh[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
  }
  __syncthreads();
  return t;
}

// Last-block reduction: every block stores its partial; the block that
// arrives last sums all partials in index order (deterministic for a fixed
// grid) and returns true with the total in *total (thread 0 only).  The _at
// form takes the block's index and the block count of its reduction, so that
// one launch can hold the reductions of several solves (a batch), each over
// its own blocks, partials and counter.
template <int NT>
__device__ __forceinline__ bool last_block_total_at(double partial, double* partials, unsigned int* counter,
                                                    double* sh, double* total, int bid, int nb) {
  __shared__ bool am_last;
  double s = block_sum<NT>(partial, sh);
  if (threadIdx.x == 0) {
    partials[bid] = s;
    __threadfence();
    unsigned int prev = atomicAdd(counter, 1u);
    am_last = (prev == (unsigned int)nb - 1);
  }
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
  double acc = 0.0;
  for (int i = threadIdx.x; i < nb; i += NT) acc += ((volatile double*)partials)[i];
  double t = block_sum<NT>(acc, sh);
  if (threadIdx.x == 0) {
    *total = t;
    *counter = 0u;  // ready for the next launch
  }
  return true;
}

template <int NT>
__device__ __forceinline__ bool last_block_total(double partial, double* partials,
                                                 unsigned int* counter, double* sh,
                                                 double* total) {
  return last_block_total_at<NT>(partial, partials, counter, sh, total, (int)blockIdx.x, (int)gridDim.x);
}

}  // namespace mg
