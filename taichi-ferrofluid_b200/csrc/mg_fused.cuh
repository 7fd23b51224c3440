// Operator preparation and the fused V-cycle for the label-uniform operator.
//
// "Label-uniform" form: every off-diagonal of a level equals -s_l between two
// FLUID cells and 0 elsewhere.  The pressure Strategy always produces it
// (pressure_project.py:56-58).  The fused kernels rebuild each coupling from
// the labels instead of reading dim coefficient arrays: the same values, and so
// the same float32 operations in the same order as the stored-coefficient
// kernels of mg_kernels.cuh (the tests check the two bit for bit).
//
// Kernels per V-cycle (mgpcg.py:125-148):
//  * k_sweep<PRE>   level l: z = 0, 2*pre_post red-black half sweeps in colour
//                   order 0,1,0,1,..., then r[l+1] = sum of the 2^d children's
//                   (r - A z) (restrict, mgpcg.py:111-118) and z[l+1] = 0.
//  * k_sweep<POST>  level l: z += z[l+1][I/2] (prolongate, mgpcg.py:120-123),
//                   then 2*pre_post half sweeps in colour order 1,0,1,0,...
//  * k_coarse       the levels from `lc` down, the bottom sweeps and back up,
//                   in ONE thread block with every grid in shared memory.
//
// k_sweep streams a tile of (TY x TX) columns through the slowest axis plane by
// plane.  A ring of NS+3 planes (tile + halo H = NS+1 per side) lives in shared
// memory; after plane p is loaded, half sweep m (m = 1..NS) is applied to plane
// p-m, so every half sweep sees its neighbours at the previous half sweep
// (temporal blocking): each cell's r, A and labels come from memory once per
// kernel instead of once per half sweep.  The in-plane region shrinks by one
// cell per half sweep; a chunk of planes starts NS+1 planes early so its first
// owned plane is exact.
//
// 16-bit storage keeps every grid scaled so that it stays inside the FP16
// range: at level l, r~ = c_l r and z~ = (c_l / kappa) z with c_0 = sigma
// (a power of two near 1/rms(r), set per V-cycle), c_{l+1} = c_l / 2^dim and
// kappa a power of two near 1/s_0 applied to the coefficients.  All factors are
// powers of two, so in float32 they change no bit; with float32 storage they
// are 1.
#pragma once
#include "mg_common.cuh"

namespace mg {

// ---------------------------------------------------------------------------
// Operator detection
// ---------------------------------------------------------------------------

// Per level, into out4: the min and max of the nonzero off-diagonals, the
// count of couplings that differ from the labels (label-uniform test), and
// the count of cells that are not FLUID or have a zero diagonal (0 for a
// whole-domain level: every cell FLUID with a nonzero diagonal).
// partials[4*b + {0..3}] hold the blocks' values; the last block combines them.
__global__ void __launch_bounds__(kRedThreads) k_detect_uniform(Level L, double* partials,
                                                                unsigned int* counter, double* out4) {
  __shared__ bool am_last;
  __shared__ double s4[4][32];
  double v[4] = {1e300, -1e300, 0.0, 0.0};
  const int n1 = L.g.n[1], n2 = L.g.n[2], dim = L.g.dim;
  const int cells = (int)L.g.count;  // levels hold fewer than 2^31 cells
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cells; i += gridDim.x * blockDim.x) {
    const int c2 = i % n2, t = i / n2;
    const int c[3] = {t / n1, t % n1, c2};
    const bool fl = L.type[i] == FLUID;
    const float ad = L.Adiag[i];
    // the fused kernels tell FLUID cells by a nonzero diagonal
    if (fl != (ad != 0.0f)) v[2] += 1.0;
    if (!fl || ad == 0.0f) v[3] += 1.0;
    for (int k = 0; k < dim; ++k) {
      const float a = L.Ax[k][i];
      const int st = k == 0 ? n1 * n2 : (k == 1 ? n2 : 1);
      const bool coupled = fl && (c[k] + 1 < L.g.n[k]) && L.type[i + st] == FLUID;
      if (a != 0.0f) {
        v[0] = fmin(v[0], (double)a);
        v[1] = fmax(v[1], (double)a);
        if (!coupled) v[2] += 1.0;
      } else if (coupled) {
        v[2] += 1.0;
      }
    }
  }
  auto combine = [&](double* x) {  // block-wide min / max / sum / sum into thread 0
    for (int o = 16; o > 0; o >>= 1) {
      x[0] = fmin(x[0], __shfl_down_sync(0xffffffffu, x[0], o));
      x[1] = fmax(x[1], __shfl_down_sync(0xffffffffu, x[1], o));
      x[2] += __shfl_down_sync(0xffffffffu, x[2], o);
      x[3] += __shfl_down_sync(0xffffffffu, x[3], o);
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
      for (int q = 0; q < 4; ++q) s4[q][w] = x[q];
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int j = 1; j < (int)(blockDim.x >> 5); ++j) {
        x[0] = fmin(x[0], s4[0][j]);
        x[1] = fmax(x[1], s4[1][j]);
        x[2] += s4[2][j];
        x[3] += s4[3][j];
      }
    }
    __syncthreads();
  };
  combine(v);
  if (threadIdx.x == 0) {
    for (int q = 0; q < 4; ++q) partials[4 * blockIdx.x + q] = v[q];
    __threadfence();
    am_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  double w[4] = {1e300, -1e300, 0.0, 0.0};
  volatile double* vp = partials;
  for (unsigned int j = threadIdx.x; j < gridDim.x; j += blockDim.x) {
    w[0] = fmin(w[0], vp[4 * j + 0]);
    w[1] = fmax(w[1], vp[4 * j + 1]);
    w[2] += vp[4 * j + 2];
    w[3] += vp[4 * j + 3];
  }
  combine(w);
  if (threadIdx.x == 0) {
    for (int q = 0; q < 4; ++q) out4[q] = w[q];
    *counter = 0u;
  }
}

// Storage-type copy of kappa * Adiag (16-bit storage only).
template <typename ST>
__global__ void k_store_diag(const float* __restrict__ ad, ST* __restrict__ out, long long n, float kappa) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = from_f<ST>(__fmul_rn(kappa, ad[i]));
}

// FLUID cell count of a level into out[0] (for the per-V-cycle r scale).
__global__ void __launch_bounds__(kRedThreads) k_count_fluid(Level L, double* partials, unsigned int* counter,
                                                             double* out) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < L.g.count;
       i += (long long)gridDim.x * blockDim.x)
    acc += L.type[i] == FLUID ? 1.0 : 0.0;
  double tot;
  if (last_block_total<kRedThreads>(acc, partials, counter, sh, &tot) && threadIdx.x == 0) *out = tot;
}

// ---------------------------------------------------------------------------
// Fused kernels
// ---------------------------------------------------------------------------

// One level as the fused kernels see it.
template <typename ST>
struct FLevel {
  int n[3];             // n[2] == 1 in 2D
  const int8_t* type;
  const ST* Ad;         // kappa * Adiag in storage type (aliases Adiag for f32)
  const void* r;        // float (level 0) or ST
  ST* z;                // written: PRE's smoothed z (into the level's second
                        // z buffer), POST's final z
  const ST* zin;        // POST: PRE's smoothed z.  Separate buffers because a
                        // block's halo cells belong to other blocks, which
                        // write their own output while it reads.
  float s;              // kappa * s_l, the coupling magnitude
  const float* ax[3];   // whole-domain stored form: Ax[k] (float32)
};

template <typename ST>
struct SweepArgs {
  FLevel<ST> f;
  ST* rc;               // PRE: coarse r (written); POST: unused
  ST* zc;               // PRE: coarse z (zeroed); POST: coarse z (read)
  int nc[3];
  float rho;            // PRE: c_{l+1} / c_l
  float pi;             // POST: c_l / c_{l+1}
  const Control* ctl;   // sigma for level 0 (scale_r)
  int r_f32;            // level 0: r is float and scaled by sigma on load
  int chunk;            // planes per block along axis 0
  int tiles_x, tiles_y; // tiles per plane
  // POST of level 0, float32: also z.r of the PCG loop (the reduction of
  // k_zr4 and its epilogue) over the cells it writes; -1 off, 0 before the
  // loop, 1 in the loop
  int zr;
  Control* zr_ctl;
  double* zr_partials;
};

// r of a level: level 0 holds the float32 CG residual, scaled by sigma on
// load when the grids are 16-bit; coarser levels hold storage-type values.
template <typename ST>
__device__ __forceinline__ float load_r(const void* r, long long i, int r_f32, float sigma) {
  if (r_f32) {
    const float v = ((const float*)r)[i];
    if constexpr (sizeof(ST) == 4) return v;
    else return __fmul_rn(sigma, v);
  }
  return to_f<ST>(((const ST*)r)[i]);
}

}  // namespace mg
