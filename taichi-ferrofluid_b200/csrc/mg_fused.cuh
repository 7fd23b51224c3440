// Operator preparation and the fused V-cycle for the label-uniform operator.
//
// "Label-uniform" form: every off-diagonal of a level equals -s_l between two
// FLUID cells and 0 elsewhere.  The pressure Strategy always produces it
// (pressure_project.py:56-58).  The kernels then rebuild each coupling from the
// labels instead of reading dim coefficient arrays: the same values, and so the
// same arithmetic, with 3 to 4 times fewer coefficient bytes per cell.
#pragma once
#include "mg_common.cuh"

namespace mg {

// Per-level check of the label-uniform form.  partials[3*b + {0,1,2}] receive
// the block's min and max of the nonzero off-diagonals and its count of cells
// whose coupling pattern differs from the labels.
__global__ void __launch_bounds__(kRedThreads) k_detect_uniform(Level L, double* partials,
                                                                unsigned int* counter, double* out3) {
  __shared__ double sh[32];
  __shared__ bool am_last;
  double vmin = 1e300, vmax = -1e300, bad = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < L.g.count;
       i += (long long)gridDim.x * blockDim.x) {
    int c[3];
    L.g.coords(i, c);
    const bool fl = L.type[i] == FLUID;
    for (int k = 0; k < L.g.dim; ++k) {
      float a = L.Ax[k][i];
      bool coupled = fl && (c[k] + 1 < L.g.n[k]) && L.type[i + L.g.stride(k)] == FLUID;
      if (a != 0.0f) {
        vmin = fmin(vmin, (double)a);
        vmax = fmax(vmax, (double)a);
        if (!coupled) bad += 1.0;
      } else if (coupled) {
        bad += 1.0;
      }
    }
  }
  // three block reductions (min, max, sum)
  for (int o = 16; o > 0; o >>= 1) {
    vmin = fmin(vmin, __shfl_down_sync(0xffffffffu, vmin, o));
    vmax = fmax(vmax, __shfl_down_sync(0xffffffffu, vmax, o));
    bad += __shfl_down_sync(0xffffffffu, bad, o);
  }
  __shared__ double s3[3][32];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    s3[0][w] = vmin;
    s3[1][w] = vmax;
    s3[2][w] = bad;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 1e300, b = -1e300, c = 0.0;
    for (int j = 0; j < (int)(blockDim.x >> 5); ++j) {
      a = fmin(a, s3[0][j]);
      b = fmax(b, s3[1][j]);
      c += s3[2][j];
    }
    partials[3 * blockIdx.x + 0] = a;
    partials[3 * blockIdx.x + 1] = b;
    partials[3 * blockIdx.x + 2] = c;
    __threadfence();
    am_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (am_last && threadIdx.x == 0) {
    __threadfence();
    double a = 1e300, b = -1e300, c = 0.0;
    volatile double* vp = partials;
    for (unsigned int j = 0; j < gridDim.x; ++j) {
      a = fmin(a, vp[3 * j + 0]);
      b = fmax(b, vp[3 * j + 1]);
      c += vp[3 * j + 2];
    }
    out3[0] = a;
    out3[1] = b;
    out3[2] = c;
    *counter = 0u;
  }
  (void)sh;
}

// Fills op_form[l] (1 label-uniform, 0 stored coefficients).  Synchronises
// `s`: the choice decides which kernels the solve graph launches.
inline int prepare_operator(Level* lv, int L, int storage, Control* ctl, double* partials, int num_sms,
                            int* op_form, float* offdiag, cudaStream_t s) {
  const int blocks = num_sms * 2 < kMaxPartials / 3 ? num_sms * 2 : kMaxPartials / 3;
  for (int l = 0; l < L; ++l) {
    k_detect_uniform<<<blocks, kRedThreads, 0, s>>>(lv[l], partials, &ctl->counter[5], &ctl->scratch[3 * 0 + 1]);
    if (cudaGetLastError() != cudaSuccess) return MG_E_CUDA;
    double h[3];
    if (cudaMemcpyAsync(h, &ctl->scratch[1], sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess) return MG_E_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return MG_E_CUDA;
    const bool none = h[0] > h[1];  // no nonzero off-diagonal at all
    const bool uniform = h[2] == 0.0 && (none || (h[0] == h[1] && h[0] < 0.0));
    op_form[l] = uniform ? 1 : 0;
    offdiag[l] = uniform && !none ? (float)(-h[0]) : 0.0f;
  }
  (void)storage;
  return MG_OK;
}

inline bool fused_supported(int dim, const Geom* geom, int L, int storage) {
  (void)dim; (void)geom; (void)L; (void)storage;
  return false;
}

inline int launch_vcycle_fused(Level* lv, int L, int dim, int pre_post, int bottom, int storage, int num_sms,
                               cudaStream_t s) {
  (void)lv; (void)L; (void)dim; (void)pre_post; (void)bottom; (void)storage; (void)num_sms; (void)s;
  return MG_E_BADARG;
}

}  // namespace mg
