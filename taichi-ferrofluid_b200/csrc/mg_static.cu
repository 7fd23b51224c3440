// mg_reduce_static: the masked inner product of the PCG loop (the reference's
// reduce, mgpcg.py:211-216) for callers that cannot allocate device memory.
//
// Who needs it: a host that owns all of the device memory (a simulation engine
// that reserves one fixed pool at start-up and forbids foreign allocations), a
// real-time step loop in which cudaMalloc/cudaFree would synchronise the device
// and stall the frame, and code that holds no solver plan — mg_reduce needs a
// plan whose workspace the caller has allocated.  This entry point takes only
// the caller's arrays and the output location; its scratch space (the per-block
// FP64 partial sums and the block-arrival counter) is a fixed array compiled
// into the library.
//
// The array is a file-scope `static __device__` object: every GPU that loads
// the library holds its 64 KB until the process exits.  Host code cannot use
// its name as a device address (the host-side symbol is only a stand-in), so
// each call looks the address up with cudaGetSymbolAddress, with the device
// current, and keeps it per device; a call made while its stream is being
// captured uses the kept address instead (the look-up is not a stream
// operation and may load the module).  The first call on a device should
// therefore come before any stream capture.  Looking it up again on every
// other call keeps the address valid after a cudaDeviceReset, which destroys
// the context that held the array.
//
// All calls share the one array and it keeps the last call's contents: the
// counter is cleared at the start of every call, and calls that overlap on the
// GPU (different streams without ordering) race on it.
#include <cstdio>
#include <mutex>

#include "mg_common.cuh"

void mg_internal_set_error(const char* msg);

namespace {

constexpr int kThreads = 256;
constexpr int kCellsPerThread = 16;
constexpr int kMaxBlocks = 8192;  // partial sums held in the static array
constexpr long long kMaxCells = (long long)kMaxBlocks * kThreads * kCellsPerThread;  // 33,554,432
constexpr int kMaxDevices = 64;

struct StaticScratch {
  double partials[kMaxBlocks];
  unsigned int counter;
  unsigned int pad[63];
};

static __device__ __align__(256) StaticScratch g_scratch;

StaticScratch* g_addr[kMaxDevices] = {};
std::mutex g_mu;

__global__ void __launch_bounds__(kThreads) k_dot_static(const int8_t* __restrict__ type, const float* __restrict__ a,
                                                         const float* __restrict__ b, long long n, StaticScratch* S,
                                                         double* out) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    if (type[i] == mg::FLUID) acc += (double)a[i] * (double)b[i];
  double tot;
  if (mg::last_block_total<kThreads>(acc, S->partials, &S->counter, sh, &tot) && threadIdx.x == 0) *out = tot;
}

int fail(int rc, const char* msg) {
  mg_internal_set_error(msg);
  return rc;
}

}  // namespace

extern "C" MG_API int mg_reduce_static(const int8_t* grid_type, const float* a, const float* b, int64_t n,
                                       double* out, void* stream) {
  if (!grid_type || !a || !b || !out) return fail(MG_E_BADARG, "bad argument: mg_reduce_static: null pointer");
  if (n < 0) return fail(MG_E_BADARG, "bad argument: mg_reduce_static: negative cell count");
  if (n > kMaxCells) {
    char msg[160];
    snprintf(msg, sizeof(msg), "mg_reduce_static: %lld cells exceed the static scratch limit of %lld",
             (long long)n, kMaxCells);
    return fail(MG_E_TOO_BIG, msg);
  }
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) return fail(MG_E_CUDA, "mg_reduce_static: cudaGetDevice failed");
  cudaStream_t s = (cudaStream_t)stream;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) {
    cudaGetLastError();  // a stream that cannot be queried: use the kept address
    cap = cudaStreamCaptureStatusActive;
  }
  StaticScratch* S;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (cap == cudaStreamCaptureStatusNone) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_scratch);
      if (e != cudaSuccess || !p) return fail(MG_E_CUDA, "mg_reduce_static: cudaGetSymbolAddress failed");
      g_addr[dev] = (StaticScratch*)p;
    } else if (!g_addr[dev]) {
      return fail(MG_E_CUDA, "mg_reduce_static: the first call on a device must come before stream capture");
    }
    S = g_addr[dev];
  }
  e = cudaMemsetAsync(&S->counter, 0, sizeof(unsigned int), s);
  if (e != cudaSuccess) return fail(MG_E_CUDA, "mg_reduce_static: clearing the counter failed");
  long long blocks = (n + (long long)kThreads * kCellsPerThread - 1) / ((long long)kThreads * kCellsPerThread);
  if (blocks < 1) blocks = 1;
  k_dot_static<<<(int)blocks, kThreads, 0, s>>>(grid_type, a, b, (long long)n, S, out);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(MG_E_CUDA, "mg_reduce_static: launch failed");
  return MG_OK;
}
