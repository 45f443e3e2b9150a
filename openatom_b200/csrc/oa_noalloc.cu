// Allocation-free PairCalculator forward product.
//
// Some callers cannot call cudaMalloc: code inside a host framework whose
// memory pool has already reserved the device memory (a further cudaMalloc
// fails or fragments the pool), or latency-critical paths where
// cudaMalloc's implicit device-wide synchronisation is not acceptable.
// oa_gpu_pc_forward needs a context,
// and creating a context allocates its scratch.  oa_gpu_pc_forward_noalloc
// computes the same product with no context and no allocation: its split-K
// partial sums live in a fixed device array declared in this file.
//
// Limits and sharing:
//   * at most OA_NOALLOC_MAX_STATES (128) states; larger calls are rejected;
//   * the array (OA_NOALLOC_KBLOCKS x 128 x 128 doubles = 4 MiB) exists on
//     every GPU that loads the library, for the life of the process;
//   * every call on a device shares it: two calls whose kernels overlap on
//     the GPU (different streams, no ordering between them) race and give
//     wrong results.  Calls on one stream are ordered and safe;
//   * each call overwrites every partial it reads, so nothing has to be
//     cleared between calls.
#include <mutex>
#include "oa_internal.h"

#define OA_NOALLOC_MAX_STATES 128
#define OA_NOALLOC_KBLOCKS 32
#define OA_NOALLOC_MAX_DEVICES 64

cudaError_t oa_launch_pc_fwd_mn(cudaStream_t s, const double* A, const double* B, int m, int n, long K,
                                long kx0_cols, double w_kx0, double alpha, double* part, int nkb, double* C);

// Split-K partials of the forward product.  In host code this name is only a
// stand-in for the device array: its device address comes from
// cudaGetSymbolAddress below.
static __device__ __align__(256) double g_pcfwd_part[OA_NOALLOC_KBLOCKS * OA_NOALLOC_MAX_STATES *
                                                     OA_NOALLOC_MAX_STATES];

static std::mutex g_noalloc_mu;
static double* g_noalloc_addr[OA_NOALLOC_MAX_DEVICES] = {};

// Device address of g_pcfwd_part on the current device, looked up once per
// device (with that device current) and cached for the life of the process.
// The cache assumes the device's primary context is not reset
// (cudaDeviceReset) while the library is loaded: after a reset the module
// may load at another address and the cached one is stale.
static oa_status noalloc_scratch(double** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) { oa_set_error(cudaGetErrorString(e), __FILE__, __LINE__); return OA_ERR_CUDA; }
  if (dev < 0 || dev >= OA_NOALLOC_MAX_DEVICES) {
    oa_set_error("device index out of range for the allocation-free entry point", __FILE__, __LINE__);
    return OA_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    double* p = nullptr;
    e = cudaGetSymbolAddress((void**)&p, g_pcfwd_part);
    if (e != cudaSuccess || !p) {
      oa_set_error(e != cudaSuccess ? cudaGetErrorString(e) : "cudaGetSymbolAddress returned null", __FILE__,
                   __LINE__);
      return OA_ERR_CUDA;
    }
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return OA_OK;
}

extern "C" oa_status oa_gpu_pc_forward_noalloc(void* stream, const double* left, const double* right, int nstate,
                                               int ng, int nkx0, double alpha, double w_kx0, double* C) {
  if (!left || !right || !C) { oa_set_error("null argument", __FILE__, __LINE__); return OA_ERR_BAD_ARG; }
  if (nstate <= 0 || ng <= 0 || nkx0 < 0 || nkx0 > ng) {
    oa_set_error("bad sizes", __FILE__, __LINE__);
    return OA_ERR_BAD_ARG;
  }
  if (nstate > OA_NOALLOC_MAX_STATES) {
    oa_set_error("oa_gpu_pc_forward_noalloc supports at most 128 states; use oa_gpu_pc_forward", __FILE__,
                 __LINE__);
    return OA_ERR_BAD_ARG;
  }
  double* part = nullptr;
  oa_status st = noalloc_scratch(&part);
  if (st != OA_OK) return st;
  const cudaError_t e = oa_launch_pc_fwd_mn((cudaStream_t)stream, left, right, nstate, nstate, 2L * ng, 2L * nkx0,
                                            w_kx0, alpha, part, OA_NOALLOC_KBLOCKS, C);
  if (e != cudaSuccess) { oa_set_error(cudaGetErrorString(e), __FILE__, __LINE__); return OA_ERR_CUDA; }
  return OA_OK;
}
