// bbt_twisted_vectors_noalloc: the twisted-factorisation singular vectors
// of bbt_twisted_vectors, for callers that must not allocate device memory.
//
// Some callers cannot call cudaMalloc: a latency-critical loop in which an
// allocation (and the device synchronisation cudaMalloc/cudaFree can bring)
// is not acceptable, a process whose device memory has been handed in full
// to another allocator (a framework's caching pool, a fixed MPS quota), or
// code that runs with an allocation budget of zero.  This entry point takes
// a stream instead of a bbt_ctx (creating a context allocates) and keeps
// its work arrays in one file-scope __device__ array of fixed size, so it
// allocates nothing; the caller still passes every input and output.
//
// The array is BBT_NOALLOC_SCRATCH_BYTES (64 MiB) and lives on every GPU
// that loads the library until the process exits.  All calls share it and
// it keeps the previous call's contents; every work array is written before
// it is read, so nothing has to be cleared between calls.  Calls whose
// kernels overlap on the GPU (two streams, or two host threads) race on the
// array: serialise them.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "internal.h"

#define BBT_NOALLOC_SCRATCH_BYTES (64u << 20)

namespace {

static __device__ __align__(256) double g_noalloc_scratch[BBT_NOALLOC_SCRATCH_BYTES / sizeof(double)];

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
double* g_addr[MAX_DEVICES] = {};   // device address of g_noalloc_scratch, per device

// The host-side symbol is only a stand-in for the array; its device address
// has to be looked up once per device with that device current.
bbt_status scratch_address(int dev, double** out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (dev < 0 || dev >= MAX_DEVICES) return BBT_ERR_ARG;
  if (!g_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      fprintf(stderr, "bbt_twisted_vectors_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
      return BBT_ERR_CUDA;
    }
    g_addr[dev] = static_cast<double*>(p);
  }
  *out = g_addr[dev];
  return BBT_OK;
}

}  // namespace

extern "C" bbt_status bbt_twisted_vectors_noalloc(void* stream, int n, int cnt, const double* d_sigma,
                                                  const double* d_alpha, const double* d_beta, double* d_U,
                                                  double* d_V) {
  if (n < 1 || cnt < 0 || cnt > n || !d_alpha || (n > 1 && !d_beta) ||
      (cnt > 0 && (!d_sigma || !d_U || !d_V)))
    return BBT_ERR_ARG;
  const size_t need = bbt::scratch_doubles_twisted(n, cnt) * sizeof(double);
  if (need > BBT_NOALLOC_SCRATCH_BYTES) {
    fprintf(stderr,
            "bbt_twisted_vectors_noalloc: n=%d cnt=%d needs %zu bytes of scratch, more than the "
            "%u-byte static array (about 7*(n+1)*cnt doubles must fit)\n",
            n, cnt, need, BBT_NOALLOC_SCRATCH_BYTES);
    return BBT_ERR_ARG;
  }
  if (cnt == 0) return BBT_OK;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return BBT_ERR_CUDA;
  double* scratch = nullptr;
  bbt_status st = scratch_address(dev, &scratch);
  if (st != BBT_OK) return st;
  bbt_ctx ctx;   // stack context: the caller's stream, no workspace, nothing allocated
  ctx.device = dev;
  ctx.stream = static_cast<cudaStream_t>(stream);
  return bbt::twisted_scratch(&ctx, n, cnt, d_sigma, d_alpha, d_beta, d_U, cnt, d_V, scratch);
}
