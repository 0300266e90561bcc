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
//
// The array's device address belongs to the CUDA context that loaded the
// module.  It is looked up (cudaGetSymbolAddress, with the device current)
// on the first call in each context and cached under the context's unique
// id, so a context that is destroyed and created again (cudaDeviceReset)
// gets a fresh lookup instead of a stale address.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "internal.h"

#define BBT_NOALLOC_SCRATCH_BYTES (64u << 20)

namespace {

static __device__ __align__(256) double g_noalloc_scratch[BBT_NOALLOC_SCRATCH_BYTES / sizeof(double)];

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
struct Cached {
  unsigned long long ctx_id = 0;   // the driver's unique id of the context the address belongs to (0: none)
  double* addr = nullptr;
};
Cached g_addr[MAX_DEVICES];

// Driver entry points reached through the runtime (no link against libcuda).
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);
CtxGetCurrentFn g_ctx_current = nullptr;
CtxGetIdFn g_ctx_id = nullptr;

bool driver_entries() {
  if (g_ctx_current && g_ctx_id) return true;
  void* a = nullptr;
  void* b = nullptr;
  cudaDriverEntryPointQueryResult qa{}, qb{};
  if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) != cudaSuccess ||
      qa != cudaDriverEntryPointSuccess || !a)
    return false;
  if (cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) != cudaSuccess ||
      qb != cudaDriverEntryPointSuccess || !b)
    return false;
  g_ctx_current = reinterpret_cast<CtxGetCurrentFn>(a);
  g_ctx_id = reinterpret_cast<CtxGetIdFn>(b);
  return true;
}

// The host-side symbol is only a stand-in for the array: its device address
// is looked up with the device current, once per CUDA context.
bbt_status scratch_address(int dev, double** out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (dev < 0 || dev >= MAX_DEVICES) return BBT_ERR_ARG;
  if (!driver_entries()) {
    fprintf(stderr, "bbt_twisted_vectors_noalloc: the driver's context queries are unavailable\n");
    return BBT_ERR_CUDA;
  }
  CUcontext cu = nullptr;
  unsigned long long id = 0;
  if (g_ctx_current(&cu) != CUDA_SUCCESS || !cu || g_ctx_id(cu, &id) != CUDA_SUCCESS || id == 0) {
    fprintf(stderr, "bbt_twisted_vectors_noalloc: no current CUDA context on device %d\n", dev);
    return BBT_ERR_CUDA;
  }
  Cached& c = g_addr[dev];
  if (c.ctx_id != id || !c.addr) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      fprintf(stderr, "bbt_twisted_vectors_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
      return BBT_ERR_CUDA;
    }
    c.addr = static_cast<double*>(p);
    c.ctx_id = id;
  }
  *out = c.addr;
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
            "%u-byte static array (2n + 6(n+1)cnt + n cnt doubles, each array rounded up to 256 bytes)\n",
            n, cnt, need, BBT_NOALLOC_SCRATCH_BYTES);
    return BBT_ERR_ARG;
  }
  if (cnt == 0) return BBT_OK;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return BBT_ERR_CUDA;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int sdev = -1;   // the array (and its address) belong to the current device: the stream must too
  if (cudaStreamGetDevice(st, &sdev) != cudaSuccess) return BBT_ERR_CUDA;
  if (sdev != dev) {
    fprintf(stderr, "bbt_twisted_vectors_noalloc: the stream belongs to device %d, the current device is %d\n",
            sdev, dev);
    return BBT_ERR_ARG;
  }
  double* scratch = nullptr;
  bbt_status s = scratch_address(dev, &scratch);
  if (s != BBT_OK) return s;
  bbt_ctx ctx;   // stack context: the caller's stream, no workspace, nothing allocated
  ctx.device = dev;
  ctx.stream = st;
  return bbt::twisted_scratch(&ctx, n, cnt, d_sigma, d_alpha, d_beta, d_U, cnt, d_V, scratch);
}
