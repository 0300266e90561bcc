// Small layout kernels shared by the pipeline.
#include <cuda_runtime.h>

#include <cstdlib>

#include "internal.h"

namespace bbt {

// Scratch cap of the passes over a long dimension.  EXCALIBUR_B200_CHUNK_BYTES
// (bytes, read at every call) overrides the default, e.g. to bound the
// workspace further on a device shared with other work.
size_t long_chunk_bytes(size_t dflt) {
  const char* v = std::getenv("EXCALIBUR_B200_CHUNK_BYTES");
  if (!v || !*v) return dflt;
  char* end = nullptr;
  const unsigned long long b = std::strtoull(v, &end, 10);
  return (end && *end == 0 && b >= ((size_t)1 << 20)) ? (size_t)b : dflt;
}

namespace {

// dst (cols x rows, row-major, ld ldd) = src^T, src rows x cols row-major (ld lds).
__global__ void transpose_kernel(int rows, int cols, const double* __restrict__ src, long lds,
                                 double* __restrict__ dst, long ldd) {
  __shared__ double t[32][33];
  const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int r = r0 + y, c = c0 + threadIdx.x;
    if (r < rows && c < cols) t[y][threadIdx.x] = src[(long)r * lds + c];
  }
  __syncthreads();
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int c = c0 + y, r = r0 + threadIdx.x;
    if (r < rows && c < cols) dst[(long)c * ldd + r] = t[threadIdx.x][y];
  }
}

__global__ void copy2d_kernel(int rows, int cols, const double* __restrict__ src, long lds,
                              double* __restrict__ dst, long ldd) {
  const long total = (long)rows * cols;
  for (long f = blockIdx.x * (long)blockDim.x + threadIdx.x; f < total; f += (long)gridDim.x * blockDim.x) {
    const long r = f / cols;
    const int c = (int)(f % cols);
    dst[r * ldd + c] = src[r * lds + c];
  }
}

// RT (m x m row-major, lower) = R^T, R the upper triangle in the top of
// column-major A (lda).
__global__ void rt_kernel(int m, const double* __restrict__ A, long lda, double* __restrict__ RT) {
  const long total = (long)m * m;
  for (long f = blockIdx.x * (long)blockDim.x + threadIdx.x; f < total; f += (long)gridDim.x * blockDim.x) {
    const int i = (int)(f / m), j = (int)(f % m);
    RT[f] = (j <= i) ? A[j + (long)i * lda] : 0.0;
  }
}

__global__ void fill_kernel(double* __restrict__ p, size_t n, double v) {
  for (size_t f = blockIdx.x * (size_t)blockDim.x + threadIdx.x; f < n; f += (size_t)gridDim.x * blockDim.x)
    p[f] = v;
}

}  // namespace

bbt_status transpose(bbt_ctx* ctx, int rows, int cols, const double* src, long lds, double* dst,
                     long ldd) {
  if (rows <= 0 || cols <= 0) return BBT_OK;
  dim3 b(32, 8), g((cols + 31) / 32, (rows + 31) / 32);
  transpose_kernel<<<g, b, 0, ctx->stream>>>(rows, cols, src, lds, dst, ldd);
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

bbt_status copy2d(bbt_ctx* ctx, int rows, int cols, const double* src, long lds, double* dst,
                  long ldd) {
  if (rows <= 0 || cols <= 0) return BBT_OK;
  copy2d_kernel<<<4 * ctx->num_sms, 256, 0, ctx->stream>>>(rows, cols, src, lds, dst, ldd);
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

bbt_status r_transpose(bbt_ctx* ctx, int m, const double* A, long lda, double* RT) {
  rt_kernel<<<4 * ctx->num_sms, 256, 0, ctx->stream>>>(m, A, lda, RT);
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

bbt_status fill(bbt_ctx* ctx, double* p, size_t n, double v) {
  if (n == 0) return BBT_OK;
  fill_kernel<<<4 * ctx->num_sms, 256, 0, ctx->stream>>>(p, n, v);
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

}  // namespace bbt
