// Singular vectors inside clusters of singular values.
//
// The twisted factorisation (bbtsvd.cpp:54-147) computes each singular
// vector on its own; inside a cluster whose relative gaps are far below
// 1e-8 the individual vectors are ill-posed, and the reference's vectors
// lose orthogonality completely (they collapse onto each other).  The
// cluster's invariant subspace, however, is well separated from the rest
// of the spectrum.  For every cluster this kernel (one CTA per cluster)
// takes the twisted vectors as a starting block and
//   1. orthonormalises them (modified Gram-Schmidt, twice),
//   2. runs two steps of block inverse iteration with B^T B - mu^2 I, mu the
//      cluster's middle value, through the differential stationary qd
//      transform (dstqds) of the exact factorisation B^T B = L D L^T
//      (D_i = a_i^2, L_i = b_i / a_i: no cancellation, so small singular
//      values keep their relative accuracy), re-orthonormalising after each,
//   3. forms u_j = B v_j / sigma_j and orthonormalises the u's,
//   4. applies the reference's sign convention (largest |u| entry positive,
//      client.cpp:988-995).
// Singular values are the bisection's, untouched.  Clusters are runs of
// consecutive values whose relative spacing is below CLUSTER_RELGAP; other
// vectors are left as the twisted factorisation produced them.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "internal.h"

namespace bbt {
namespace {

constexpr int CT = 256;
constexpr int CW = CT / 32;
constexpr double CLUSTER_RELGAP = 1e-7;

__device__ double csum(double v, double* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double s = 0.0;
  for (int k = 0; k < CW; ++k) s += sh[k];
  __syncthreads();
  return s;
}

// Modified Gram-Schmidt, two sweeps, on p rows of length n (row stride n).
__device__ void mgs2(double* Y, int p, int n, double* sh) {
  for (int sweep = 0; sweep < 2; ++sweep)
    for (int j = 0; j < p; ++j) {
      double* yj = Y + (long)j * n;
      for (int i = 0; i < j; ++i) {
        const double* yi = Y + (long)i * n;
        double s = 0.0;
        for (int t = threadIdx.x; t < n; t += CT) s += yi[t] * yj[t];
        s = csum(s, sh);
        for (int t = threadIdx.x; t < n; t += CT) yj[t] -= s * yi[t];
        __syncthreads();
      }
      double s = 0.0;
      for (int t = threadIdx.x; t < n; t += CT) s += yj[t] * yj[t];
      s = csum(s, sh);
      const double inv = s > 0.0 ? 1.0 / sqrt(s) : 0.0;
      for (int t = threadIdx.x; t < n; t += CT) yj[t] *= inv;
      __syncthreads();
    }
}

__global__ void __launch_bounds__(CT)
cluster_kernel(int n, int k, const double* __restrict__ a, const double* __restrict__ b,
               const double* __restrict__ sigma, const int2* __restrict__ ranges, double* __restrict__ U,
               double* __restrict__ V, double* __restrict__ scratch) {
  __shared__ double sh[CW];
  const int2 rg = ranges[blockIdx.x];
  const int s0 = rg.x, p = rg.y - rg.x;
  // scratch per cluster: Y (p x n), L+ (n), D+ (n) -- offsets by the cluster's first index
  double* Y = scratch + (long)s0 * n;
  double* Lp = scratch + (long)k * n + (long)blockIdx.x * 2 * n;
  double* Dp = Lp + n;
  // 1. start from the twisted v's (a vector the qd recurrences broke down on,
  //    inf/NaN, is replaced by a fixed pseudo-random one)
  for (int j = 0; j < p; ++j) {
    double bad = 0.0;
    for (int t = threadIdx.x; t < n; t += CT) {
      const double x = V[(long)(s0 + j) * n + t];
      Y[(long)j * n + t] = x;
      if (!isfinite(x)) bad = 1.0;
    }
    bad = csum(bad, sh);
    if (bad > 0.0)
      for (int t = threadIdx.x; t < n; t += CT) {
        unsigned h = (unsigned)(t + 1) * 2654435761u ^ (unsigned)(s0 + j + 1) * 40503u;
        h ^= h >> 13; h *= 0x5bd1e995u; h ^= h >> 15;
        Y[(long)j * n + t] = (double)(h & 0xffffff) / 16777216.0 - 0.5;
      }
    __syncthreads();
  }
  mgs2(Y, p, n, sh);
  // 2. dstqds of L D L^T - mu^2 I, D_i = a_i^2, L_i = b_i / a_i
  const double mu = sigma[s0 + p / 2];
  const double tau = mu * mu;
  if (threadIdx.x == 0) {
    double s = -tau;
    for (int i = 0; i + 1 < n; ++i) {
      const double Di = a[i] * a[i], Li = b[i] / a[i];
      double dp = Di + s;
      if (fabs(dp) < 1e-300) dp = dp < 0 ? -1e-300 : 1e-300;
      Dp[i] = dp;
      const double lp = Di * Li / dp;
      Lp[i] = lp;
      s = lp * Li * s - tau;
    }
    double dp = a[n - 1] * a[n - 1] + s;
    if (fabs(dp) < 1e-300) dp = dp < 0 ? -1e-300 : 1e-300;
    Dp[n - 1] = dp;
  }
  __syncthreads();
  for (int it = 0; it < 2; ++it) {
    // solve (L+ D+ L+^T) y = x for each of the p columns: one thread per column
    for (int j = threadIdx.x; j < p; j += CT) {
      double* y = Y + (long)j * n;
      double z = y[0];
      y[0] = z;
      for (int i = 0; i + 1 < n; ++i) {   // forward: L+ z = x
        z = y[i + 1] - Lp[i] * z;
        y[i + 1] = z;
      }
      for (int i = 0; i < n; ++i) y[i] /= Dp[i];
      double w = y[n - 1];
      for (int i = n - 2; i >= 0; --i) {  // backward: L+^T y = z / D+
        w = y[i] - Lp[i] * w;
        y[i] = w;
      }
    }
    __syncthreads();
    mgs2(Y, p, n, sh);
  }
  // 3. v_j <- Y_j; u_j = B v_j / sigma_j, orthonormalised (reuse Y for the u's
  //    after writing the v's back)
  for (int j = 0; j < p; ++j)
    for (int t = threadIdx.x; t < n; t += CT) V[(long)(s0 + j) * n + t] = Y[(long)j * n + t];
  __syncthreads();
  for (int j = 0; j < p; ++j) {
    const double* v = V + (long)(s0 + j) * n;
    const double inv = 1.0 / sigma[s0 + j];
    for (int t = threadIdx.x; t < n; t += CT)
      Y[(long)j * n + t] = (a[t] * v[t] + (t + 1 < n ? b[t] * v[t + 1] : 0.0)) * inv;
  }
  __syncthreads();
  mgs2(Y, p, n, sh);
  // 4. sign convention, write u back (column s0+j of U, n x k row-major)
  for (int j = 0; j < p; ++j) {
    double* y = Y + (long)j * n;
    // first index of the largest |u|: block argmax
    double best = -1.0;
    int bi = 0;
    for (int t = threadIdx.x; t < n; t += CT) {
      const double v = fabs(y[t]);
      if (v > best) { best = v; bi = t; }
    }
    __shared__ double bv[CT];
    __shared__ int bx[CT];
    bv[threadIdx.x] = best;
    bx[threadIdx.x] = bi;
    __syncthreads();
    for (int o = CT / 2; o > 0; o >>= 1) {
      if (threadIdx.x < o) {
        const double v2 = bv[threadIdx.x + o];
        const int i2 = bx[threadIdx.x + o];
        if (v2 > bv[threadIdx.x] || (v2 == bv[threadIdx.x] && i2 < bx[threadIdx.x])) {
          bv[threadIdx.x] = v2;
          bx[threadIdx.x] = i2;
        }
      }
      __syncthreads();
    }
    const double sg = y[bx[0]] < 0 ? -1.0 : 1.0;
    __syncthreads();
    for (int t = threadIdx.x; t < n; t += CT) U[(long)t * k + s0 + j] = sg * y[t];
    if (sg < 0)
      for (int t = threadIdx.x; t < n; t += CT) V[(long)(s0 + j) * n + t] = -V[(long)(s0 + j) * n + t];
    __syncthreads();
  }
}

}  // namespace

bbt_status refine_clusters(bbt_ctx* ctx, int n, int k, const double* a, const double* b, const double* sigma,
                           double* U, double* V, int* nclusters) {
  *nclusters = 0;
  if (k < 2) return BBT_OK;
  std::vector<double> hs(k);
  BBT_CUDA(ctx, cudaMemcpyAsync(hs.data(), sigma, k * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  BBT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  std::vector<int2> rg;
  for (int i = 0; i < k;) {
    int j = i + 1;
    while (j < k && (hs[j - 1] - hs[j]) < CLUSTER_RELGAP * hs[j - 1]) ++j;
    if (j - i >= 2) rg.push_back(make_int2(i, j));
    i = j;
  }
  if (rg.empty()) return BBT_OK;
  size_t mark = ctx->ws.top;
  int2* dr = ctx->ws.take<int2>(rg.size());
  double* scratch = ctx->ws.take<double>((size_t)k * n + rg.size() * 2 * (size_t)n);
  if (!scratch) return fail(ctx, BBT_ERR_NOMEM, "clusters: workspace");
  BBT_CUDA(ctx, cudaMemcpyAsync(dr, rg.data(), rg.size() * sizeof(int2), cudaMemcpyHostToDevice, ctx->stream));
  {
    ProfScope prof(ctx, BBT_PROF_TWISTED, 0.0);
    cluster_kernel<<<(unsigned)rg.size(), CT, 0, ctx->stream>>>(n, k, a, b, sigma, dr, U, V, scratch);
    BBT_LAUNCHED(ctx);
  }
  BBT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));   // rg (host) is used by the copy above
  ctx->ws.top = mark;
  *nclusters = (int)rg.size();
  return BBT_OK;
}

}  // namespace bbt
