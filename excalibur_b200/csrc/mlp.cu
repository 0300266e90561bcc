// Learned bisection brackets: a small MLP trained and evaluated by this
// library's own kernels.
//
// Model: x (F = 10 features) -> tanh(W1 x + b1) (H = 32) -> tanh(W2 h1 + b2)
// (H) -> (mu, ell) = W3 h2 + b3.  For the j-th largest singular value of a
// bidiagonal, mu predicts log2(sigma_j / g) with g the Gershgorin-type bound
// max_i (|a_i| + max(|b_{i-1}|, |b_i|)) >= sigma_max, and exp(ell) is the
// predicted spread of that estimate (log2 units).  Training minimises the
// Gaussian negative log-likelihood 0.5 ((y - mu) e^-ell)^2 + ell with Adam.
// Parameters are one flat FP64 vector: W1 (H x F, row-major), b1, W2 (H x H),
// b2, W3 (2 x H), b3.
//
// Features of (a, b, j) (all log2 ratios to g, clipped to [-64, 16] and
// divided by 16): ||a||_2, ||b||_2, max|a|, max|b|, min|a|; then log2(k)/16,
// t = (j + 1/2) / k, t^2, sqrt(t), log2(t) / 16.
//
// The brackets never change an answer: sturm.cu snaps each one to a node of
// the reference's bisection tree, verifies it with exact Sturm counts and
// only then lets the bisection skip to it.
#include <cuda_runtime.h>

#include "internal.h"

namespace bbt {
namespace {

constexpr int F = MLP_FEATURES, H = MLP_HIDDEN;
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + H * F, OFF_W2 = OFF_B1 + H, OFF_B2 = OFF_W2 + H * H,
              OFF_W3 = OFF_B2 + H, OFF_B3 = OFF_W3 + 2 * H, NPARAM = OFF_B3 + 2;
static_assert(NPARAM == MLP_PARAMS, "parameter layout");

__device__ __forceinline__ double clip_log(double r) {   // log2 of a ratio, clipped to [-64, 16], scaled
  const double l = r > 0.0 ? log2(r) : -64.0;
  return fmin(16.0, fmax(-64.0, l)) / 16.0;
}

// Per-bidiagonal summary (one block): s[0..5] = ||a||, ||b||, max|a|, max|b|, min|a|, g.
__global__ void summary_kernel(int k, const double* __restrict__ a, const double* __restrict__ b,
                               double* __restrict__ s) {
  __shared__ double sh[6][256];
  double sa = 0, sb = 0, ma = 0, mb = 0, mn = 1e300, g = 0;
  for (int i = threadIdx.x; i < k; i += blockDim.x) {
    const double ai = fabs(a[i]);
    const double bl = i > 0 ? fabs(b[i - 1]) : 0.0, br = i + 1 < k ? fabs(b[i]) : 0.0;
    sa += ai * ai;
    ma = fmax(ma, ai);
    mn = fmin(mn, ai);
    if (i + 1 < k) { sb += br * br; mb = fmax(mb, br); }
    g = fmax(g, ai + fmax(bl, br));
  }
  sh[0][threadIdx.x] = sa; sh[1][threadIdx.x] = sb; sh[2][threadIdx.x] = ma;
  sh[3][threadIdx.x] = mb; sh[4][threadIdx.x] = mn; sh[5][threadIdx.x] = g;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      sh[0][threadIdx.x] += sh[0][threadIdx.x + o];
      sh[1][threadIdx.x] += sh[1][threadIdx.x + o];
      sh[2][threadIdx.x] = fmax(sh[2][threadIdx.x], sh[2][threadIdx.x + o]);
      sh[3][threadIdx.x] = fmax(sh[3][threadIdx.x], sh[3][threadIdx.x + o]);
      sh[4][threadIdx.x] = fmin(sh[4][threadIdx.x], sh[4][threadIdx.x + o]);
      sh[5][threadIdx.x] = fmax(sh[5][threadIdx.x], sh[5][threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    s[0] = sqrt(sh[0][0]); s[1] = sqrt(sh[1][0]); s[2] = sh[2][0];
    s[3] = sh[3][0]; s[4] = sh[4][0]; s[5] = sh[5][0];
  }
}

// X (count x F): features of indices j = 0 .. count-1 of a k x k bidiagonal.
__global__ void features_kernel(int k, int count, const double* __restrict__ s, double* __restrict__ X) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= count) return;
  const double g = s[5] > 0.0 ? s[5] : 1.0;
  const double t = (j + 0.5) / k;
  double* x = X + (long)j * F;
  x[0] = clip_log(s[0] / g);
  x[1] = clip_log(s[1] / g);
  x[2] = clip_log(s[2] / g);
  x[3] = clip_log(s[3] / g);
  x[4] = clip_log(s[4] / g);
  x[5] = log2((double)k) / 16.0;
  x[6] = t;
  x[7] = t * t;
  x[8] = sqrt(t);
  x[9] = log2(t) / 16.0;
}

// Forward pass of one sample; h1, h2 kept for the backward pass.
__device__ __forceinline__ void forward(const double* __restrict__ p, const double* __restrict__ x, double* h1,
                                        double* h2, double* out) {
#pragma unroll 4
  for (int u = 0; u < H; ++u) {
    double z = p[OFF_B1 + u];
#pragma unroll
    for (int f = 0; f < F; ++f) z += p[OFF_W1 + u * F + f] * x[f];
    h1[u] = tanh(z);
  }
#pragma unroll 4
  for (int u = 0; u < H; ++u) {
    double z = p[OFF_B2 + u];
    for (int v = 0; v < H; ++v) z += p[OFF_W2 + u * H + v] * h1[v];
    h2[u] = tanh(z);
  }
  for (int o = 0; o < 2; ++o) {
    double z = p[OFF_B3 + o];
    for (int v = 0; v < H; ++v) z += p[OFF_W3 + o * H + v] * h2[v];
    out[o] = z;
  }
}

__global__ void __launch_bounds__(128) forward_kernel(int B, const double* __restrict__ X,
                                                      const double* __restrict__ theta, double* __restrict__ out) {
  __shared__ double p[NPARAM];
  for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) p[i] = theta[i];
  __syncthreads();
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= B) return;
  double x[F], h1[H], h2[H], o[2];
#pragma unroll
  for (int f = 0; f < F; ++f) x[f] = X[(long)s * F + f];
  forward(p, x, h1, h2, o);
  out[2 * s] = o[0];
  out[2 * s + 1] = o[1];
}

// Per-sample loss and gradient: G[q][s] = d loss_s / d theta_q (theta-major,
// so the writes of a warp are contiguous), loss[s].
__global__ void __launch_bounds__(128) grad_kernel(int B, const double* __restrict__ X, const double* __restrict__ y,
                                                   const double* __restrict__ theta, double* __restrict__ G,
                                                   double* __restrict__ loss) {
  __shared__ double p[NPARAM];
  for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) p[i] = theta[i];
  __syncthreads();
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= B) return;
  double x[F], h1[H], h2[H], o[2];
#pragma unroll
  for (int f = 0; f < F; ++f) x[f] = X[(long)s * F + f];
  forward(p, x, h1, h2, o);
  const double r = y[s] - o[0];
  const double e2 = exp(-2.0 * o[1]);
  loss[s] = 0.5 * r * r * e2 + o[1];
  const double d3[2] = {-r * e2, 1.0 - r * r * e2};   // d loss / d (mu, ell)
  auto put = [&](int q, double v) { G[(long)q * B + s] = v; };
  for (int oo = 0; oo < 2; ++oo) {
    put(OFF_B3 + oo, d3[oo]);
    for (int v = 0; v < H; ++v) put(OFF_W3 + oo * H + v, d3[oo] * h2[v]);
  }
  double d2[H];
  for (int u = 0; u < H; ++u) {
    const double g = d3[0] * p[OFF_W3 + u] + d3[1] * p[OFF_W3 + H + u];
    d2[u] = g * (1.0 - h2[u] * h2[u]);
    put(OFF_B2 + u, d2[u]);
    for (int v = 0; v < H; ++v) put(OFF_W2 + u * H + v, d2[u] * h1[v]);
  }
  for (int v = 0; v < H; ++v) {
    double g = 0.0;
    for (int u = 0; u < H; ++u) g += d2[u] * p[OFF_W2 + u * H + v];
    const double d1 = g * (1.0 - h1[v] * h1[v]);
    put(OFF_B1 + v, d1);
#pragma unroll
    for (int f = 0; f < F; ++f) put(OFF_W1 + v * F + f, d1 * x[f]);
  }
}

// grad[q] = mean_s G[q][s] (one warp per parameter, fixed order); loss[0] = mean loss.
__global__ void reduce_kernel(int B, const double* __restrict__ G, const double* __restrict__ ls,
                              double* __restrict__ grad, double* __restrict__ loss) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w > NPARAM) return;
  const double* src = (w < NPARAM) ? G + (long)w * B : ls;
  double acc = 0.0;
  for (int s = lane; s < B; s += 32) acc += src[s];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) {
    if (w < NPARAM) grad[w] = acc / B;
    else loss[0] = acc / B;
  }
}

__global__ void adam_kernel(double* __restrict__ theta, const double* __restrict__ grad, double* __restrict__ m,
                            double* __restrict__ v, double lr, double b1, double b2, double eps, int t) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= NPARAM) return;
  const double g = grad[q];
  m[q] = b1 * m[q] + (1.0 - b1) * g;
  v[q] = b2 * v[q] + (1.0 - b2) * g * g;
  const double mh = m[q] / (1.0 - pow(b1, (double)t)), vh = v[q] / (1.0 - pow(b2, (double)t));
  theta[q] -= lr * mh / (sqrt(vh) + eps);
}

// Brackets [lo, hi] of sigma_j (descending j) from the model outputs.
__global__ void brackets_kernel(int count, const double* __restrict__ s, const double* __restrict__ out, double z,
                                double* __restrict__ br) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= count) return;
  const double g = s[5];
  const double mu = out[2 * j], w = z * exp(fmin(out[2 * j + 1], 8.0));
  br[2 * j] = g * exp2(mu - w);
  br[2 * j + 1] = g * exp2(mu + w);
}

}  // namespace

bbt_status mlp_summary(bbt_ctx* ctx, int k, const double* a, const double* b, double* s6) {
  summary_kernel<<<1, 256, 0, ctx->stream>>>(k, a, b, s6);
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

bbt_status mlp_features(bbt_ctx* ctx, int k, int count, const double* s6, double* X) {
  features_kernel<<<(count + 127) / 128, 128, 0, ctx->stream>>>(k, count, s6, X);
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

bbt_status mlp_forward(bbt_ctx* ctx, int B, const double* X, const double* theta, double* out) {
  if (B <= 0) return BBT_OK;
  forward_kernel<<<(B + 127) / 128, 128, 0, ctx->stream>>>(B, X, theta, out);
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

bbt_status mlp_grad(bbt_ctx* ctx, int B, const double* X, const double* y, const double* theta, double* grad,
                    double* loss) {
  if (B <= 0) return fail(ctx, BBT_ERR_ARG, "mlp_grad: empty batch");
  const size_t mark = ctx->ws.top;
  double* G = ctx->ws.take<double>((size_t)NPARAM * B);
  double* ls = ctx->ws.take<double>(B);
  if (!ls) return fail(ctx, BBT_ERR_NOMEM, "mlp_grad: workspace");
  grad_kernel<<<(B + 127) / 128, 128, 0, ctx->stream>>>(B, X, y, theta, G, ls);
  BBT_LAUNCHED(ctx);
  const int warps = NPARAM + 1;
  reduce_kernel<<<(warps * 32 + 255) / 256, 256, 0, ctx->stream>>>(B, G, ls, grad, loss);
  BBT_LAUNCHED(ctx);
  ctx->ws.top = mark;
  return BBT_OK;
}

bbt_status mlp_adam(bbt_ctx* ctx, double* theta, const double* grad, double* m, double* v, double lr, int t) {
  adam_kernel<<<(NPARAM + 127) / 128, 128, 0, ctx->stream>>>(theta, grad, m, v, lr, 0.9, 0.999, 1e-8, t);
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

bbt_status mlp_brackets(bbt_ctx* ctx, int k, int count, const double* a, const double* b, const double* theta,
                        double z, double* br) {
  const size_t mark = ctx->ws.top;
  double* s6 = ctx->ws.take<double>(8);
  double* X = ctx->ws.take<double>((size_t)count * F);
  double* out = ctx->ws.take<double>((size_t)count * 2);
  if (!out) return fail(ctx, BBT_ERR_NOMEM, "mlp_brackets: workspace");
  BBT_TRY(mlp_summary(ctx, k, a, b, s6));
  BBT_TRY(mlp_features(ctx, k, count, s6, X));
  BBT_TRY(mlp_forward(ctx, count, X, theta, out));
  brackets_kernel<<<(count + 127) / 128, 128, 0, ctx->stream>>>(count, s6, out, z, br);
  BBT_LAUNCHED(ctx);
  ctx->ws.top = mark;
  return BBT_OK;
}

}  // namespace bbt
