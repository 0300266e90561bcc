// Twisted-factorisation singular vectors and the bidiagonal SVD driver.
//
// Excalibur src/bbtsvd.cpp:54-147 computes, per singular value w, a
// stationary (dstqds) and a progressive (dpqds) qd transform of the
// LDL^T factorisation of B^T B - w^2 I, twists at argmin |gamma|, solves for
// v, couples the factorisation over to B B^T - w^2 I and solves for u.
// Each singular value is an independent O(n) recurrence, so one thread owns
// one singular value.  The recurrences' work arrays are laid out
// interleaved, element i of every thread's array contiguous
// ([i][thread]), so a warp's loads and stores are coalesced; u lands
// directly in U (n x cnt row-major, the reference's layout) and v goes
// through the same interleaved layout and a tiled transpose into V.
//
// As in sturm.cu every operation is rounded separately (no FMA) in the
// reference's order, and the 2-norm is the scaled sum of squares, so results
// match the oracle bit for bit and the reference to rounding of its BLAS
// dnrm2.
#include <cuda_runtime.h>

#include "internal.h"

namespace bbt {
namespace {

#define MUL __dmul_rn
#define DIV __ddiv_rn
#define ADD __dadd_rn
#define SUB __dsub_rn

// LDL^T of B^T B, bbtsvd.cpp:54-63 (one thread: an O(n) recurrence).
__global__ void ldl_kernel(int n, const double* __restrict__ a, const double* __restrict__ b,
                           double* __restrict__ L, double* __restrict__ D) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  D[0] = MUL(a[0], a[0]);
  for (int i = 1; i < n; ++i) {
    const double ab = MUL(a[i - 1], b[i - 1]);
    L[i - 1] = DIV(ab, D[i - 1]);
    D[i] = SUB(ADD(MUL(a[i], a[i]), MUL(b[i - 1], b[i - 1])), DIV(MUL(ab, ab), D[i - 1]));
  }
}

// Scaled sum-of-squares 2-norm in ascending index order (the oracle's norm).
struct Nrm {
  double scale = 0.0, ssq = 1.0;
  __device__ __forceinline__ void add(double x) {
    const double v = fabs(x);
    if (v != 0.0) {
      if (scale < v) {
        const double r = DIV(scale, v);
        ssq = ADD(1.0, MUL(MUL(ssq, r), r));
        scale = v;
      } else {
        const double r = DIV(v, scale);
        ssq = ADD(ssq, MUL(r, r));
      }
    }
  }
  __device__ __forceinline__ double get() const { return MUL(scale, sqrt(ssq)); }
};

// x[k] = 1, backward with lo, forward with up, normalise.  x has stride ld.
// Returns the first index of max |x_i| after scaling.  Every loop reads its
// operands PF elements ahead into registers (the recurrences depend only on
// the previous value, not on the loads), so the L2 latency of the work arrays
// is paid once per PF elements; the arithmetic and its order are unchanged.
constexpr int PF = 8;

__device__ int twisted_solve(int n, int k, const double* lo, const double* up, long ldw, double* x,
                             long ld) {
  x[(long)k * ld] = 1.0;
  double prev = 1.0;
  for (int i0 = k - 1; i0 >= 0; i0 -= PF) {
    double v[PF];
#pragma unroll
    for (int u = 0; u < PF; ++u) v[u] = (i0 - u >= 0) ? lo[(long)(i0 - u) * ldw] : 0.0;
#pragma unroll
    for (int u = 0; u < PF; ++u)
      if (i0 - u >= 0) {
        prev = MUL(-v[u], prev);
        x[(long)(i0 - u) * ld] = prev;
      }
  }
  prev = 1.0;
  for (int i0 = k + 1; i0 < n; i0 += PF) {
    double v[PF];
#pragma unroll
    for (int u = 0; u < PF; ++u) v[u] = (i0 + u < n) ? up[(long)(i0 + u - 1) * ldw] : 0.0;
#pragma unroll
    for (int u = 0; u < PF; ++u)
      if (i0 + u < n) {
        prev = MUL(-v[u], prev);
        x[(long)(i0 + u) * ld] = prev;
      }
  }
  Nrm nr;
  for (int i0 = 0; i0 < n; i0 += PF) {
    double v[PF];
#pragma unroll
    for (int u = 0; u < PF; ++u) v[u] = (i0 + u < n) ? x[(long)(i0 + u) * ld] : 0.0;
#pragma unroll
    for (int u = 0; u < PF; ++u)
      if (i0 + u < n) nr.add(v[u]);
  }
  const double r = DIV(1.0, nr.get());
  int best = 0;
  double bv = 0.0;
  for (int i0 = 0; i0 < n; i0 += PF) {
    double v[PF];
#pragma unroll
    for (int u = 0; u < PF; ++u) v[u] = (i0 + u < n) ? x[(long)(i0 + u) * ld] : 0.0;
#pragma unroll
    for (int u = 0; u < PF; ++u)
      if (i0 + u < n) {
        const int i = i0 + u;
        const double vs = MUL(v[u], r);
        x[(long)i * ld] = vs;
        const double av = fabs(vs);
        if (i == 0 || av > bv) { bv = av; best = i; }   // first largest |x_i| (cblas_idamax)
      }
  }
  return best;
}

// One thread per singular value j (bbtsvd.cpp:93-135, then the v sign rule
// of :944-955 when sign_fix).  Work arrays are [i * cnt + j].
__global__ void __launch_bounds__(64) twisted_kernel(
    int n, int cnt, const double* __restrict__ sigma, const double* __restrict__ a,
    const double* __restrict__ b, const double* __restrict__ L, const double* __restrict__ D,
    double* __restrict__ S, double* __restrict__ Pp, double* __restrict__ DP, double* __restrict__ RP,
    double* __restrict__ LP, double* __restrict__ UP, double* __restrict__ Vt, double* __restrict__ U,
    int ldu, signed char* __restrict__ vsign, int sign_fix) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= cnt) return;
  const long w = cnt;   // interleave stride
  double* s = S + j;
  double* p = Pp + j;
  double* dp = DP + j;
  double* rp = RP + j;
  double* lp = LP + j;
  double* up = UP + j;
  const double om = sigma[j];
  const double w2 = MUL(om, om);
  // dstqds, bbtsvd.cpp:73-81
  double si = -w2;
  s[0] = si;
  for (int i = 0; i + 1 < n; ++i) {
    const double d = ADD(D[i], si);
    dp[(long)i * w] = d;
    const double l = DIV(MUL(D[i], L[i]), d);
    lp[(long)i * w] = l;
    si = SUB(MUL(MUL(l, L[i]), si), w2);
    s[(long)(i + 1) * w] = si;
  }
  dp[(long)(n - 1) * w] = ADD(D[n - 1], si);
  // dpqds, bbtsvd.cpp:83-91, with gamma (:107) and its argmin (:108)
  double pi = SUB(D[n - 1], w2);
  p[(long)(n - 1) * w] = pi;
  // first index of the smallest |gamma_i| in ascending order; a NaN
  // gamma_0 wins outright and other NaNs never do (the oracle's argmin)
  int k = n - 1;
  double gbest = fabs(ADD(ADD(s[(long)(n - 1) * w], pi), w2));
  double g0 = gbest;
  for (int i0 = n - 2; i0 >= 0; i0 -= PF) {
    double sv[PF];
#pragma unroll
    for (int u = 0; u < PF; ++u) sv[u] = (i0 - u >= 0) ? s[(long)(i0 - u) * w] : 0.0;
#pragma unroll
    for (int u = 0; u < PF; ++u) {
      const int i = i0 - u;
      if (i >= 0) {
        const double r = ADD(MUL(D[i], MUL(L[i], L[i])), pi);
        rp[(long)(i + 1) * w] = r;
        up[(long)i * w] = DIV(MUL(L[i], D[i]), r);
        pi = SUB(DIV(MUL(pi, D[i]), r), w2);
        p[(long)i * w] = pi;
        const double g = fabs(ADD(ADD(sv[u], pi), w2));
        if (g == g && (gbest != gbest || g <= gbest)) { gbest = g; k = i; }
        g0 = g;
      }
    }
  }
  if (g0 != g0) k = 0;
  rp[0] = pi;
  // v (:111)
  const int pv = twisted_solve(n, k, lp, up, w, Vt + j, w);
  // coupling (:114-124): s[n] = -w2, p[n] = 1, rp[n] = 1
  int k2 = 0;
  double g2best = 0.0;
  double dprev = 0.0;
  for (int i0 = 0; i0 < n; i0 += PF) {
    // s, p, rp at i0 .. i0 + PF (one past the batch), dp at i0 .. i0 + PF - 1
    double sv[PF + 1], pv2[PF + 1], rv[PF + 1], dv[PF];
#pragma unroll
    for (int u = 0; u <= PF; ++u) {
      const int i = i0 + u;
      sv[u] = (i < n) ? s[(long)i * w] : -w2;
      pv2[u] = (i < n) ? p[(long)i * w] : 1.0;
      rv[u] = (i < n) ? rp[(long)i * w] : 1.0;
      if (u < PF) dv[u] = (i < n) ? dp[(long)i * w] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < PF; ++u) {
    const int i = i0 + u;
    if (i >= n) break;
    const double s_i = sv[u];
    const double s_n = sv[u + 1];
    const double p_i = pv2[u];
    const double p_n = pv2[u + 1];
    const double r_n = rv[u + 1];
    const double d_new = MUL(DIV(s_n, s_i), dv[u]);
    const double g_old = ADD(ADD(s_i, p_i), w2);
    const double g_new = fabs(DIV(MUL(MUL(-w2, g_old), r_n), MUL(s_i, p_n)));
    if (i == 0 || g_new < g2best) { g2best = g_new; k2 = i; }
    const double r_new = MUL(DIV(p_i, p_n), r_n);
    if (i > 0) {
      lp[(long)(i - 1) * w] = MUL(DIV(a[i], dprev), b[i - 1]);
      up[(long)(i - 1) * w] = MUL(DIV(a[i], r_new), b[i - 1]);
    }
    dprev = d_new;
    }
  }
  // u (:126), column j of U
  twisted_solve(n, k2, lp, up, w, U + j, ldu);
  signed char sg = 1;
  if (sign_fix) {   // bbtsvd.cpp:944-955: align v with B^T u at v's largest entry
    const double vp = Vt[(long)pv * w + j];
    double sgn;
    if (pv == 0) sgn = DIV(MUL(U[j], a[0]), om);
    else sgn = DIV(ADD(MUL(U[(long)(pv - 1) * ldu + j], b[pv - 1]), MUL(U[(long)pv * ldu + j], a[pv])), om);
    if (MUL(sgn, vp) < 0) sg = -1;
  }
  vsign[j] = sg;
}

// V (cnt x n) = sign_j * Vt^T, Vt interleaved (n x cnt).
__global__ void vtranspose_kernel(int n, int cnt, const double* __restrict__ Vt,
                                  const signed char* __restrict__ vsign, double* __restrict__ V) {
  __shared__ double tile[32][33];
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = i0 + r, j = j0 + threadIdx.x;
    if (i < n && j < cnt) tile[r][threadIdx.x] = Vt[(long)i * cnt + j];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int j = j0 + r, i = i0 + threadIdx.x;
    if (i < n && j < cnt) {
      const double v = tile[threadIdx.x][r];
      V[(long)j * n + i] = vsign[j] < 0 ? -v : v;
    }
  }
}

// bbtsvd.cpp:957-967: a value equal (to 1e-15) to alpha_i gets unit vectors.
__global__ void check_none_kernel(int k, int top_k, const double* __restrict__ sigma,
                                  const double* __restrict__ a, double* __restrict__ U,
                                  double* __restrict__ V) {
  const int i = blockIdx.x;
  if (i >= top_k) return;
  if (!(fabs(SUB(sigma[i], a[i])) < 1e-15)) return;
  for (int j = threadIdx.x; j < k; j += blockDim.x) {
    if (j == i) U[(long)i * top_k + i] = 1.0;
    if (j > i && j < top_k) U[(long)i * top_k + j] = 0.0;
    if (j > i) U[(long)j * top_k + i] = 0.0;
    V[(long)i * k + j] = (j == i) ? 1.0 : 0.0;
  }
}

// client.cpp:988-995: make the largest |entry| of each u positive, flipping
// u and v together.  One thread per column of U (k x cnt row-major).
// client.cpp:987-995: each column of U (k x cnt, row-major) made positive at
// its first largest |entry|, the matching row of V (cnt x k) flipped with it.
// One thread per column finds the entry (loads read PF rows ahead) and flips
// U's column, coalesced across the warp; the rows of V are flipped by
// vflip_kernel, coalesced along each row.
__global__ void global_sign_kernel(int k, int cnt, double* __restrict__ U, signed char* __restrict__ flip) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= cnt) return;
  int best = 0;
  double bv = fabs(U[j]);
  for (int i0 = 1; i0 < k; i0 += PF) {
    double v[PF];
#pragma unroll
    for (int u = 0; u < PF; ++u) v[u] = (i0 + u < k) ? fabs(U[(long)(i0 + u) * cnt + j]) : 0.0;
#pragma unroll
    for (int u = 0; u < PF; ++u)
      if (i0 + u < k && v[u] > bv) { bv = v[u]; best = i0 + u; }
  }
  const bool neg = U[(long)best * cnt + j] < 0;
  flip[j] = neg ? 1 : 0;
  if (neg)
    for (int i = 0; i < k; ++i) U[(long)i * cnt + j] = -U[(long)i * cnt + j];
}

__global__ void vflip_kernel(int k, int cnt, const signed char* __restrict__ flip, double* __restrict__ V) {
  const long total = (long)k * cnt;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x)
    if (flip[e / k]) V[e] = -V[e];
}

// ||a||^2 + ||b||^2 with the scaled norm (bbtsvd.cpp:936), one thread.
__global__ void bound_kernel(int n, const double* __restrict__ a, const double* __restrict__ b,
                             double* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  Nrm na, nb;
  for (int i = 0; i < n; ++i) na.add(a[i]);
  for (int i = 0; i + 1 < n; ++i) nb.add(b[i]);
  const double x = na.get(), y = nb.get();
  out[0] = ADD(MUL(x, x), MUL(y, y));
}

// bbtsvd.cpp:65-71 (inverse_iteration) on one vector: twisted_solve.
__global__ void inverse_iteration_kernel(int n, int k, const double* __restrict__ l, const double* __restrict__ u,
                                         double* __restrict__ v, long ldv) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  twisted_solve(n, k, l, u, 1, v, ldv);
}

}  // namespace

// The reference's per-step helpers on device arrays (the bbtsvd.hpp entry
// points of the compatibility layer): LDL^T of B^T B, one inverse
// iteration, and one singular pair by the twisted factorisation (no sign
// rule: bbtsvd.cpp:93-136 leaves it to the driver).
bbt_status ldl_factor(bbt_ctx* ctx, int n, const double* a, const double* b, double* L, double* D) {
  ldl_kernel<<<1, 1, 0, ctx->stream>>>(n, a, b, L, D);
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

bbt_status inverse_iteration_dev(bbt_ctx* ctx, int n, int k, const double* l, const double* u, double* v, long ldv) {
  if (n < 1 || k < 0 || k >= n) return fail(ctx, BBT_ERR_ARG, "inverse iteration: n=%d k=%d", n, k);
  inverse_iteration_kernel<<<1, 1, 0, ctx->stream>>>(n, k, l, u, v, ldv);
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

size_t twisted_pair_scratch_doubles(int n) { return 6 * ((size_t)n + 1) + 1; }

bbt_status twisted_pair(bbt_ctx* ctx, int n, const double* omega, const double* L, const double* D, const double* a,
                        const double* b, double* v, double* u, int ldu, double* scratch) {
  if (n < 1) return fail(ctx, BBT_ERR_ARG, "twisted pair: n=%d", n);
  const size_t c = (size_t)n + 1;
  double* p = scratch;
  twisted_kernel<<<1, 32, 0, ctx->stream>>>(n, 1, omega, a, b, L, D, p, p + c, p + 2 * c, p + 3 * c, p + 4 * c,
                                            p + 5 * c, v, u, ldu, reinterpret_cast<signed char*>(p + 6 * c), 0);
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

bbt_status twisted(bbt_ctx* ctx, int n, int cnt, const double* sigma, const double* a,
                   const double* b, double* U, int ldu, double* V, bool sign_fix) {
  if (n < 1 || cnt < 0 || cnt > n) return fail(ctx, BBT_ERR_ARG, "twisted: n=%d cnt=%d", n, cnt);
  if (cnt == 0) return BBT_OK;
  size_t mark = ctx->ws.top;
  const size_t col = (size_t)(n + 1) * cnt;
  double* L = ctx->ws.take<double>(n);
  double* D = ctx->ws.take<double>(n);
  double* S = ctx->ws.take<double>(col);
  double* P = ctx->ws.take<double>(col);
  double* DP = ctx->ws.take<double>(col);
  double* RP = ctx->ws.take<double>(col);
  double* LP = ctx->ws.take<double>(col);
  double* UPa = ctx->ws.take<double>(col);
  double* Vt = ctx->ws.take<double>((size_t)n * cnt);
  signed char* vs = ctx->ws.take<signed char>(cnt);
  if (!vs)
    return fail(ctx, BBT_ERR_NOMEM, "twisted: workspace (%zu MB)",
                ((2 * (size_t)n + 6 * col + (size_t)n * cnt) * 8 + cnt) >> 20);
  ProfScope prof(ctx, BBT_PROF_TWISTED, 0.0);
  ldl_kernel<<<1, 1, 0, ctx->stream>>>(n, a, b, L, D);
  BBT_LAUNCHED(ctx);
  twisted_kernel<<<(cnt + 31) / 32, 32, 0, ctx->stream>>>(n, cnt, sigma, a, b, L, D, S, P, DP, RP, LP,
                                                         UPa, Vt, U, ldu, vs, sign_fix ? 1 : 0);
  BBT_LAUNCHED(ctx);
  dim3 tb(32, 8), tg((n + 31) / 32, (cnt + 31) / 32);
  vtranspose_kernel<<<tg, tb, 0, ctx->stream>>>(n, cnt, Vt, vs, V);
  BBT_LAUNCHED(ctx);
  ctx->ws.top = mark;
  return BBT_OK;
}

// Same kernels as twisted(), with every work array carved from a caller-
// provided device scratch region instead of the context's workspace.  The
// scratch needs scratch_doubles_twisted(n, cnt) doubles; each array is
// written before it is read, so the region's previous contents are never
// observed.
size_t scratch_doubles_twisted(int n, int cnt) {
  const size_t col = (size_t)(n + 1) * cnt;
  auto up = [](size_t d) { return (d + 31) & ~size_t(31); };   // 256-byte steps
  return up(n) * 2 + up(col) * 6 + up((size_t)n * cnt) + up((cnt + 7) / 8);
}

bbt_status twisted_scratch(bbt_ctx* ctx, int n, int cnt, const double* sigma, const double* a,
                           const double* b, double* U, int ldu, double* V, double* scratch) {
  if (n < 1 || cnt < 0 || cnt > n) return fail(ctx, BBT_ERR_ARG, "twisted: n=%d cnt=%d", n, cnt);
  if (cnt == 0) return BBT_OK;
  const size_t col = (size_t)(n + 1) * cnt;
  auto up = [](size_t d) { return (d + 31) & ~size_t(31); };
  double* p = scratch;
  double* L = p; p += up(n);
  double* D = p; p += up(n);
  double* S = p; p += up(col);
  double* P = p; p += up(col);
  double* DP = p; p += up(col);
  double* RP = p; p += up(col);
  double* LP = p; p += up(col);
  double* UPa = p; p += up(col);
  double* Vt = p; p += up((size_t)n * cnt);
  signed char* vs = reinterpret_cast<signed char*>(p);
  ldl_kernel<<<1, 1, 0, ctx->stream>>>(n, a, b, L, D);
  BBT_LAUNCHED(ctx);
  twisted_kernel<<<(cnt + 31) / 32, 32, 0, ctx->stream>>>(n, cnt, sigma, a, b, L, D, S, P, DP, RP, LP,
                                                         UPa, Vt, U, ldu, vs, 0);
  BBT_LAUNCHED(ctx);
  dim3 tb(32, 8), tg((n + 31) / 32, (cnt + 31) / 32);
  vtranspose_kernel<<<tg, tb, 0, ctx->stream>>>(n, cnt, Vt, vs, V);
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

bbt_status bidiag_bound(bbt_ctx* ctx, int n, const double* a, const double* b, double* out) {
  bound_kernel<<<1, 1, 0, ctx->stream>>>(n, a, b, out);
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

bbt_status bidiag_svd(bbt_ctx* ctx, int k, const double* a, const double* b, double* U, double* V,
                      double* sigma, int top_k, bool global_sign) {
  if (k < 1 || top_k < 1 || top_k > k) return fail(ctx, BBT_ERR_ARG, "bidiagonal svd: k=%d top_k=%d", k, top_k);
  size_t mark = ctx->ws.top;
  double* bound = ctx->ws.take<double>(1);
  if (!bound) return fail(ctx, BBT_ERR_NOMEM, "bidiagonal svd: workspace");
  bound_kernel<<<1, 1, 0, ctx->stream>>>(k, a, b, bound);
  BBT_LAUNCHED(ctx);
  double hb = 0;
  BBT_CUDA(ctx, cudaMemcpyAsync(&hb, bound, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  BBT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  int cnt = 0;
  double* br = nullptr;
  if (ctx->bracket_theta) {   // learned brackets (verified inside bisect; never change the result)
    br = ctx->ws.take<double>(2 * (size_t)top_k);
    if (!br) return fail(ctx, BBT_ERR_NOMEM, "bidiagonal svd: bracket workspace");
    BBT_TRY(mlp_brackets(ctx, k, top_k, a, b, ctx->bracket_theta, ctx->bracket_z, br));
  }
  BBT_TRY(bisect(ctx, k, a, b, 0.0, hb, 1e-20, top_k, sigma, &cnt, br, ctx->bisect_stats));
  if (cnt < top_k) {
    ctx->ws.top = mark;
    return fail(ctx, BBT_ERR_COUNT, "bisection found %d singular values, %d requested", cnt, top_k);
  }
  BBT_TRY(twisted(ctx, k, top_k, sigma, a, b, U, top_k, V, true));
  check_none_kernel<<<top_k, 128, 0, ctx->stream>>>(k, top_k, sigma, a, U, V);
  BBT_LAUNCHED(ctx);
  if (global_sign) {
    signed char* flip = ctx->ws.take<signed char>(top_k);
    if (!flip) return fail(ctx, BBT_ERR_NOMEM, "bidiagonal svd: sign workspace");
    global_sign_kernel<<<(top_k + 63) / 64, 64, 0, ctx->stream>>>(k, top_k, U, flip);
    BBT_LAUNCHED(ctx);
    vflip_kernel<<<2 * ctx->num_sms, 256, 0, ctx->stream>>>(k, top_k, flip, V);
    BBT_LAUNCHED(ctx);
  }
  ctx->ws.top = mark;
  return BBT_OK;
}

}  // namespace bbt
