// Blocked Householder QR (LAPACK dgeqrf / dorgqr / dormqr semantics) for
// the reference's local and global QR (Excalibur src/client.cpp:417-445,
// 705-794) and for applying the Ralha reflectors (client.cpp:1176).
//
// Column-major A (rows x cols, lda), rows >= cols, panels of nb <= 32
// columns.  A panel is factored one column at a time by panel_step_kernel:
// one launch per column updates the panel with the previous column's
// reflector and, in the same pass over the rows, produces the partial dot
// products the next column's reflector needs, so each column costs a single
// read+write of the remaining panel.  Every CTA then sums the per-CTA
// partials itself in the same fixed order (deterministic, no atomics).  The
// reflectors of a panel are merged into compact-WY form I - V T V^T (T by
// the dlarft recurrence from V^T V) and applied to the trailing matrix with
// three DMMA GEMMs: W = V^T C, W = T^T W, C -= V W.
#include <cuda_runtime.h>

#include "internal.h"
#include "sync.cuh"

namespace bbt {
namespace {

constexpr int NBMAX = 32;
constexpr int PTHREADS = 256;
constexpr int ROWS_PER_THREAD = 8;
constexpr int PROWS = PTHREADS * ROWS_PER_THREAD;   // rows per CTA in the panel kernel

// Householder scalars from (alpha, ||x||^2) as LAPACK dlarfg: beta =
// -sign(alpha) * hypot(alpha, ||x||), tau = (beta - alpha) / beta, v = x / (alpha - beta).
__device__ __forceinline__ void reflector(double alpha, double xx, double& beta, double& tau,
                                          double& scale) {
  if (xx == 0.0) {
    beta = alpha;
    tau = 0.0;
    scale = 0.0;
    return;
  }
  const double xn = sqrt(xx);
  const double h = hypot(alpha, xn);
  beta = -copysign(h, alpha);
  tau = (beta - alpha) / beta;
  scale = 1.0 / (alpha - beta);
}

// Panel step for column jj (jj = -1: prologue, only the partials of column 0).
// P: the panel, m rows (row 0 = the panel's first row), b columns, ld.
// pin/pout: per-CTA partials [cta][NBMAX]; entry c holds sum over rows > jj of
// A[i][jj] * A[i][c] (entry jj: the squared norm).  prow_in/out: pivot row.
__device__ __forceinline__ void panel_step(double* __restrict__ P, long m, int b, long ld, int jj,
                                           const double* __restrict__ pin, const double* __restrict__ prow_in,
                                           double* __restrict__ pout, double* __restrict__ prow_out,
                                           double* __restrict__ tau) {
  __shared__ double red[PTHREADS / 32][NBMAX];
  __shared__ double wv[NBMAX];
  __shared__ double sc[3];   // beta, tau, scale
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int ncta = gridDim.x;
  const int nx = jj + 1;   // next column
  // 1. reduce the previous step's partials, the same way in every CTA: each
  //    thread sums a strided subset of the CTAs, then a fixed-order tree
  //    over the threads (all loads of a thread are independent: one round
  //    trip to L2 instead of ncta serial ones)
  if (jj >= 0) {
    double part[NBMAX];
#pragma unroll
    for (int c = 0; c < NBMAX; ++c) part[c] = 0.0;
    for (int q = tid; q < ncta; q += PTHREADS) {
#pragma unroll
      for (int c = 0; c < NBMAX; ++c)
        if (c >= jj && c < b) part[c] += pin[(long)q * NBMAX + c];
    }
#pragma unroll
    for (int c = 0; c < NBMAX; ++c) {
      if (c < jj || c >= b) continue;
      double v = part[c];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0) red[warp][c] = v;
    }
    __syncthreads();
    for (int c = tid; c < b; c += PTHREADS) {
      if (c < jj) continue;
      double v = 0.0;
      for (int w = 0; w < PTHREADS / 32; ++w) v += red[w][c];
      wv[c] = v;
    }
    __syncthreads();
    if (tid == 0) {
      double be, ta, scl;
      reflector(prow_in[jj], wv[jj], be, ta, scl);
      sc[0] = be; sc[1] = ta; sc[2] = scl;
      if (blockIdx.x == 0) tau[jj] = ta;
    }
    __syncthreads();
    for (int c = jj + 1 + tid; c < b; c += PTHREADS) wv[c] = prow_in[c] + sc[2] * wv[c];  // v^T A[:,c]
    __syncthreads();
  }
  const double beta = jj >= 0 ? sc[0] : 0.0, ta = jj >= 0 ? sc[1] : 0.0, scl = jj >= 0 ? sc[2] : 0.0;
  double acc[NBMAX];
#pragma unroll
  for (int c = 0; c < NBMAX; ++c) acc[c] = 0.0;
  // 2. update this CTA's row chunks and accumulate the next column's dots
  for (long r0 = (long)blockIdx.x * PROWS; r0 < m; r0 += (long)gridDim.x * PROWS) {
    for (int rr = 0; rr < ROWS_PER_THREAD; ++rr) {
      const long i = r0 + rr * PTHREADS + tid;
      if (i >= m || i < jj) continue;
      double* row = P + i;   // element c at row[c*ld]
      double vi = 0.0;
      if (jj >= 0) {
        if (i == jj) {
          row[(long)jj * ld] = beta;
          vi = 1.0;
        } else {
          vi = row[(long)jj * ld] * scl;
          row[(long)jj * ld] = vi;
        }
      }
      double y = 0.0;   // updated A[i][nx]
#pragma unroll
      for (int c = 0; c < NBMAX; ++c) {
        if (c <= jj || c >= b) continue;
        double a = row[(long)c * ld];
        if (jj >= 0) {
          a -= ta * wv[c] * vi;
          row[(long)c * ld] = a;
        }
        if (c == nx) y = a;
        if (i > nx) acc[c] += y * a;   // c >= nx here, y already set at c == nx
      }
      if (i == nx && nx < b)
        for (int c = nx; c < b; ++c) prow_out[c] = row[(long)c * ld];
    }
  }
  if (nx >= b) return;
  // 3. block-reduce the partials for column nx
  __syncthreads();   // red[] was read in step 1
#pragma unroll
  for (int c = 0; c < NBMAX; ++c) {
    if (c < nx || c >= b) continue;
    double v = acc[c];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp][c] = v;
  }
  __syncthreads();
  for (int c = tid; c < b; c += PTHREADS) {
    if (c < nx) continue;
    double s = 0.0;
    for (int w = 0; w < PTHREADS / 32; ++w) s += red[w][c];
    pout[(long)blockIdx.x * NBMAX + c] = s;
  }
}

// Panel step for column jj (jj = -1: prologue, only the partials of column 0).
// P: the panel, m rows (row 0 = the panel's first row), b columns, ld.
// pin/pout: per-CTA partials [cta][NBMAX]; entry c holds sum over rows > jj of
// A[i][jj] * A[i][c] (entry jj: the squared norm).  prow_in/out: pivot row.
__global__ void __launch_bounds__(PTHREADS)
panel_step_kernel(double* __restrict__ P, long m, int b, long ld, int jj, const double* __restrict__ pin,
                  const double* __restrict__ prow_in, double* __restrict__ pout,
                  double* __restrict__ prow_out, double* __restrict__ tau) {
  panel_step(P, m, b, ld, jj, pin, prow_in, pout, prow_out, tau);
}

// All b column steps of a leaf panel in one cooperative launch, one bounded
// grid barrier between consecutive steps (the partials and pivot row of step
// jj are read by every CTA in step jj+1).
__global__ void __launch_bounds__(PTHREADS)
panel_leaf_kernel(double* __restrict__ P, long m, int b, long ld, double* __restrict__ pa,
                  double* __restrict__ pb, double* __restrict__ ra, double* __restrict__ rb,
                  double* __restrict__ tau, unsigned* bar, int* err) {
  double *pin = pa, *pout = pb, *rin = ra, *rout = rb;
  for (int jj = -1; jj < b; ++jj) {
    panel_step(P, m, b, ld, jj, pin, rin, pout, rout, tau);
    if (jj + 1 < b && !grid_sync(bar, err)) return;
    double* t = pin; pin = pout; pout = t;
    t = rin; rin = rout; rout = t;
  }
}

// Explicit unit-lower reflector block: Vb[i + c*m] = V(i, c) for i > c, 1 on
// the diagonal, 0 above; V(r, c) is read at src[r*rs + c*cs].
__global__ void make_vbuf(const double* __restrict__ src, long rs, long cs, long m, int b,
                          double* __restrict__ Vb) {
  const long total = m * b;
  for (long f = blockIdx.x * (long)blockDim.x + threadIdx.x; f < total; f += (long)gridDim.x * blockDim.x) {
    const long i = f % m;
    const int c = (int)(f / m);
    double v;
    if (i > c) v = src[i * rs + (long)c * cs];
    else v = (i == c) ? 1.0 : 0.0;
    Vb[f] = v;
  }
}

// dlarft (forward, columnwise): T upper triangular b x b (col-major, ld b)
// from G = V^T V and tau.  T(i,i) = tau_i; T(0:i, i) = -tau_i T(0:i,0:i) G(0:i, i).
// b <= TMAX; T is built in shared memory (dynamic, (TMAX+1) * b doubles).
constexpr int TMAX = 128;
__global__ void larft_kernel(int b, const double* __restrict__ G, const double* __restrict__ tau,
                             double* __restrict__ T) {
  extern __shared__ double t_[];   // t[j][l] at t_[j * (b + 1) + l]
  const int j = threadIdx.x, ld = b + 1;
  for (int f = j; f < b * ld; f += blockDim.x) t_[f] = 0.0;
  __syncthreads();
  for (int i = 0; i < b; ++i) {
    const double ti = tau[i];
    if (j < i) {
      double s = 0.0;
      for (int l = j; l < i; ++l) s += t_[j * ld + l] * G[l + (long)i * b];
      t_[j * ld + i] = -ti * s;
    }
    if (j == i) t_[i * ld + i] = ti;
    __syncthreads();
  }
  for (int f = j; f < b * b; f += blockDim.x) T[f] = t_[(f % b) * ld + f / b];
}

// A panel (m x b, ld) += I on its top b x b block, rows [-above, 0) zeroed.
__global__ void panel_identity(double* __restrict__ P, long ld, int b, long above) {
  const long total = (above + b) * b;
  for (long f = blockIdx.x * (long)blockDim.x + threadIdx.x; f < total; f += (long)gridDim.x * blockDim.x) {
    const int c = (int)(f / (above + b));
    const long r = f % (above + b) - above;   // relative to the panel's first row
    double* e = P + r + (long)c * ld;
    if (r < 0) *e = 0.0;
    else if (r == c) *e += 1.0;
  }
}

}  // namespace

namespace {

bbt_status larft(bbt_ctx* ctx, int b, const double* G, const double* tau, double* T) {
  const int smem = (b + 1) * b * (int)sizeof(double);
  static bool attr = false;
  if (!attr) {
    BBT_CUDA(ctx, cudaFuncSetAttribute(larft_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (TMAX + 1) * TMAX * (int)sizeof(double)));
    attr = true;
  }
  larft_kernel<<<1, TMAX, smem, ctx->stream>>>(b, G, tau, T);
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

// Column-by-column factorisation of a panel of b <= NBMAX columns: one
// cooperative launch when the grid fits on the GPU at once, otherwise one
// launch per column.
bbt_status panel_columns(bbt_ctx* ctx, double* P, long m, int b, long ld, double* tau) {
  static int coop_blocks = -1;   // co-resident CTAs of panel_leaf_kernel per SM
  if (coop_blocks < 0) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, panel_leaf_kernel, PTHREADS, 0) != cudaSuccess)
      per_sm = 0;
    coop_blocks = per_sm;
  }
  size_t mark = ctx->ws.top;
  long nblk = (m + PROWS - 1) / PROWS;
  const long coop_max = (long)coop_blocks * ctx->num_sms;
  const bool coop = coop_max > 0 && ctx->allow_coop;
  if (coop && nblk > coop_max) nblk = coop_max;   // grid-stride over the row chunks
  double* pa = ctx->ws.take<double>((size_t)nblk * NBMAX);
  double* pb = ctx->ws.take<double>((size_t)nblk * NBMAX);
  double* ra = ctx->ws.take<double>(NBMAX);
  double* rb = ctx->ws.take<double>(NBMAX);
  if (!rb) return fail(ctx, BBT_ERR_NOMEM, "panel: workspace");
  if (coop) {
    ProfScope prof(ctx, BBT_PROF_PANEL, 8.0 * (double)m * (double)b * (double)(b + 1));
    BBT_CUDA(ctx, cudaMemsetAsync(ctx->d_barrier, 0, 2 * sizeof(unsigned), ctx->stream));
    BBT_CUDA(ctx, cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), ctx->stream));
    void* args[] = {&P, &m, &b, &ld, &pa, &pb, &ra, &rb, &tau, &ctx->d_barrier, &ctx->d_flag};
    BBT_CUDA(ctx, cudaLaunchCooperativeKernel((void*)panel_leaf_kernel, dim3((unsigned)nblk), dim3(PTHREADS),
                                              args, 0, ctx->stream));
    BBT_LAUNCHED(ctx);
  } else {
    double *pin = pa, *pout = pb, *rin = ra, *rout = rb;
    for (int jj = -1; jj < b; ++jj) {
      ProfScope prof(ctx, BBT_PROF_PANEL, 16.0 * (double)m * (double)(b - jj));
      panel_step_kernel<<<(int)nblk, PTHREADS, 0, ctx->stream>>>(P, m, b, ld, jj, pin, rin, pout, rout, tau);
      BBT_LAUNCHED(ctx);
      double* t = pin; pin = pout; pout = t;
      t = rin; rin = rout; rout = t;
    }
  }
  ctx->ws.top = mark;
  return BBT_OK;
}

// Recursive panel factorisation (Elmroth-Gustavson): factor the left half,
// apply its block reflector to the right half with GEMMs, factor the right
// half.  Leaves of <= leaf columns are factored column by column; a leaf of
// a tall panel (rows x 16 doubles) stays resident in L2 across its column
// steps.
bbt_status panel_factor(bbt_ctx* ctx, double* P, long m, int b, long ld, double* tau, int leaf) {
  if (b <= leaf) return panel_columns(ctx, P, m, b, ld, tau);
  const int h = b / 2;
  BBT_TRY(panel_factor(ctx, P, m, h, ld, tau, leaf));
  size_t mark = ctx->ws.top;
  double* Vb = ctx->ws.take<double>((size_t)m * h);
  double* G = ctx->ws.take<double>((size_t)h * h);
  double* T = ctx->ws.take<double>((size_t)h * h);
  double* W = ctx->ws.take<double>((size_t)h * (b - h));
  double* W2 = ctx->ws.take<double>((size_t)h * (b - h));
  if (!W2) return fail(ctx, BBT_ERR_NOMEM, "panel: workspace");
  make_vbuf<<<4 * ctx->num_sms, 256, 0, ctx->stream>>>(P, 1, ld, m, h, Vb);
  BBT_LAUNCHED(ctx);
  BBT_TRY(dgemm(ctx, true, false, h, h, m, 1.0, Vb, m, Vb, m, 0.0, G, h));
  BBT_TRY(larft(ctx, h, G, tau, T));
  double* A2 = P + (long)h * ld;
  BBT_TRY(dgemm(ctx, true, false, h, b - h, m, 1.0, Vb, m, A2, ld, 0.0, W, h));
  BBT_TRY(dgemm(ctx, true, false, h, b - h, h, 1.0, T, h, W, h, 0.0, W2, h));
  BBT_TRY(dgemm(ctx, false, false, (int)m, b - h, h, -1.0, Vb, m, W2, h, 1.0, A2, ld));
  ctx->ws.top = mark;
  return panel_factor(ctx, P + h + (long)h * ld, m - h, b - h, ld, tau + h, leaf);
}

}  // namespace

size_t qr_workspace_bytes(long rows, int cols, int ncols_apply, const QrPlan& plan) {
  const int nb = plan.nb;
  const long nblk = (rows + PROWS - 1) / PROWS;
  const int wide = cols > ncols_apply ? cols : ncols_apply;
  size_t b = 0;
  b += (size_t)rows * nb * 8 + 256;                 // Vbuf of the panel
  b += (size_t)rows * (nb / 2) * 8 + 256;           // Vbuf of the recursion
  b += 2 * (size_t)nblk * NBMAX * 8 + 1024;         // partials, pivot rows
  b += 3 * (size_t)nb * wide * 8 + 768;             // W, W2, M
  b += 6 * (size_t)nb * nb * 8 + 1536;              // G, T (+ recursion)
  b += (size_t)257 * nb * wide * 8 + 256;           // split-K partials
  return b;
}

bbt_status geqrf(bbt_ctx* ctx, long rows, int cols, double* A, long lda, double* tau, double* Tst,
                 const QrPlan& plan) {
  const int nb = plan.nb;
  if (nb < 1 || nb > TMAX || plan.leaf < 1 || plan.leaf > NBMAX)
    return fail(ctx, BBT_ERR_ARG, "geqrf: nb=%d leaf=%d", nb, plan.leaf);
  if (rows < cols || cols < 1) return fail(ctx, BBT_ERR_ARG, "geqrf: rows=%ld cols=%d", rows, cols);
  size_t mark = ctx->ws.top;
  double* Vb = ctx->ws.take<double>((size_t)rows * nb);
  double* W = ctx->ws.take<double>((size_t)nb * cols);
  double* W2 = ctx->ws.take<double>((size_t)nb * cols);
  double* G = ctx->ws.take<double>((size_t)nb * nb);
  if (!G) return fail(ctx, BBT_ERR_NOMEM, "geqrf: workspace");
  for (int p0 = 0, pi = 0; p0 < cols; p0 += nb, ++pi) {
    const int b = cols - p0 < nb ? cols - p0 : nb;
    const long m = rows - p0;
    double* Pn = A + p0 + (long)p0 * lda;
    BBT_TRY(panel_factor(ctx, Pn, m, b, lda, tau + p0, plan.leaf));
    make_vbuf<<<4 * ctx->num_sms, 256, 0, ctx->stream>>>(Pn, 1, lda, m, b, Vb);
    BBT_LAUNCHED(ctx);
    BBT_TRY(dgemm(ctx, true, false, b, b, m, 1.0, Vb, m, Vb, m, 0.0, G, b));
    double* T = Tst + (size_t)pi * nb * nb;
    BBT_TRY(larft(ctx, b, G, tau + p0, T));
    const int nc = cols - p0 - b;
    if (nc > 0) {   // C <- (I - V T V^T)^T C
      double* C = A + p0 + (long)(p0 + b) * lda;
      BBT_TRY(dgemm(ctx, true, false, b, nc, m, 1.0, Vb, m, C, lda, 0.0, W, b));
      BBT_TRY(dgemm(ctx, true, false, b, nc, b, 1.0, T, b, W, b, 0.0, W2, b));
      BBT_TRY(dgemm(ctx, false, false, (int)m, nc, b, -1.0, Vb, m, W2, b, 1.0, C, lda));
    }
  }
  ctx->ws.top = mark;
  return BBT_OK;
}

bbt_status orgqr(bbt_ctx* ctx, long rows, int cols, double* A, long lda, const double* tau,
                 const double* Tst, const QrPlan& plan) {
  const int nb = plan.nb;
  size_t mark = ctx->ws.top;
  double* Vb = ctx->ws.take<double>((size_t)rows * nb);
  double* W = ctx->ws.take<double>((size_t)nb * cols);
  double* W2 = ctx->ws.take<double>((size_t)nb * cols);
  double* M = ctx->ws.take<double>((size_t)nb * nb);
  if (!M) return fail(ctx, BBT_ERR_NOMEM, "orgqr: workspace");
  const int npan = (cols + nb - 1) / nb;
  for (int pi = npan - 1; pi >= 0; --pi) {
    const int p0 = pi * nb;
    const int b = cols - p0 < nb ? cols - p0 : nb;
    const long m = rows - p0;
    double* Pn = A + p0 + (long)p0 * lda;
    const double* T = Tst + (size_t)pi * nb * nb;
    make_vbuf<<<4 * ctx->num_sms, 256, 0, ctx->stream>>>(Pn, 1, lda, m, b, Vb);
    BBT_LAUNCHED(ctx);
    const int nc = cols - p0 - b;
    if (nc > 0) {   // Q[p0:, p0+b:] = H_p Q[p0:, p0+b:]
      double* C = A + p0 + (long)(p0 + b) * lda;
      BBT_TRY(dgemm(ctx, true, false, b, nc, m, 1.0, Vb, m, C, lda, 0.0, W, b));
      BBT_TRY(dgemm(ctx, false, false, b, nc, b, 1.0, T, b, W, b, 0.0, W2, b));
      BBT_TRY(dgemm(ctx, false, false, (int)m, nc, b, -1.0, Vb, m, W2, b, 1.0, C, lda));
    }
    // panel columns: E - V (T V1^T), rows above the panel zeroed
    BBT_TRY(dgemm(ctx, false, true, b, b, b, 1.0, T, b, Vb, m, 0.0, M, b));
    BBT_TRY(dgemm(ctx, false, false, (int)m, b, b, -1.0, Vb, m, M, b, 0.0, Pn, lda));
    panel_identity<<<ctx->num_sms, 256, 0, ctx->stream>>>(Pn, lda, b, p0);
    BBT_LAUNCHED(ctx);
  }
  ctx->ws.top = mark;
  return BBT_OK;
}

bbt_status ormqr_left_notrans(bbt_ctx* ctx, long rows, int k, const double* V, long rs, long cs,
                              const double* tau, double* C, long ldc, int ncols, bool c_rowmajor,
                              const QrPlan& plan) {
  if (k < 1 || rows < k) return fail(ctx, BBT_ERR_ARG, "ormqr: rows=%ld k=%d", rows, k);
  const int nb = plan.nb;
  size_t mark = ctx->ws.top;
  double* Vb = ctx->ws.take<double>((size_t)rows * nb);
  double* W = ctx->ws.take<double>((size_t)nb * ncols);
  double* W2 = ctx->ws.take<double>((size_t)nb * ncols);
  double* G = ctx->ws.take<double>((size_t)nb * nb);
  double* T = ctx->ws.take<double>((size_t)nb * nb);
  if (!T) return fail(ctx, BBT_ERR_NOMEM, "ormqr: workspace");
  const int npan = (k + nb - 1) / nb;
  for (int pi = npan - 1; pi >= 0; --pi) {
    const int p0 = pi * nb;
    const int b = k - p0 < nb ? k - p0 : nb;
    const long m = rows - p0;
    make_vbuf<<<4 * ctx->num_sms, 256, 0, ctx->stream>>>(V + p0 * rs + (long)p0 * cs, rs, cs, m, b, Vb);
    BBT_LAUNCHED(ctx);
    BBT_TRY(dgemm(ctx, true, false, b, b, m, 1.0, Vb, m, Vb, m, 0.0, G, b));
    BBT_TRY(larft(ctx, b, G, tau + p0, T));
    if (!c_rowmajor) {   // C col-major rows x ncols
      double* Cp = C + p0;
      BBT_TRY(dgemm(ctx, true, false, b, ncols, m, 1.0, Vb, m, Cp, ldc, 0.0, W, b));
      BBT_TRY(dgemm(ctx, false, false, b, ncols, b, 1.0, T, b, W, b, 0.0, W2, b));
      BBT_TRY(dgemm(ctx, false, false, (int)m, ncols, b, -1.0, Vb, m, W2, b, 1.0, Cp, ldc));
    } else {             // C row-major rows x ncols = col-major C^T (ncols x rows, ld ldc)
      double* Ct = C + (long)p0 * ldc;
      // W^T (ncols x b) = C^T V ; W2^T = W^T T^T ; C^T -= W2^T V^T
      BBT_TRY(dgemm(ctx, false, false, ncols, b, m, 1.0, Ct, ldc, Vb, m, 0.0, W, ncols));
      BBT_TRY(dgemm(ctx, false, true, ncols, b, b, 1.0, W, ncols, T, b, 0.0, W2, ncols));
      BBT_TRY(dgemm(ctx, false, true, ncols, (int)m, b, -1.0, W2, ncols, Vb, m, 1.0, Ct, ldc));
    }
  }
  ctx->ws.top = mark;
  return BBT_OK;
}

}  // namespace bbt
