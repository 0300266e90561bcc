// Two-sided Householder bidiagonalisation A = Q B P^T of a dense n x n
// column-major matrix (LAPACK dgebrd semantics and storage), blocked:
// panels of NB columns and rows are reduced by one persistent cooperative
// kernel each, and the rest of the matrix is brought up to date once per
// panel by two rank-NB GEMMs on the FP64 tensor cores (dgemm.cu).
//
// Used for the dense-matrix SVD (the 8192^2 stress case), where the
// reference's one-sided Ralha recurrence (client.cpp:829-910) is not
// backward stable: on clustered spectra it loses ~1e-6 relative accuracy in
// the small singular values.  B is upper bidiagonal; v_j is stored below the
// diagonal of column j, u_j right of the superdiagonal of row j (the unit
// entries implied), d and e hold B.
//
// Within a panel (local indices; V, U the panel's column and row reflectors,
// X, Y their companions) the matrix is never updated in place except for the
// panel's own column j and row j: the current matrix is
//   A_j = A - V(:, :j) Y(:, :j)^T - X(:, :j) U(:j, :),
// and each column step needs the two matrix-vector products
//   y_j = tauq_j (A^T v_j - Y (V^T v_j) - U^T (X^T v_j))    (gemv pass 1)
//   x_j = taup_j (A u_j  - V (Y^T u_j)  - X (U u_j))         (gemv pass 2)
// over the trailing part of the panel-start matrix.  Those two read-only
// passes are the kernel's HBM traffic (16 bytes per trailing element and
// column step, against 24 for the unblocked two-sided update); everything
// else is O(n NB) per step.  After the panel, A(NB:, NB:) -= V Y^T + X U.
//
// Column step j, five phases separated by bounded grid barriers:
//   B: column reflector of the updated column j (its norm from per-CTA
//      partials), gemv pass 1 (one warp per column and chunk of rows,
//      per-chunk partials) and the partials of V^T v_j, X^T v_j;
//   C: y_j, the updated row j (its norm's partials); v_j written to A;
//   D: row reflector, gemv pass 2 (32-row x cch-column tiles, per-chunk
//      partials) and the partials of Y^T u_j, U u_j; u_j written to A;
//   E: x_j, and the update of column j+1 with the partials of its norm.
// Every reduction is summed in a fixed order, so the result is deterministic.
// The gemv chunks are sized per panel to minimise the busiest warp's work
// (its items times the chunk length): many short items while the trailing
// matrix is small (the passes are latency-bound there), few long ones with
// no ragged last round when it is large (bandwidth-bound); loads of a row or
// column are issued before the stores that follow them.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "internal.h"
#include "sync.cuh"

namespace bbt {
namespace {

constexpr int NB = 32;      // panel width
constexpr int GT = 256;
constexpr int GW = GT / 32;
constexpr int PG = 32;      // CTAs that form the panel-correction partials

struct PanelArgs {
  int M;           // trailing order at this panel
  int nbp;         // columns (and rows) reduced by this panel
  long ld;
  double* A;       // panel origin, column-major, ld
  double* d;       // at the panel origin
  double* e;
  double* tauq;
  double* taup;
  double* X;       // M x NB, ld M
  double* Y;       // M x NB, ld M
  double* g;       // [nr1][M]: gemv pass 1 partials, by row chunk
  double* rowb;    // M: the updated row j
  double* hp;      // [ncc][M]: gemv pass 2 partials, by column chunk
  int nr1, r1;     // gemv pass 1: row chunks (of r1 rows) per column
  int ncc, cch;    // gemv pass 2: column chunks (of cch columns) per 32-row block
  double* colp;    // [grid]
  double* rowp;    // [grid]
  double* pq;      // [PG][2 NB]
  double* st;      // [PG][2 NB]
  unsigned* bar;
  int* err;
};

__device__ double bsum(double v, double* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double s = 0.0;
  for (int k = 0; k < GW; ++k) s += sh[k];
  __syncthreads();
  return s;
}

// Sum of the per-CTA partials p[0..g), in index order (the same in every CTA).
__device__ double psum(const double* p, int g, double* sh) {
  double s = 0.0;
  for (int k = threadIdx.x; k < g; k += GT) s += p[k];
  return bsum(s, sh);
}

// dlarfg on (alpha, ||x||^2): beta, tau, scale (x -> scale * x).
__device__ void larfg(double alpha, double xx, double* beta, double* tau, double* scale) {
  if (xx == 0.0) { *beta = alpha; *tau = 0.0; *scale = 0.0; return; }
  const double h = hypot(alpha, sqrt(xx));
  const double b = -copysign(h, alpha);
  *beta = b;
  *tau = (b - alpha) / b;
  *scale = 1.0 / (alpha - b);
}

// out[kk] (kk < cnt) = sum over the PG partial rows of part[b * 2NB + kk].
__device__ void sum_partials(const double* part, int cnt, double* out) {
  for (int kk = threadIdx.x; kk < cnt; kk += GT) {
    double s = 0.0;
    for (int b = 0; b < PG; ++b) s += part[b * 2 * NB + kk];
    out[kk] = s;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(GT) labrd_kernel(PanelArgs P) {
  __shared__ double sh[GW];
  __shared__ double sc[8];
  __shared__ double cor[2 * NB];
  const int M = P.M, tid = threadIdx.x, G = gridDim.x;
  const long ld = P.ld;
  double* A = P.A;
  const double* X = P.X;
  const double* Y = P.Y;
  const int lane = tid & 31, gw = blockIdx.x * GW + (tid >> 5), nwarps = G * GW;
  const long gtid = (long)blockIdx.x * GT + tid, nthr = (long)G * GT;
  // the panel's first column: its norm's partials (no pending updates)
  {
    double s = 0.0;
    for (long r = 1 + gtid; r < M; r += nthr) { const double x = A[r]; s += x * x; }
    s = bsum(s, sh);
    if (tid == 0) P.colp[blockIdx.x] = s;
  }
  if (!grid_sync(P.bar, P.err)) return;
  for (int j = 0; j < P.nbp; ++j) {
    double* cj = A + j * ld;
    // ---- B: column reflector, gemv pass 1, partials of V^T v and X^T v
    {
      const double s = psum(P.colp, G, sh);
      if (tid == 0) {
        double be, ta, scl;
        larfg(cj[j], s, &be, &ta, &scl);
        sc[0] = be; sc[1] = ta; sc[2] = scl;
      }
      __syncthreads();
    }
    const double tq = sc[1], sq = sc[2];
    if (blockIdx.x == 0 && tid == 0) { P.d[j] = sc[0]; P.tauq[j] = tq; }
    if (j == M - 1) break;   // the last diagonal entry: no row reflector
    {   // g_c = v^T A(j:, c), v_j(j) = 1: one warp per (column, chunk of r1 rows), partials by chunk
      const int ncol = M - j - 1, items = ncol * P.nr1;
      for (int it = gw; it < items; it += nwarps) {
        const int c = j + 1 + it % ncol, rc = it / ncol;
        const double* col = A + c * ld;
        const int re = min(M, (rc + 1) * P.r1);
        double s = 0.0, s1 = 0.0;
        int r = max(j + 1, rc * P.r1) + lane;
        if (r + 7 * 32 < re) {   // batches of eight loads per lane, the next batch issued first
          double a[8], v[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) { a[u] = col[r + u * 32]; v[u] = cj[r + u * 32]; }
          for (; r + 7 * 32 < re; r += 8 * 32) {
            const bool more = r + 8 * 32 + 7 * 32 < re;
            double a2[8], v2[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
              a2[u] = more ? col[r + 256 + u * 32] : 0.0;
              v2[u] = more ? cj[r + 256 + u * 32] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 8; u += 2) {
              s += a[u] * v[u];
              s1 += a[u + 1] * v[u + 1];
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) { a[u] = a2[u]; v[u] = v2[u]; }
          }
        }
        for (; r < re; r += 32) s += col[r] * cj[r];
        s += s1;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) P.g[(long)rc * M + c] = s;
      }
    }
    if (blockIdx.x < PG && j > 0) {   // rows split over PG CTAs: p_k = V(:, k)^T v, q_k = X(:, k)^T v
      const int rows = M - j, per = (rows + PG - 1) / PG;
      const int r0 = j + blockIdx.x * per, r1 = min(M, r0 + per);
      for (int kk = tid >> 5; kk < 2 * j; kk += GW) {
        const double* src = kk < j ? A + kk * ld : X + (long)(kk - j) * M;
        double s = 0.0;
        for (int r = r0 + lane; r < r1; r += 32) s += src[r] * (r == j ? 1.0 : cj[r] * sq);
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) P.pq[blockIdx.x * 2 * NB + kk] = s;
      }
    }
    if (!grid_sync(P.bar, P.err)) return;
    // ---- C: y_j, the updated row j and its norm's partials; v_j into A
    if (j > 0) sum_partials(P.pq, 2 * j, cor);
    {
      double pr = 0.0;
      for (long c = j + 1 + gtid; c < M; c += nthr) {
        // column j still holds the updated column a_j (scaled to v_j below)
        double gs = 0.0;
        for (int rc = 0; rc < P.nr1; ++rc) gs += P.g[(long)rc * M + c];
        double gy = A[j + c * ld] + sq * gs;
        for (int k = 0; k < j; ++k) gy -= Y[c + (long)k * M] * cor[k] + A[k + c * ld] * cor[j + k];
        gy *= tq;
        double r = A[j + c * ld] - gy;   // V(j, j) = 1
        for (int k = 0; k < j; ++k) r -= A[j + k * ld] * Y[c + (long)k * M] + X[j + (long)k * M] * A[k + c * ld];
        P.Y[c + (long)j * M] = gy;   // stores after every load of the row
        P.rowb[c] = r;
        if (c >= j + 2) pr += r * r;
      }
      pr = bsum(pr, sh);
      if (tid == 0) P.rowp[blockIdx.x] = pr;
      for (long r = j + 1 + gtid; r < M; r += nthr) cj[r] *= sq;   // v_j
      if (blockIdx.x == 0 && tid == 0) cj[j] = sc[0];
    }
    if (!grid_sync(P.bar, P.err)) return;
    // ---- D: row reflector, gemv pass 2, partials of Y^T u and U u; u_j into A
    {
      const double s = psum(P.rowp, G, sh);
      if (tid == 0) {
        double be, ta, scl;
        larfg(P.rowb[j + 1], s, &be, &ta, &scl);
        sc[3] = be; sc[4] = ta; sc[5] = scl;
      }
      __syncthreads();
    }
    const double tp = sc[4], sp = sc[5];
    if (blockIdx.x == 0 && tid == 0) { P.e[j] = sc[3]; P.taup[j] = tp; }
    {
      // (32-row block, column chunk cc of cch columns) per warp; the chunks are
      // absolute (columns [cc cch, (cc + 1) cch) past j), so phase E sums the
      // same ncc partials in the same order for every step of the panel
      const int r0 = j + 1;
      const int nrb = (M - r0 + 31) / 32, ncc = P.ncc;
      for (int item = gw; item < nrb * ncc; item += nwarps) {
        const int rb = item % nrb, cc = item / nrb;
        const int r = r0 + rb * 32 + lane;
        const int ca = max(j + 1, cc * P.cch), cb = min(M, (cc + 1) * P.cch);
        double s = 0.0, s1 = 0.0;
        if (r < M) {
          int c = ca;
          if (c + 7 < cb) {   // batches of eight columns, the next batch's loads issued first
            double a[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) a[q] = A[r + (c + q) * ld];
            for (; c + 7 < cb; c += 8) {
              const bool more = c + 15 < cb;
              double a2[8];
#pragma unroll
              for (int q = 0; q < 8; ++q) a2[q] = more ? A[r + (c + 8 + q) * ld] : 0.0;
              double u[8];
#pragma unroll
              for (int q = 0; q < 8; ++q) u[q] = (c + q == j + 1) ? 1.0 : P.rowb[c + q] * sp;
#pragma unroll
              for (int q = 0; q < 8; q += 2) {
                s += a[q] * u[q];
                s1 += a[q + 1] * u[q + 1];
              }
#pragma unroll
              for (int q = 0; q < 8; ++q) a[q] = a2[q];
            }
          }
          for (; c < cb; ++c) s += A[r + c * ld] * ((c == j + 1) ? 1.0 : P.rowb[c] * sp);
          P.hp[(long)cc * M + r] = s + s1;
        }
      }
    }
    if (blockIdx.x < PG) {   // columns split over PG CTAs: s_k = Y(:, k)^T u (k <= j), t_k = U(k, :) u (k < j)
      const int cols = M - (j + 1), per = (cols + PG - 1) / PG;
      const int ca = j + 1 + blockIdx.x * per, cb = min(M, ca + per);
      for (int kk = tid >> 5; kk < 2 * j + 1; kk += GW) {
        double s = 0.0;
        for (int c = ca + lane; c < cb; c += 32) {
          const double u = (c == j + 1) ? 1.0 : P.rowb[c] * sp;
          s += (kk <= j ? Y[c + (long)kk * M] : A[(kk - j - 1) + c * ld]) * u;
        }
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) P.st[blockIdx.x * 2 * NB + kk] = s;
      }
    }
    for (long c = j + 2 + gtid; c < M; c += nthr) A[j + c * ld] = P.rowb[c] * sp;   // u_j (row j is not read here)
    if (blockIdx.x == 0 && tid == 0) A[j + (j + 1) * ld] = (j == P.nbp - 1 && j + 1 < M) ? 1.0 : sc[3];
    if (!grid_sync(P.bar, P.err)) return;
    // ---- E: x_j and the update of column j+1 (and its norm's partials)
    sum_partials(P.st, 2 * j + 1, cor);
    {
      const int ncc = P.ncc;
      const bool next = j + 1 < P.nbp;
      double* cn = A + (j + 1) * ld;
      double pn = 0.0;
      for (long r = j + 1 + gtid; r < M; r += nthr) {
        double h = 0.0;
        for (int cc = 0; cc < ncc; ++cc) h += P.hp[(long)cc * M + r];
        for (int k = 0; k <= j; ++k) h -= A[r + k * ld] * cor[k];
        for (int k = 0; k < j; ++k) h -= X[r + (long)k * M] * cor[j + 1 + k];
        const double x = tp * h;
        if (next) {   // column j+1 of A_{j+1}: U(k, j+1) = A(k, j+1) for k < j, U(j, j+1) = 1
          double a = cn[r] - x;
          for (int k = 0; k <= j; ++k) a -= A[r + k * ld] * Y[(j + 1) + (long)k * M];
          for (int k = 0; k < j; ++k) a -= X[r + (long)k * M] * A[k + (j + 1) * ld];
          cn[r] = a;
          if (r >= j + 2) pn += a * a;
        }
        P.X[r + (long)j * M] = x;   // after the loads of X above
      }
      pn = bsum(pn, sh);
      if (tid == 0) P.colp[blockIdx.x] = pn;
    }
    if (!grid_sync(P.bar, P.err)) return;
  }
}

// A(j, j+1) <- e_j after the trailing update used the unit entry there.
__global__ void put_e_kernel(double* a, const double* e) { *a = *e; }

}  // namespace

bbt_status gebrd(bbt_ctx* ctx, int n, double* A, double* d, double* e, double* tauq, double* taup) {
  if (n < 2) return fail(ctx, BBT_ERR_ARG, "gebrd: n=%d", n);
  const size_t mark = ctx->ws.top;
  int per_sm = 0;
  BBT_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, labrd_kernel, GT, 0));
  if (per_sm < 1) return fail(ctx, BBT_ERR_CUDA, "gebrd: kernel does not fit an SM");
  const int grid = std::max(PG, ctx->num_sms * std::min(per_sm, 2));
  PanelArgs P;
  P.ld = n;
  P.X = ctx->ws.take<double>((size_t)n * NB);
  P.Y = ctx->ws.take<double>((size_t)n * NB);
  P.rowb = ctx->ws.take<double>(n);
  const int nwarps = grid * GW;
  const int nr1_max = 16, ncc_max = (n + 63) / 64;
  P.g = ctx->ws.take<double>((size_t)nr1_max * n);
  P.hp = ctx->ws.take<double>((size_t)ncc_max * n);
  P.colp = ctx->ws.take<double>(grid);
  P.rowp = ctx->ws.take<double>(grid);
  P.pq = ctx->ws.take<double>(PG * 2 * NB);
  P.st = ctx->ws.take<double>(PG * 2 * NB);
  if (!P.st) return fail(ctx, BBT_ERR_NOMEM, "gebrd: workspace");
  P.bar = ctx->d_barrier;
  P.err = ctx->d_flag;
  BBT_CUDA(ctx, cudaMemsetAsync(taup, 0, (size_t)n * sizeof(double), ctx->stream));
  BBT_CUDA(ctx, cudaMemsetAsync(ctx->d_barrier, 0, 2 * sizeof(unsigned), ctx->stream));
  BBT_CUDA(ctx, cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), ctx->stream));
  const double traffic = 16.0 * (double)n * n * n / 3.0;   // the two gemv passes
  {
    ProfScope prof(ctx, BBT_PROF_RALHA, traffic);
    for (int i0 = 0; i0 < n; i0 += NB) {
      const int M = n - i0;
      P.M = M;
      P.nbp = std::min(NB, M);
      P.A = A + i0 + (long)i0 * n;
      P.d = d + i0;
      P.e = e + i0;
      P.tauq = tauq + i0;
      P.taup = taup + i0;
      // gemv chunking: the chunk count that minimises the busiest warp's work,
      // (items per warp, rounded up) x (chunk length), so that neither a long
      // tail round (large trailing matrix) nor long serial chunks (small one)
      // set the step's time
      auto best_chunks = [&](int units, int len, int cap, int align) {
        int best = 1;
        long cost = -1;
        for (int c = 1; c <= cap; ++c) {
          const long chunk = ((len + c - 1) / c + align - 1) / align * align;
          const long rounds = ((long)units * c + nwarps - 1) / nwarps;
          const long cst = rounds * chunk + 8L * c;   // + the partials summed per output
          if (cost < 0 || cst < cost) { cost = cst; best = c; }
        }
        return best;
      };
      P.nr1 = best_chunks(M, M, nr1_max, 32);
      P.r1 = ((M + P.nr1 - 1) / P.nr1 + 31) / 32 * 32;
      const int nrb = (M + 31) / 32;
      P.ncc = best_chunks(nrb, M, std::max(1, std::min(ncc_max, (M + 63) / 64)), 8);
      P.cch = ((M + P.ncc - 1) / P.ncc + 7) / 8 * 8;
      void* args[] = {&P};
      BBT_CUDA(ctx, cudaLaunchCooperativeKernel((void*)labrd_kernel, dim3(grid), dim3(GT), args, 0, ctx->stream));
      BBT_LAUNCHED(ctx);
      if (M > NB) {   // A(NB:, NB:) -= V Y^T + X U on the FP64 tensor cores
        const int T = M - NB;
        double* A22 = P.A + NB + (long)NB * n;
        BBT_TRY(dgemm(ctx, false, true, T, T, NB, -1.0, P.A + NB, n, P.Y + NB, M, 1.0, A22, n));
        BBT_TRY(dgemm(ctx, false, false, T, T, NB, -1.0, P.X + NB, M, P.A + (long)NB * n, n, 1.0, A22, n));
        put_e_kernel<<<1, 1, 0, ctx->stream>>>(P.A + (NB - 1) + (long)NB * n, P.e + NB - 1);
        BBT_LAUNCHED(ctx);
      }
    }
  }
  int herr = 0;
  BBT_CUDA(ctx, cudaMemcpyAsync(&herr, ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  BBT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->ws.top = mark;
  if (herr) return fail(ctx, BBT_ERR_TIMEOUT, "gebrd: grid barrier timed out");
  return BBT_OK;
}

}  // namespace bbt
