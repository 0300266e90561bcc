// Two-sided Householder bidiagonalisation (LAPACK dgebd2 semantics) of a
// dense n x n column-major matrix, as one persistent cooperative kernel.
//
// Used for the dense-matrix SVD (the 8192^2 stress case), where the
// reference's one-sided Ralha recurrence (client.cpp:829-910) is not
// backward stable: on clustered spectra it loses ~1e-6 relative accuracy in
// the small singular values.  A = Q B P^T with B upper bidiagonal; the
// reflectors are stored as LAPACK's dgebrd stores them (v_i below the
// diagonal of column i, u_i right of the superdiagonal of row i).
//
// Step i, with v the column reflector of A(i:, i) and u the row reflector
// of the updated row i:
//   phase 1 (every CTA): the reflector H_i from ||A(i+1:, i)||^2, summed
//           from per-CTA partials left by the previous pass 2;
//   pass 1  (column-partitioned): w_j = v^T A(i:, j) for j > i and the
//           updated row i, r_j = A(i, j) - tauq w_j, with per-CTA partials
//           of sum r_j^2 and sum w_j r_j;
//   barrier;
//   phase 2 (every CTA): the reflector G_i of r and w . u from the partials;
//   pass 2  (row-partitioned, 8 rows x 4 column phases per warp): z_r = (A u)_r -
//           tauq v_r (w . u), then A(r, j) -= tauq v_r w_j + taup z_r u_j
//           and A(r, i) <- v_r; the partials of the next column's norm;
//   barrier.
// Every reduction is summed in a fixed order, so the result is deterministic.
// Two grid barriers per step, bounded (sync.cuh).
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "internal.h"
#include "sync.cuh"

namespace bbt {
namespace {

constexpr int GT = 256;
constexpr int GW = GT / 32;

struct BrdArgs {
  int n;
  double* A;      // n x n column-major, lda = n
  double* d;      // n
  double* e;      // n-1
  double* tauq;   // n
  double* taup;   // n
  double* w;      // n
  double* rowb;   // n: updated row i
  double* colp;   // 2 x grid: per-CTA ||A(i+1:, i)||^2, ping-pong between steps
  double* rowp;   // grid: per-CTA sum_{j >= i+2} rowb_j^2
  double* wup;    // grid: per-CTA sum_{j >= i+2} w_j rowb_j
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

__global__ void __launch_bounds__(GT) gebrd_kernel(BrdArgs P) {
  __shared__ double sh[GW];
  __shared__ double sc[8];
  const int n = P.n, tid = threadIdx.x, G = gridDim.x;
  double* A = P.A;
  const long ld = n;
  const int lane = tid & 31, gw = blockIdx.x * GW + (tid >> 5), nwarps = G * GW;
  // ---- set-up: per-CTA partials of ||A(1:, 0)||^2
  {
    double s = 0.0;
    for (int r = 1 + blockIdx.x * GT + tid; r < n; r += G * GT) { const double x = A[r]; s += x * x; }
    s = bsum(s, sh);
    if (tid == 0) P.colp[blockIdx.x] = s;
  }
  if (!grid_sync(P.bar, P.err)) return;
  for (int i = 0; i < n; ++i) {
    // ---- phase 1: column reflector of A(i:, i) from the partials of ||A(i+1:, i)||^2
    {
      const double s = psum(P.colp + (i & 1) * G, G, sh);
      if (tid == 0) {
        double be, ta, scl;
        larfg(A[i + i * ld], s, &be, &ta, &scl);
        sc[0] = be; sc[1] = ta; sc[2] = scl;
      }
      __syncthreads();
    }
    const double tq = sc[1], sq = sc[2];
    if (blockIdx.x == 0 && tid == 0) { P.d[i] = sc[0]; P.tauq[i] = tq; }
    if (i == n - 1) break;
    // ---- pass 1: w_j = v^T A(i:, j), r_j = A(i,j) - tauq w_j, one warp per column;
    //      per-CTA partials of sum r_j^2 and sum w_j r_j over j >= i+2
    {
      double prr = 0.0, pwr = 0.0;
      for (int j = i + 1 + gw; j < n; j += nwarps) {
        const double* col = A + j * ld;
        const double* ci = A + i * ld;
        double s = 0.0;
        for (int r = i + lane; r < n; r += 32) {
          const double vr = (r == i) ? 1.0 : ci[r] * sq;
          s += vr * col[r];
        }
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        const double rb = col[i] - tq * s;
        if (lane == 0) {
          P.w[j] = s;
          P.rowb[j] = rb;
          if (j >= i + 2) { prr += rb * rb; pwr += s * rb; }
        }
      }
      prr = bsum(prr, sh);
      pwr = bsum(pwr, sh);
      if (tid == 0) { P.rowp[blockIdx.x] = prr; P.wup[blockIdx.x] = pwr; }
    }
    if (!grid_sync(P.bar, P.err)) return;
    // ---- phase 2: row reflector of r = rowb(i+1:), and w . u
    {
      const double s = psum(P.rowp, G, sh);
      const double t = psum(P.wup, G, sh);
      if (tid == 0) {
        double be, ta, scl;
        larfg(P.rowb[i + 1], s, &be, &ta, &scl);
        sc[3] = be; sc[4] = ta; sc[5] = scl;
        sc[6] = P.w[i + 1] + scl * t;   // w . u, u = (1, scl * rowb(i+2:))
      }
      __syncthreads();
    }
    const double tp = sc[4], sp = sc[5], wu = sc[6];
    if (blockIdx.x == 0 && tid == 0) { P.e[i] = sc[3]; P.taup[i] = tp; }
    // ---- pass 2: rows r > i, 8 rows per warp; lane = (row r0 + lane % 8,
    //      column phase lane / 8), so each load covers 8 consecutive rows of
    //      4 columns: whole 32-byte sectors of the column-major matrix.  The
    //      lanes of column i+1 also sum the next column norm's partial.
    double cn = 0.0;
    {
      const int ro = lane & 7, co = lane >> 3;
      const int nblk8 = (n - i - 1 + 7) / 8;
      for (int rb = gw; rb < nblk8; rb += nwarps) {
        const int r = i + 1 + rb * 8 + ro;
        const bool live = r < n;
        const double vr = live ? A[r + i * ld] * sq : 0.0;
        double s = 0.0;
        if (live)
          for (int j = i + 1 + co; j < n; j += 4) {
            const double uj = (j == i + 1) ? 1.0 : P.rowb[j] * sp;
            s += A[r + j * ld] * uj;
          }
        s += __shfl_xor_sync(0xffffffffu, s, 8);
        s += __shfl_xor_sync(0xffffffffu, s, 16);
        if (live) {
          const double z = s - tq * vr * wu;
          for (int j = i + 1 + co; j < n; j += 4) {
            const double uj = (j == i + 1) ? 1.0 : P.rowb[j] * sp;
            const double x = A[r + j * ld] - (tq * vr * P.w[j] + tp * z * uj);
            A[r + j * ld] = x;
            if (j == i + 1 && r > i + 1) cn += x * x;
          }
          if (co == 0) A[r + i * ld] = vr;   // the other lanes of this row read A(r, i) above
        }
      }
    }
    cn = bsum(cn, sh);
    if (tid == 0) P.colp[((i + 1) & 1) * G + blockIdx.x] = cn;
    if (blockIdx.x == 0) {   // pivot row: d_i on the diagonal, e_i then u to the right
      for (int j = i + 1 + tid; j < n; j += GT)
        A[i + j * ld] = (j == i + 1) ? sc[3] : P.rowb[j] * sp;
      if (tid == 0) A[i + i * ld] = sc[0];
    }
    if (!grid_sync(P.bar, P.err)) return;
  }
}

}  // namespace

bbt_status gebrd(bbt_ctx* ctx, int n, double* A, double* d, double* e, double* tauq, double* taup) {
  if (n < 2) return fail(ctx, BBT_ERR_ARG, "gebrd: n=%d", n);
  size_t mark = ctx->ws.top;
  BrdArgs P;
  P.n = n;
  P.A = A;
  P.d = d;
  P.e = e;
  P.tauq = tauq;
  P.taup = taup;
  P.w = ctx->ws.take<double>(n);
  P.rowb = ctx->ws.take<double>(n);
  P.colp = ctx->ws.take<double>(2 * 1024);
  P.rowp = ctx->ws.take<double>(1024);
  P.wup = ctx->ws.take<double>(1024);
  if (!P.wup) return fail(ctx, BBT_ERR_NOMEM, "gebrd: workspace");
  P.bar = ctx->d_barrier;
  P.err = ctx->d_flag;
  BBT_CUDA(ctx, cudaMemsetAsync(taup, 0, (size_t)n * sizeof(double), ctx->stream));
  BBT_CUDA(ctx, cudaMemsetAsync(ctx->d_barrier, 0, 2 * sizeof(unsigned), ctx->stream));
  BBT_CUDA(ctx, cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), ctx->stream));
  int per_sm = 0;
  BBT_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gebrd_kernel, GT, 0));
  if (per_sm < 1) return fail(ctx, BBT_ERR_CUDA, "gebrd: kernel does not fit an SM");
  int grid = ctx->num_sms * (per_sm > 2 ? 2 : per_sm);
  if (grid > 1024) grid = 1024;
  if (grid < 1) grid = 1;
  void* args[] = {&P};
  {
    ProfScope prof(ctx, BBT_PROF_RALHA, 4.0 * 8.0 * (double)n * n * n / 3.0);
    BBT_CUDA(ctx, cudaLaunchCooperativeKernel((void*)gebrd_kernel, dim3(grid), dim3(GT), args, 0, ctx->stream));
    BBT_LAUNCHED(ctx);
  }
  int herr = 0;
  BBT_CUDA(ctx, cudaMemcpyAsync(&herr, ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  BBT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->ws.top = mark;
  if (herr) return fail(ctx, BBT_ERR_TIMEOUT, "gebrd: grid barrier timed out");
  return BBT_OK;
}

}  // namespace bbt
