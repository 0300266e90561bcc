// Mixed-precision local QR of a wide participant block (the split-precision
// replacement of client.cpp:417-445's dgeqrf/dorgqr), for precision mode 1.
//
// A = X_c^T (n x m, column-major; n >> m).  The R factor is built by
// sketch-preconditioned Cholesky QR:
//   1. sketch Y = S A (N x m, N = 2m rounded up to 128, S a +-1 Rademacher
//      matrix) as a BF16x3 product on the tensor cores (sketch.cu);
//   2. R_p = chol(Y^T Y + shift) in FP64 -- a preconditioner: Q_p = A R_p^{-1}
//      has condition number ~ (1 + sqrt(m/N)) / (1 - sqrt(m/N)) times
//      (1 + (sketch error) cond(A)), small for cond(A) up to ~1e7;
//   3. FP64 refinement pass: Q_p = A R_p^{-1} (triangular solve), G = Q_p^T
//      Q_p, R_3 = chol(G), R = R_3 R_p, and Q = Q_p R_3^{-1} is orthonormal
//      to ~ eps cond(Q_p)^2.
// Only step 1 runs in split precision; the Gram matrix, the Cholesky factors
// and the solve that define R are FP64, so R is the R factor of A to FP64
// accuracy (up to the signs of its rows: R has a positive diagonal, which the
// rest of the pipeline does not depend on).  Q is kept implicitly as Q_p
// (overwriting X_c) and W = R_3^{-1}; the V back-transform multiplies by
// Q_p W instead of the explicit Q of dorgqr.
//   4. the row signs of dgeqrf's R are recovered from the top m x m block of
//      Q (householder_signs, chol.cu) and applied to R and W, so the rest of
//      the pipeline -- whose sign convention is applied in the basis these
//      signs define (client.cpp:988-995) -- reproduces the reference's
//      vectors, not only their subspaces.
#include <cuda_runtime.h>

#include <algorithm>

#include "internal.h"

namespace bbt {

constexpr int GRAM_BITS = 50;   // rows of Q_p rounded to 50 bits for the CRT Gram (15 moduli at c2's sizes)

bbt_status clear_tc_flags(bbt_ctx* ctx) {
  BBT_CUDA(ctx, cudaMemsetAsync(ctx->d_flag + FLAG_SKETCH, 0, 2 * sizeof(int), ctx->stream));
  return BBT_OK;
}

bbt_status check_tc_flags(bbt_ctx* ctx, const char* what) {
  int h[2] = {0, 0};
  BBT_CUDA(ctx, cudaMemcpyAsync(h, ctx->d_flag + FLAG_SKETCH, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
  BBT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (h[0]) return fail(ctx, BBT_ERR_TIMEOUT, "%s: a device wait gave up (code %d)", what, h[0]);
  if (h[1]) return fail(ctx, BBT_ERR_NUMERIC, "%s: Cholesky pivot not positive (rank-deficient block?)", what);
  return BBT_OK;
}

size_t mixed_qr_workspace_bytes(const bbt_ctx* ctx, int m, long n) {
  const int N = sketch_rows(m);
  size_t s = sketch_workspace_bytes(ctx, m, n, N);
  s = std::max(s, dgemm_workspace_bytes(ctx, m, m, n));
  s = std::max(s, dgemm_workspace_bytes(ctx, m, m, N));
  s = std::max(s, oz_workspace_bytes(ctx, m, m, n, true));                   // Gram
  s = std::max(s, crt_gemm_workspace_bytes(ctx, m, m, n, GRAM_BITS, true, true));
  s = std::max(s, oz_workspace_bytes(ctx, (int)n, m - (m / 2 + 31) / 32 * 32, (m / 2 + 31) / 32 * 32, false));
  return s + ((size_t)N * m + 3 * (size_t)m * m + m) * 8 + 8192;
}

bbt_status mixed_local_qr(bbt_ctx* ctx, int m, long n, double* X, const void* S, long spitch, double* R,
                          double* W) {
  const int N = sketch_rows(m);
  const size_t mark = ctx->ws.top;
  double* Y = ctx->ws.take<double>((size_t)N * m);
  double* Gp = ctx->ws.take<double>((size_t)m * m);
  double* G = ctx->ws.take<double>((size_t)m * m);
  double* Wl = W ? W : ctx->ws.take<double>((size_t)m * m);
  double* dsig = ctx->ws.take<double>(m);
  if (!dsig) return fail(ctx, BBT_ERR_NOMEM, "mixed local QR: workspace");
  int* flag = ctx->d_flag + FLAG_CHOL;
  // 1. Y^T (m x N row-major) = X S^T  ==  Y = S A (N x m column-major)
  BBT_TRY(sketch_bf16x3(ctx, m, n, X, n, N, S, spitch, Y));
  // 2. R_p = chol(Y^T Y + 1e-14 max diag)
  BBT_TRY(dgemm(ctx, true, false, m, m, N, 1.0, Y, N, Y, N, 0.0, Gp, m, 0, true));
  BBT_TRY(symmetrize_upper(ctx, m, Gp, m));
  BBT_TRY(shift_diag(ctx, m, Gp, m, 1e-14));
  BBT_TRY(potrf_upper(ctx, m, Gp, m, flag));
  // 3. Q_p = A R_p^{-1} (in place), G = Q_p^T Q_p, R_3 = chol(G), R = R_3 R_p; the large
  //    products from exact int8 slices on the tensor cores (ozaki.cu), FP64-accurate
  BBT_TRY(trsm_right_upper(ctx, n, m, Gp, m, X, n, true));
  if (crt_worthwhile(m, m, n))   // exact product of 50-bit rows (crt.cu): errors ~2^-50 relative, as R needs
    BBT_TRY(gemm_crt(ctx, m, m, n, 1.0, X, n, 1, X, n, 1, 0.0, G, m, true, true, GRAM_BITS));
  else if (oz_worthwhile(m, m, n))   // 7 slices: the Gram's errors act on R multiplicatively (~2^-50 relative)
    BBT_TRY(gemm_oz(ctx, m, m, n, 1.0, X, n, 1, X, n, 1, 0.0, G, m, true, true, 7));
  else
    BBT_TRY(dgemm(ctx, true, false, m, m, n, 1.0, X, n, X, n, 0.0, G, m, 0, true));
  BBT_TRY(symmetrize_upper(ctx, m, G, m));
  BBT_TRY(potrf_upper(ctx, m, G, m, flag));
  BBT_TRY(dgemm(ctx, false, false, m, m, m, 1.0, G, m, Gp, m, 0.0, R, m));
  // 4. W = R_3^{-1}, so Q = Q_p W
  BBT_TRY(identity(ctx, m, Wl, m));
  BBT_TRY(trsm_right_upper(ctx, m, m, G, m, Wl, m));
  // 5. dgeqrf's row signs: from the top m x m block of Q (Gp is free again)
  BBT_TRY(dgemm(ctx, false, false, m, m, m, 1.0, X, n, Wl, m, 0.0, Gp, m));
  BBT_TRY(householder_signs(ctx, m, m, Gp, m, dsig));
  BBT_TRY(apply_signs(ctx, m, dsig, R, W));
  ctx->ws.top = mark;
  return BBT_OK;
}

}  // namespace bbt
