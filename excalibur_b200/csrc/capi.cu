// extern "C" entry points (include/bbtsvd_b200.h): argument checks, context
// and workspace management (the host-buffer and file entries of the pipeline
// are in hostio.cu).  All arithmetic is in the kernels of the other sources.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include "internal.h"

namespace bbt {

cudaError_t Arena::reserve(size_t bytes) {
  if (bytes <= cap) return cudaSuccess;
  if (base) {
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return e;
    cudaFree(base);
    base = nullptr;
    cap = 0;
  }
  cudaError_t e = cudaMalloc(&base, bytes);
  if (e != cudaSuccess) {
    base = nullptr;
    return e;
  }
  cap = bytes;
  top = 0;
  return cudaSuccess;
}

bbt_status fail(bbt_ctx* ctx, bbt_status s, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (ctx) ctx->err = buf;
  return s;
}

bbt_status cuda_fail(bbt_ctx* ctx, cudaError_t e, const char* what) {
  return fail(ctx, e == cudaErrorMemoryAllocation ? BBT_ERR_NOMEM : BBT_ERR_CUDA, "%s: %s", what,
              cudaGetErrorString(e));
}

namespace {

// Scratch for the single-call entries: grow the arena to at least `bytes`.
bbt_status ensure(bbt_ctx* ctx, size_t bytes) {
  ctx->ws.reset();
  if (ctx->ws.cap < bytes) BBT_CUDA(ctx, ctx->ws.reserve(bytes));
  return BBT_OK;
}

bool bad(const void* p) { return p == nullptr || (reinterpret_cast<uintptr_t>(p) & 7) != 0; }

}  // namespace
}  // namespace bbt

using namespace bbt;

extern "C" {

const char* bbt_status_string(bbt_status s) {
  switch (s) {
    case BBT_OK: return "ok";
    case BBT_ERR_ARG: return "invalid argument";
    case BBT_ERR_CUDA: return "CUDA error";
    case BBT_ERR_COUNT: return "fewer singular values than requested";
    case BBT_ERR_NOMEM: return "out of device memory";
    case BBT_ERR_TIMEOUT: return "device-side wait timed out";
    case BBT_ERR_UNSUPPORTED: return "unsupported shape or mode";
    case BBT_ERR_NUMERIC: return "Cholesky breakdown in the mixed-precision local QR";
    case BBT_ERR_IO: return "input file missing, of the wrong size or unreadable";
  }
  return "unknown status";
}

bbt_status bbt_create(bbt_ctx** out, int device) {
  if (!out) return BBT_ERR_ARG;
  *out = nullptr;
  bbt_ctx* ctx = new bbt_ctx();
  ctx->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->own, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_flag, 64);
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_barrier, 64);
  if (e == cudaSuccess) e = cudaMemset(ctx->d_flag, 0, 64);
  if (e == cudaSuccess) e = cudaMemset(ctx->d_barrier, 0, 64);
  if (e != cudaSuccess) {
    fprintf(stderr, "bbt_create: %s\n", cudaGetErrorString(e));
    if (ctx->own) cudaStreamDestroy(ctx->own);
    delete ctx;
    return e == cudaErrorMemoryAllocation ? BBT_ERR_NOMEM : BBT_ERR_CUDA;
  }
  ctx->stream = ctx->own;
  *out = ctx;
  return BBT_OK;
}

bbt_status bbt_destroy(bbt_ctx* ctx) {
  if (!ctx) return BBT_ERR_ARG;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  if (ctx->qr_graph) cudaGraphExecDestroy(ctx->qr_graph);
  for (auto s : ctx->side) cudaStreamDestroy(s);
  for (auto e : ctx->side_ev) cudaEventDestroy(e);
  if (ctx->ws.base) cudaFree(ctx->ws.base);
  if (ctx->d_flag) cudaFree(ctx->d_flag);
  if (ctx->d_barrier) cudaFree(ctx->d_barrier);
  if (ctx->bracket_theta) cudaFree(ctx->bracket_theta);
  if (ctx->io_ws.base) cudaFree(ctx->io_ws.base);
  if (ctx->mask_pinned) cudaFreeHost(ctx->mask_pinned);
  if (ctx->copy_in) cudaStreamDestroy(ctx->copy_in);
  if (ctx->copy_out) cudaStreamDestroy(ctx->copy_out);
  for (auto e : ctx->in_ready) cudaEventDestroy(e);
  for (auto e : ctx->vt_done) cudaEventDestroy(e);
  if (ctx->io_pinned) cudaFreeHost(ctx->io_pinned);
  for (auto e : ctx->io_stage_ev)
    if (e) cudaEventDestroy(e);
  if (ctx->own) cudaStreamDestroy(ctx->own);
  delete ctx;
  return BBT_OK;
}

bbt_status bbt_set_stream(bbt_ctx* ctx, void* stream) {
  if (!ctx) return BBT_ERR_ARG;
  ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own;
  return BBT_OK;
}

bbt_status bbt_synchronize(bbt_ctx* ctx) {
  if (!ctx) return BBT_ERR_ARG;
  BBT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return BBT_OK;
}

const char* bbt_last_error(const bbt_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

uint64_t bbt_kernel_launches(const bbt_ctx* ctx) { return ctx ? ctx->launches : 0; }

bbt_status bbt_negative_count(bbt_ctx* ctx, int n, const double* a, const double* b, const double* mu,
                              int nmu, int* counts) {
  if (!ctx) return BBT_ERR_ARG;
  if (n < 1 || nmu < 0 || bad(a) || (n > 1 && bad(b)) || (nmu > 0 && (bad(mu) || !counts)))
    return fail(ctx, BBT_ERR_ARG, "negative_count: bad arguments");
  BBT_TRY(ensure(ctx, (size_t)n * 16 + (1 << 20)));
  return sturm_counts(ctx, n, a, b, mu, nmu, counts);
}

bbt_status bbt_bisection(bbt_ctx* ctx, int n, const double* a, const double* b, double lo, double hi,
                         double tol, int top_k, double* sigma, int* count) {
  if (!ctx) return BBT_ERR_ARG;
  if (!count) return fail(ctx, BBT_ERR_ARG, "bisection: count is NULL");
  *count = 0;
  if (n < 1 || bad(a) || (n > 1 && bad(b)) || (top_k > 0 && bad(sigma)))
    return fail(ctx, BBT_ERR_ARG, "bisection: bad arguments");
  BBT_TRY(ensure(ctx, bisect_workspace_bytes(n, top_k) + (1 << 20)));
  return bisect(ctx, n, a, b, lo, hi, tol, top_k, sigma, count);
}

bbt_status bbt_bisection_bracketed(bbt_ctx* ctx, int n, const double* a, const double* b, double lo, double hi,
                                   double tol, int top_k, const double* brackets, double* sigma, int* count,
                                   long long* stats) {
  if (!ctx) return BBT_ERR_ARG;
  if (!count) return fail(ctx, BBT_ERR_ARG, "bisection: count is NULL");
  *count = 0;
  if (n < 1 || bad(a) || (n > 1 && bad(b)) || (top_k > 0 && (bad(sigma) || bad(brackets))))
    return fail(ctx, BBT_ERR_ARG, "bisection: bad arguments");
  const int tk = top_k < n ? top_k : n;
  BBT_TRY(ensure(ctx, bisect_workspace_bytes(n, tk) + (size_t)tk * 64 + (1 << 20)));
  long st[4];
  BBT_TRY(bisect(ctx, n, a, b, lo, hi, tol, top_k, sigma, count, brackets, st));
  if (stats) for (int i = 0; i < 4; ++i) stats[i] = st[i];
  return BBT_OK;
}

int bbt_mlp_param_count(void) { return MLP_PARAMS; }

bbt_status bbt_mlp_features(bbt_ctx* ctx, int k, const double* a, const double* b, int count, double* X) {
  if (!ctx) return BBT_ERR_ARG;
  if (k < 1 || count < 0 || count > k || bad(a) || (k > 1 && bad(b)) || (count > 0 && bad(X)))
    return fail(ctx, BBT_ERR_ARG, "mlp_features: bad arguments");
  BBT_TRY(ensure(ctx, 1 << 20));
  double* s6 = ctx->ws.take<double>(8);
  BBT_TRY(mlp_summary(ctx, k, a, b, s6));
  return count > 0 ? mlp_features(ctx, k, count, s6, X) : BBT_OK;
}

bbt_status bbt_mlp_forward(bbt_ctx* ctx, int B, const double* X, const double* theta, double* out) {
  if (!ctx) return BBT_ERR_ARG;
  if (B < 0 || (B > 0 && (bad(X) || bad(theta) || bad(out)))) return fail(ctx, BBT_ERR_ARG, "mlp_forward: bad arguments");
  return mlp_forward(ctx, B, X, theta, out);
}

bbt_status bbt_mlp_grad(bbt_ctx* ctx, int B, const double* X, const double* y, const double* theta, double* grad,
                        double* loss) {
  if (!ctx) return BBT_ERR_ARG;
  if (B < 1 || bad(X) || bad(y) || bad(theta) || bad(grad) || bad(loss))
    return fail(ctx, BBT_ERR_ARG, "mlp_grad: bad arguments");
  BBT_TRY(ensure(ctx, ((size_t)MLP_PARAMS + 2) * B * 8 + (1 << 20)));
  return mlp_grad(ctx, B, X, y, theta, grad, loss);
}

bbt_status bbt_mlp_adam(bbt_ctx* ctx, double* theta, const double* grad, double* m, double* v, double lr, int step) {
  if (!ctx) return BBT_ERR_ARG;
  if (bad(theta) || bad(grad) || bad(m) || bad(v) || step < 1) return fail(ctx, BBT_ERR_ARG, "mlp_adam: bad arguments");
  return mlp_adam(ctx, theta, grad, m, v, lr, step);
}

bbt_status bbt_mlp_brackets(bbt_ctx* ctx, int k, const double* a, const double* b, int count, const double* theta,
                            double z, double* br) {
  if (!ctx) return BBT_ERR_ARG;
  if (k < 1 || count < 1 || count > k || bad(a) || (k > 1 && bad(b)) || bad(theta) || bad(br))
    return fail(ctx, BBT_ERR_ARG, "mlp_brackets: bad arguments");
  BBT_TRY(ensure(ctx, (size_t)count * 8 * 14 + (1 << 20)));
  return mlp_brackets(ctx, k, count, a, b, theta, z, br);
}

bbt_status bbt_set_bracket_model(bbt_ctx* ctx, const double* theta, double z) {
  if (!ctx) return BBT_ERR_ARG;
  BBT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (!theta) {
    if (ctx->bracket_theta) cudaFree(ctx->bracket_theta);
    ctx->bracket_theta = nullptr;
    return BBT_OK;
  }
  if (!(z > 0.0)) return fail(ctx, BBT_ERR_ARG, "set_bracket_model: z must be positive");
  if (!ctx->bracket_theta) BBT_CUDA(ctx, cudaMalloc(&ctx->bracket_theta, MLP_PARAMS * sizeof(double)));
  BBT_CUDA(ctx, cudaMemcpy(ctx->bracket_theta, theta, MLP_PARAMS * sizeof(double), cudaMemcpyHostToDevice));
  ctx->bracket_z = z;
  return BBT_OK;
}

bbt_status bbt_bisection_stats(bbt_ctx* ctx, long long* stats) {
  if (!ctx || !stats) return BBT_ERR_ARG;
  for (int i = 0; i < 4; ++i) stats[i] = ctx->bisect_stats[i];
  return BBT_OK;
}

bbt_status bbt_gebrd(bbt_ctx* ctx, int n, double* A, double* d, double* e) {
  if (!ctx) return BBT_ERR_ARG;
  if (n < 2 || bad(A) || bad(d) || bad(e)) return fail(ctx, BBT_ERR_ARG, "gebrd: bad arguments");
  BBT_TRY(ensure(ctx, (size_t)n * 4 * 8 + (1 << 20)));
  double* tq = ctx->ws.take<double>(n);
  double* tp = ctx->ws.take<double>(n);
  return gebrd(ctx, n, A, d, e, tq, tp);
}

bbt_status bbt_twisted_vectors(bbt_ctx* ctx, int n, int cnt, const double* sigma, const double* a,
                               const double* b, double* U, double* V) {
  if (!ctx) return BBT_ERR_ARG;
  if (n < 1 || cnt < 0 || cnt > n || bad(a) || (n > 1 && bad(b)) || (cnt > 0 && (bad(sigma) || bad(U) || bad(V))))
    return fail(ctx, BBT_ERR_ARG, "twisted_vectors: bad arguments");
  BBT_TRY(ensure(ctx, (size_t)(n + 1) * cnt * 8 * 8 + (size_t)n * 32 + (1 << 20)));
  return twisted(ctx, n, cnt, sigma, a, b, U, cnt, V, false);
}

bbt_status bbt_bidiagonal_svd(bbt_ctx* ctx, int k, const double* a, const double* b, double* U,
                              double* V, double* sigma, int top_k) {
  if (!ctx) return BBT_ERR_ARG;
  if (k < 1 || top_k < 1 || top_k > k || bad(a) || (k > 1 && bad(b)) || bad(U) || bad(V) || bad(sigma))
    return fail(ctx, BBT_ERR_ARG, "bidiagonal_svd: bad arguments (k=%d top_k=%d)", k, top_k);
  BBT_TRY(ensure(ctx, (size_t)(k + 1) * top_k * 8 * 8 + bisect_workspace_bytes(k, top_k) + (2 << 20)));
  return bidiag_svd(ctx, k, a, b, U, V, sigma, top_k, false);
}

bbt_status bbt_givens_mask(bbt_ctx* ctx, size_t m, size_t n, size_t t, double* x, int mask, int is_left,
                           unsigned seed) {
  if (!ctx) return BBT_ERR_ARG;
  if ((m * n > 0 && bad(x)) || t > 4096) return fail(ctx, BBT_ERR_ARG, "givens_mask: bad arguments");
  const size_t k = is_left ? m : n;
  BBT_TRY(ensure(ctx, t * (k + 2) * 24 + (1 << 20)));
  return givens_mask(ctx, m, n, t, x, mask != 0, is_left != 0, seed);
}

bbt_status bbt_block_shift_mask(bbt_ctx* ctx, size_t m, size_t n, size_t t, double* x, int mask,
                                int is_left, unsigned seed) {
  if (!ctx) return BBT_ERR_ARG;
  if ((m * n > 0 && bad(x)) || t > 4096) return fail(ctx, BBT_ERR_ARG, "block_shift_mask: bad arguments");
  const size_t k = is_left ? m : n;
  BBT_TRY(ensure(ctx, 2 * m * n * 8 + 2 * t * (k + 2) * 24 + 2 * (m + n + 20000) * 8 + (4 << 20)));
  return block_shift_mask(ctx, m, n, t, x, mask != 0, is_left != 0, seed);
}

bbt_status bbt_local_qr(bbt_ctx* ctx, size_t m, size_t local_n, double* x, double* rt, int compute_q) {
  if (!ctx) return BBT_ERR_ARG;
  if (m < 1 || local_n <= m || bad(x) || bad(rt) || local_n > (size_t)1 << 31)
    return fail(ctx, BBT_ERR_ARG, "local_qr: needs local_n > m (client.cpp:419)");
  QrPlan qp;
  const size_t tq = ((m + qp.nb - 1) / qp.nb) * qp.nb * qp.nb;
  BBT_TRY(ensure(ctx, qr_workspace_bytes((long)local_n, (int)m, (int)m, qp) + (tq + m) * 8 + (4 << 20)));
  double* tau = ctx->ws.take<double>(m);
  double* T = ctx->ws.take<double>(tq);
  const long n = (long)local_n;
  BBT_TRY(geqrf(ctx, n, (int)m, x, n, tau, T, qp));
  BBT_TRY(r_transpose(ctx, (int)m, x, n, rt));   // the reference's shrinked_x (client.cpp:437-442)
  if (compute_q) BBT_TRY(orgqr(ctx, n, (int)m, x, n, tau, T, qp));
  return BBT_OK;
}

bbt_status bbt_fedsvd_run(bbt_ctx* ctx, const bbt_fedsvd_config* cfg, double* const* blocks,
                          double* sigma, double* U, double* const* VT, int* k) {
  if (!ctx) return BBT_ERR_ARG;
  if (!cfg || !blocks || !k || bad(sigma)) return fail(ctx, BBT_ERR_ARG, "fedsvd: NULL argument");
  const bool want_u = cfg->svd_mode != 3 && cfg->svd_mode != 4, want_v = cfg->svd_mode != 2;
  if (cfg->svd_mode == 4 && bad(cfg->labels)) return fail(ctx, BBT_ERR_ARG, "fedsvd: svd_mode 4 labels");
  if ((want_u && bad(U)) || (want_v && !VT)) return fail(ctx, BBT_ERR_ARG, "fedsvd: NULL output");
  for (int c = 0; c < cfg->participants; ++c)
    if (bad(blocks[c]) || (want_v && bad(VT[c]))) return fail(ctx, BBT_ERR_ARG, "fedsvd: participant %d buffer", c);
  return fedsvd(ctx, cfg, blocks, sigma, U, VT, k);
}

bbt_status bbt_dgemm(bbt_ctx* ctx, int transa, int transb, int M, int N, long K, double alpha, const double* A,
                     long lda, const double* B, long ldb, double beta, double* C, long ldc) {
  if (!ctx) return BBT_ERR_ARG;
  if (M < 0 || N < 0 || K < 0 || (M > 0 && N > 0 && (bad(C) || (K > 0 && (bad(A) || bad(B))))))
    return fail(ctx, BBT_ERR_ARG, "dgemm: bad arguments");
  const long am = transa ? K : M, bm = transb ? N : K;
  if (lda < (am > 1 ? am : 1) || ldb < (bm > 1 ? bm : 1) || ldc < (M > 1 ? M : 1))
    return fail(ctx, BBT_ERR_ARG, "dgemm: leading dimension too small");
  BBT_TRY(ensure(ctx, dgemm_workspace_bytes(ctx, M, N, K) + (1 << 20)));
  return dgemm(ctx, transa != 0, transb != 0, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
}

bbt_status bbt_dgemm_ozaki(bbt_ctx* ctx, int transa, int transb, int M, int N, long K, double alpha, const double* A,
                           long lda, const double* B, long ldb, double beta, double* C, long ldc, int upper) {
  if (!ctx) return BBT_ERR_ARG;
  if (M < 1 || N < 1 || K < 1 || bad(A) || bad(B) || bad(C) || (upper && M != N))
    return fail(ctx, BBT_ERR_ARG, "dgemm_ozaki: bad arguments");
  const long am = transa ? K : M, bm = transb ? N : K;
  if (lda < am || ldb < bm || ldc < M) return fail(ctx, BBT_ERR_ARG, "dgemm_ozaki: leading dimension too small");
  BBT_TRY(ensure(ctx, oz_workspace_bytes(ctx, M, N, K, false) + (1 << 20)));
  BBT_TRY(clear_tc_flags(ctx));
  const long rsA = transa ? lda : 1, csA = transa ? 1 : lda;
  const long rsB = transb ? 1 : ldb, csB = transb ? ldb : 1;
  BBT_TRY(gemm_oz(ctx, M, N, K, alpha, A, rsA, csA, B, rsB, csB, beta, C, ldc, false, upper != 0));
  return check_tc_flags(ctx, "dgemm_ozaki");
}

bbt_status bbt_dgemm_crt(bbt_ctx* ctx, int M, int N, long K, double alpha, const double* A, long lda, const double* B,
                         long ldb, double beta, double* C, long ldc, int bits) {
  if (!ctx) return BBT_ERR_ARG;
  if (M < 1 || N < 1 || K < 1 || bad(A) || bad(B) || bad(C) || lda < K || ldb < K || ldc < M || bits < 8 || bits > 53)
    return fail(ctx, BBT_ERR_ARG, "dgemm_crt: bad arguments");
  const int n = crt_moduli(bits, bits, K);
  if (n < 1) return fail(ctx, BBT_ERR_ARG, "dgemm_crt: %d bits over K=%ld", bits, K);
  const long Kp = crt_pitch(K);
  BBT_TRY(ensure(ctx, (size_t)n * (M + N) * Kp + crt_product_bytes(ctx, M, N, K, n, false) + (size_t)(M + N) * 16 +
                          (4 << 20)));
  BBT_TRY(clear_tc_flags(ctx));
  BBT_TRY(gemm_crt(ctx, M, N, K, alpha, A, lda, 1, B, ldb, 1, beta, C, ldc, false, false, bits));
  return check_tc_flags(ctx, "dgemm_crt");
}

bbt_status bbt_gram_dd(bbt_ctx* ctx, int m, long n, const double* X, long ldx, double* Gh, double* Gl) {
  if (!ctx) return BBT_ERR_ARG;
  if (m < 1 || n < 1 || bad(X) || bad(Gh) || bad(Gl) || ldx < n) return fail(ctx, BBT_ERR_ARG, "gram_dd: bad arguments");
  if (crt_moduli(53, 53, n) < 1) return fail(ctx, BBT_ERR_ARG, "gram_dd: n=%ld too long", n);
  BBT_TRY(ensure(ctx, exact_gram_workspace_bytes(ctx, m, n) + (size_t)m * 16 + (4 << 20)));
  BBT_TRY(clear_tc_flags(ctx));
  double* s = ctx->ws.take<double>(m);
  if (!s) return fail(ctx, BBT_ERR_NOMEM, "gram_dd: workspace");
  BBT_TRY(exact_gram_dd(ctx, m, n, X, ldx, s, nullptr, Gh, Gl));
  return check_tc_flags(ctx, "gram_dd");
}

bbt_status bbt_exact_local_qr(bbt_ctx* ctx, int m, size_t local_n, const double* x, double* R, double* W, double* Rp,
                              double* scale) {
  if (!ctx) return BBT_ERR_ARG;
  if (m < 2 || local_n < (size_t)m || local_n > ((size_t)1 << 31) || bad(x) || bad(R) || bad(W) || bad(Rp) ||
      bad(scale))
    return fail(ctx, BBT_ERR_ARG, "exact_local_qr: bad arguments");
  const int mi = m, N = sketch_rows(mi);
  const long pitch = sketch_pitch((long)local_n);
  const size_t sbytes = (size_t)N * pitch * 2 + 256;
  BBT_TRY(ensure(ctx, exact_qr_workspace_bytes(ctx, mi, (long)local_n) + sbytes + (16 << 20)));
  void* S = ctx->ws.take<char>(sbytes);
  BBT_TRY(rademacher(ctx, N, (long)local_n, S, 0x5EED5EEDull));
  BBT_TRY(clear_tc_flags(ctx));
  BBT_TRY(exact_local_qr(ctx, mi, (long)local_n, x, S, pitch, R, W, Rp, scale));
  return check_tc_flags(ctx, "exact_local_qr");
}

bbt_status bbt_exact_apply_q(bbt_ctx* ctx, int m, size_t rows, const double* x, long ldx, const double* scale,
                             const double* Rp, const double* Z, int k, double* C, long ldc) {
  if (!ctx) return BBT_ERR_ARG;
  if (m < 2 || rows < 1 || rows > ((size_t)1 << 31) || k < 1 || k > 65535 || ldx < (long)rows || ldc < (long)rows ||
      bad(x) || bad(scale) || bad(Rp) || bad(Z) || bad(C))
    return fail(ctx, BBT_ERR_ARG, "exact_apply_q: bad arguments");
  BBT_TRY(ensure(ctx, exact_apply_workspace_bytes(ctx, (long)rows, m, k) + (16 << 20)));
  BBT_TRY(clear_tc_flags(ctx));
  BBT_TRY(exact_apply_q(ctx, m, (long)rows, x, ldx, scale, Rp, Z, k, C, ldc));
  return check_tc_flags(ctx, "exact_apply_q");
}

bbt_status bbt_rademacher(bbt_ctx* ctx, int N, size_t local_n, unsigned long long seed, void* d_S) {
  if (!ctx) return BBT_ERR_ARG;
  if (N < 1 || local_n < 1 || local_n > ((size_t)1 << 31) || bad(d_S))
    return fail(ctx, BBT_ERR_ARG, "rademacher: bad arguments");
  return rademacher(ctx, N, (long)local_n, d_S, seed);
}

bbt_status bbt_sketch_bf16x3(bbt_ctx* ctx, int m, size_t local_n, const double* d_x, int N, const void* d_S,
                             double* d_Y) {
  if (!ctx) return BBT_ERR_ARG;
  if (m < 1 || local_n < 1 || local_n > ((size_t)1 << 31) || N < 128 || N % 128 != 0 || bad(d_x) || bad(d_S) ||
      bad(d_Y))
    return fail(ctx, BBT_ERR_ARG, "sketch: bad arguments (N must be a positive multiple of 128)");
  BBT_TRY(ensure(ctx, sketch_workspace_bytes(ctx, m, (long)local_n, N) + (1 << 20)));
  BBT_TRY(clear_tc_flags(ctx));
  BBT_TRY(sketch_bf16x3(ctx, m, (long)local_n, d_x, (long)local_n, N, d_S, sketch_pitch((long)local_n), d_Y));
  return check_tc_flags(ctx, "sketch");
}

bbt_status bbt_mixed_local_qr(bbt_ctx* ctx, size_t m, size_t local_n, double* d_x, double* d_r, double* d_w) {
  if (!ctx) return BBT_ERR_ARG;
  if (m < 1 || local_n <= m || local_n > ((size_t)1 << 31) || m > 65536 || bad(d_x) || bad(d_r))
    return fail(ctx, BBT_ERR_ARG, "mixed_local_qr: needs local_n > m");
  const int mi = (int)m, N = sketch_rows(mi);
  const long n = (long)local_n;
  BBT_TRY(ensure(ctx, mixed_qr_workspace_bytes(ctx, mi, n) + (size_t)N * sketch_pitch(n) * 2 + (1 << 20)));
  void* S = ctx->ws.take<char>((size_t)N * sketch_pitch(n) * 2);
  BBT_TRY(rademacher(ctx, N, n, S, 0x5EED5EEDull));
  BBT_TRY(clear_tc_flags(ctx));
  BBT_TRY(mixed_local_qr(ctx, mi, n, d_x, S, sketch_pitch(n), d_r, d_w));
  return check_tc_flags(ctx, "mixed_local_qr");
}

bbt_status bbt_profile(bbt_ctx* ctx, int enable) {
  if (!ctx) return BBT_ERR_ARG;
  BBT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (auto& r : ctx->recs) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
  ctx->recs.clear();
  for (int i = 0; i < BBT_PROF_CLASSES; ++i) { ctx->prof_ms[i] = 0; ctx->prof_work[i] = 0; ctx->prof_n[i] = 0; }
  ctx->prof = enable != 0;
  return BBT_OK;
}

bbt_status bbt_profile_get(bbt_ctx* ctx, int cls, double* ms, uint64_t* launches, double* work) {
  if (!ctx || cls < 0 || cls >= BBT_PROF_CLASSES) return BBT_ERR_ARG;
  BBT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (auto& r : ctx->recs) {
    float t = 0;
    BBT_CUDA(ctx, cudaEventElapsedTime(&t, r.a, r.b));
    ctx->prof_ms[r.cls] += t;
    ctx->prof_n[r.cls] += 1;
    ctx->prof_work[r.cls] += r.work;
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  ctx->recs.clear();
  if (ms) *ms = ctx->prof_ms[cls];
  if (launches) *launches = ctx->prof_n[cls];
  if (work) *work = ctx->prof_work[cls];
  return BBT_OK;
}

bbt_status bbt_fedsvd_tune(bbt_ctx* ctx, const bbt_fedsvd_config* cfg, int* streams, int* nb, double* ms) {
  if (!ctx) return BBT_ERR_ARG;
  if (!cfg) return fail(ctx, BBT_ERR_ARG, "fedsvd_tune: NULL config");
  return fedsvd_tune(ctx, cfg, streams, nb, ms);
}

bbt_status bbt_svd_dense(bbt_ctx* ctx, int m, double* X, int top_k, double* sigma, double* U, double* VT,
                         int* k) {
  if (!ctx) return BBT_ERR_ARG;
  if (!k || m < 1 || bad(X) || bad(sigma) || bad(U) || bad(VT)) return fail(ctx, BBT_ERR_ARG, "svd_dense: bad arguments");
  return svd_dense(ctx, m, X, top_k, sigma, U, VT, k);
}

bbt_status bbt_fedsvd_stage_ms(const bbt_ctx* ctx, double* ms, int n) {
  if (!ctx || !ms || n < 6) return BBT_ERR_ARG;
  for (int i = 0; i < 6; ++i) ms[i] = ctx->stage_ms[i];
  return BBT_OK;
}

}  // extern "C"
