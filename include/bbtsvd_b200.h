/*
 * bbtsvd_b200.h — C ABI of the B200 (sm_100a) implementation of Excalibur's
 * matrix-factorisation hot path.
 *
 * Two layers:
 *   1. The reference's own C++ API (Excalibur include/bbtsvd.hpp:22-47) is
 *      exported with identical mangled signatures by libexcalibur_b200.so
 *      (host pointers in, host pointers out), so the reference's
 *      DecentralizedClient links it in place of src/bbtsvd.cpp.
 *   2. This header: extern "C", device pointers, stream-ordered, every call
 *      returns a bbt_status instead of asserting.  The entries for the math
 *      that the reference keeps inline in DecentralizedClient::run()
 *      (local QR, global QR, Ralha bidiagonalisation, back-transforms) and
 *      a whole-pipeline entry for P participants held as separate device
 *      buffers on one GPU are additions with a cited reference site each.
 *
 * Layout conventions follow the reference: "row-major m x n" means element
 * (i, j) at x[i*n + j]; a participant's block is row-major m x local_n.
 * Device pointers must be 8-byte aligned.  A bbt_ctx owns one CUDA stream
 * (or borrows the caller's), a device workspace and the last error text; it
 * is not thread-safe — use one context per host thread.
 */
#ifndef BBTSVD_B200_H
#define BBTSVD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  BBT_OK = 0,
  BBT_ERR_ARG = 1,          /* invalid size / pointer / option */
  BBT_ERR_CUDA = 2,         /* a CUDA runtime call failed */
  BBT_ERR_COUNT = 3,        /* bisection found fewer singular values than requested
                               (the reference asserts here, bbtsvd.cpp:938) */
  BBT_ERR_NOMEM = 4,        /* device allocation failed */
  BBT_ERR_TIMEOUT = 5,      /* a bounded device-side wait gave up */
  BBT_ERR_UNSUPPORTED = 6,  /* shape or mode outside what the reference supports */
  BBT_ERR_NUMERIC = 7,      /* a Cholesky pivot of the mixed-precision local QR was not
                               positive (rank-deficient block); rerun with precision 0 */
  BBT_ERR_IO = 8            /* an input file is missing, of the wrong size or unreadable */
} bbt_status;

typedef struct bbt_ctx bbt_ctx;

/* ---- context ----------------------------------------------------------- */
bbt_status bbt_create(bbt_ctx** ctx, int device);
bbt_status bbt_destroy(bbt_ctx* ctx);
/* Borrow a cudaStream_t (passed as void*); NULL restores the context's own. */
bbt_status bbt_set_stream(bbt_ctx* ctx, void* stream);
bbt_status bbt_synchronize(bbt_ctx* ctx);
const char* bbt_last_error(const bbt_ctx* ctx);
const char* bbt_status_string(bbt_status s);
/* Kernels launched by this context since creation (all are this library's). */
uint64_t bbt_kernel_launches(const bbt_ctx* ctx);

/* ---- bidiagonal SVD (Excalibur src/bbtsvd.cpp) ---------------------------
 * alpha[n] is the diagonal, beta[n-1] the superdiagonal of an upper
 * bidiagonal B.                                                             */

/* Sturm count of B^T B - mu^2 I for nmu shifts: counts[i] = number of
 * negative pivots at mu[i].  Replaces negative_count, bbtsvd.cpp:7-17. */
bbt_status bbt_negative_count(bbt_ctx* ctx, int n, const double* d_alpha, const double* d_beta,
                              const double* d_mu, int nmu, int* d_counts);

/* Singular values in (lo, hi] by the reference's bisection tree (upper half
 * first, stop when the midpoint no longer splits the interval or the width
 * is <= tol), at most top_k, descending; *h_count receives how many.
 * Replaces bisection_singular_values, bbtsvd.cpp:19-52. */
bbt_status bbt_bisection(bbt_ctx* ctx, int n, const double* d_alpha, const double* d_beta,
                         double lo, double hi, double tol, int top_k, double* d_sigma,
                         int* h_count);

/* Twisted-factorisation singular vectors for cnt singular values:
 * v_i -> row i of d_V (cnt x n), u_i -> column i of d_U (n x cnt).
 * Replaces two_side_singular_vectors_twisted_factorization,
 * bbtsvd.cpp:138-147. */
bbt_status bbt_twisted_vectors(bbt_ctx* ctx, int n, int cnt, const double* d_sigma,
                               const double* d_alpha, const double* d_beta, double* d_U,
                               double* d_V);

/* Top-k bisection + twisted vectors + the reference's sign fixes.
 * d_U: k x top_k row-major, d_V: top_k x k row-major, d_sigma: top_k.
 * Replaces bidiagonal_bisection_twisted_svd (top-k overload),
 * bbtsvd.cpp:932-968. */
bbt_status bbt_bidiagonal_svd(bbt_ctx* ctx, int k, const double* d_alpha, const double* d_beta,
                              double* d_U, double* d_V, double* d_sigma, int top_k);

/* bbt_twisted_vectors for callers that must not allocate device memory (an
 * allocation-free hot loop, memory handed in full to another allocator, a
 * zero allocation budget).  No counterpart in the reference: an addition.
 * Takes a cudaStream_t (as void*; NULL = the default stream) of the current
 * device (another device's stream returns BBT_ERR_ARG) instead of a context
 * and keeps its work arrays in one static 64 MiB __device__ array that every
 * GPU loading the library holds until exit.  Needs 2n + 6(n+1)cnt + n*cnt
 * doubles of it (each of its arrays rounded up to 256 bytes; n = cnt = 1094
 * fits, 1095 does not); larger shapes return BBT_ERR_ARG with a message on
 * stderr.  The first call in each CUDA context looks up the array's device
 * address (cudaGetSymbolAddress, with that device current), and again after
 * the context is recreated (cudaDeviceReset); make that first call before
 * any stream capture.  All calls share the array and
 * it keeps the last call's contents (every work array is written before it
 * is read, so nothing needs clearing); calls that overlap on the GPU race.
 * Same results as bbt_twisted_vectors. */
bbt_status bbt_twisted_vectors_noalloc(void* stream, int n, int cnt, const double* d_sigma,
                                       const double* d_alpha, const double* d_beta, double* d_U,
                                       double* d_V);

/* ---- data masks (Excalibur src/bbtsvd.cpp) --------------------------------
 * The random tables are drawn on the host with the reference's own calls
 * (srand(seed), std::default_random_engine(seed), std::shuffle, rand()), so
 * the result equals the reference's bit for bit and glibc's rand() state is
 * left as the reference leaves it.                                          */

/* Replaces givens_mask_cache_optimized_parallel_with_simd,
 * bbtsvd.cpp:727-876.  In place on d_x (row-major m x n). */
bbt_status bbt_givens_mask(bbt_ctx* ctx, size_t m, size_t n, size_t mask_times, double* d_x,
                           int mask, int is_left, unsigned seed);

/* Replaces block_shift_mask, bbtsvd.cpp:533-669 (direct path for a rotated
 * dimension <= 10000, near-square virtual-matrix path above it). */
bbt_status bbt_block_shift_mask(bbt_ctx* ctx, size_t m, size_t n, size_t mask_times, double* d_x,
                                int mask, int is_left, unsigned seed);

/* ---- QR (Excalibur src/client.cpp) ----------------------------------------
 * Householder QR of A = X^T, X row-major m x local_n (so A is column-major
 * local_n x m, local_n >= m).  d_rt receives R^T (row-major m x m, lower
 * triangular: the reference's shrinked_x).  With compute_q, d_x is
 * overwritten by Q^T (row-major m x local_n; the reference's local_v);
 * otherwise d_x holds the Householder vectors.
 * Replaces DecentralizedClient::local_qr_reduction, client.cpp:417-445. */
bbt_status bbt_local_qr(bbt_ctx* ctx, size_t m, size_t local_n, double* d_x, double* d_rt,
                        int compute_q);

/* ---- FP64 GEMM ------------------------------------------------------------
 * Column-major BLAS convention: C = alpha op(A) op(B) + beta C, op(A) M x K,
 * op(B) K x N (trans: 0 = 'N', 1 = 'T').  On the FP64 tensor path (DMMA).
 * Replaces the cblas_dgemm calls of the back-transforms, client.cpp:1011,
 * 1018, 1179, 1190. */
bbt_status bbt_dgemm(bbt_ctx* ctx, int transa, int transb, int M, int N, long K, double alpha,
                     const double* d_A, long lda, const double* d_B, long ldb, double beta,
                     double* d_C, long ldc);

/* ---- learned bisection brackets -------------------------------------------
 * A small MLP (parameters: bbt_mlp_param_count() doubles) maps per-bidiagonal
 * features (norms of a and b, their maxima, min |a|, dimension) and the index
 * fraction of the j-th largest singular value to (mu, ell): a centre log2
 * (sigma_j / g), g = max_i(|a_i| + max(|b_{i-1}|, |b_i|)), and a log spread.
 * Training runs on the device through these entries (features, forward,
 * per-batch gradient of the Gaussian negative log-likelihood, Adam).
 * bbt_mlp_brackets: br[2j], br[2j+1] = g 2^(mu -/+ z e^ell) for j < count.
 * bbt_bisection_bracketed: bbt_bisection with such brackets.  Each bracket
 * is snapped to a node of the reference's bisection tree; once the bisection
 * has isolated that value in an interval strictly containing the node, two
 * exact Sturm counts verify the node and the interval jumps to it (skipping
 * the levels in between); a node that fails is ignored.  The result is
 * bit-identical to bbt_bisection; stats (may be NULL) = {Sturm evaluations
 * (verification included), rounds, jumps taken, verification evaluations}.
 * bbt_set_bracket_model: use these parameters (host array, copied; NULL
 * turns the model off) inside bbt_bidiagonal_svd, bbt_fedsvd_run and
 * bbt_svd_dense; bbt_bisection_stats reports the stats of the last
 * bisection run by those.
 * bbt_gebrd: Householder bidiagonalisation (diagonal d, superdiagonal e) of a
 * dense column-major n x n matrix (overwritten), to generate training data.
 * Additive: the reference's bisection has no learned part (bbtsvd.cpp:19-52). */
int bbt_mlp_param_count(void);
bbt_status bbt_mlp_features(bbt_ctx* ctx, int k, const double* d_a, const double* d_b, int count, double* d_X);
bbt_status bbt_mlp_forward(bbt_ctx* ctx, int batch, const double* d_X, const double* d_theta, double* d_out);
bbt_status bbt_mlp_grad(bbt_ctx* ctx, int batch, const double* d_X, const double* d_y, const double* d_theta,
                        double* d_grad, double* d_loss);
bbt_status bbt_mlp_adam(bbt_ctx* ctx, double* d_theta, const double* d_grad, double* d_m, double* d_v, double lr,
                        int step);
bbt_status bbt_mlp_brackets(bbt_ctx* ctx, int k, const double* d_a, const double* d_b, int count,
                            const double* d_theta, double z, double* d_brackets);
bbt_status bbt_bisection_bracketed(bbt_ctx* ctx, int n, const double* d_alpha, const double* d_beta, double lo,
                                   double hi, double tol, int top_k, const double* d_brackets, double* d_sigma,
                                   int* count, long long* stats);
bbt_status bbt_set_bracket_model(bbt_ctx* ctx, const double* theta, double z);
bbt_status bbt_bisection_stats(bbt_ctx* ctx, long long* stats);
bbt_status bbt_gebrd(bbt_ctx* ctx, int n, double* d_A, double* d_d, double* d_e);

/* ---- split-precision sketch and mixed-precision local QR -----------------
 * bbt_rademacher: d_S (N x local_n bf16, row pitch round_up(local_n, 8)
 * elements) <- independent +-1 entries drawn from `seed`.
 * bbt_sketch_bf16x3: d_Y (row-major m x N, FP64) = X S^T for X row-major
 * m x local_n FP64, as three bf16 pieces of X times the exact bf16 S on the
 * tensor cores (tcgen05, FP32 accumulation per K-chunk, FP64 across chunks).
 * N must be a multiple of 128.
 * bbt_mixed_local_qr: the precision-1 local QR.  d_x (row-major m x
 * local_n, local_n > m) is overwritten by Q_p^T, d_r receives R (m x m
 * column-major, upper triangular with dgeqrf's row signs; equal as memory to
 * the row-major R^T of bbt_local_qr), d_w (may be NULL) receives W (m x m
 * column-major) with Q = Q_p W orthonormal and A = X^T = Q R.
 * Additive: the reference has no split-precision path (its local QR is
 * client.cpp:417-445). */
bbt_status bbt_rademacher(bbt_ctx* ctx, int N, size_t local_n, unsigned long long seed, void* d_S);
/* bbt_dgemm_ozaki: bbt_dgemm's contract (column-major, op = 'N'/'T') computed
 * from exact int8 slices on the tensor cores (tcgen05 kind::i8): each row of
 * op(A) and column of op(B) is scaled by a power of two and split into 8
 * slices of at most 7 bits (rounded to nearest); the 36 slice pairs with
 * p + q < 8 are accumulated exactly in int32 and combined in FP64, accurate
 * to ~2^-56 of the row and column scales per term.  upper (M == N): only the tiles touching the upper
 * triangle of C are computed, the rest of C is left as it was. */
bbt_status bbt_dgemm_ozaki(bbt_ctx* ctx, int transa, int transb, int M, int N, long K, double alpha,
                           const double* d_A, long lda, const double* d_B, long ldb, double beta,
                           double* d_C, long ldc, int upper);
bbt_status bbt_sketch_bf16x3(bbt_ctx* ctx, int m, size_t local_n, const double* d_x, int N,
                             const void* d_S, double* d_Y);
bbt_status bbt_mixed_local_qr(bbt_ctx* ctx, size_t m, size_t local_n, double* d_x, double* d_r,
                              double* d_w);

/* ---- kernel profiling -------------------------------------------------------
 * With profiling on, every launch of the library's kernels of a class is
 * bracketed by CUDA events on the launching stream.  bbt_profile_get
 * (synchronises) returns, per class, the summed event time, the number of
 * launches and the algorithmic work (flops for BBT_PROF_DGEMM and
 * BBT_PROF_PANEL, bytes moved for BBT_PROF_MASK) since profiling was
 * switched on. */
enum { BBT_PROF_DGEMM = 0, BBT_PROF_PANEL = 1, BBT_PROF_MASK = 2, BBT_PROF_RALHA = 3,
       BBT_PROF_BISECT = 4, BBT_PROF_TWISTED = 5, BBT_PROF_SKETCH = 6, BBT_PROF_CHOL = 7,
       BBT_PROF_OZAKI = 8, BBT_PROF_CRT = 9, BBT_PROF_CRT_PREP = 10, BBT_PROF_CRT_COMBINE = 11,
       BBT_PROF_DD = 12, BBT_PROF_CLASSES = 13 };
bbt_status bbt_profile(bbt_ctx* ctx, int enable);
bbt_status bbt_profile_get(bbt_ctx* ctx, int cls, double* ms, uint64_t* launches, double* work);

/* ---- dense SVD ---------------------------------------------------------------
 * SVD X = U diag(sigma) VT of one dense m x m matrix (row-major,
 * overwritten): two-sided Householder bidiagonalisation (LAPACK dgebrd
 * semantics; the reference's one-sided Ralha recurrence, client.cpp:829-910,
 * is not accurate enough for small singular values of a dense matrix), the
 * Sturm count of singular values (client.cpp:966-971), bisection + twisted
 * vectors with the sign conventions (client.cpp:984-995, bbtsvd.cpp:932-968)
 * and the two reflector back-transforms.  Outputs: d_sigma[k] descending,
 * d_U row-major m x k, d_VT row-major k x m; top_k <= 0 means all. */
bbt_status bbt_svd_dense(bbt_ctx* ctx, int m, double* d_X, int top_k, double* d_sigma, double* d_U,
                         double* d_VT, int* h_k);

/* ---- exact integer products on the int8 tensor cores (CRT) ---------------
 * Rows of each operand are rounded to `bits`-bit integers relative to a
 * power-of-two row scale (bits <= 53: every double whose exponent is within
 * bits - 53 of its row's largest stays exact); their integer product is
 * computed exactly from int8 residues modulo up to 24 pairwise coprime
 * moduli <= 256 (one tcgen05 int8 GEMM per modulus) and rebuilt by the
 * Chinese remainder theorem.
 * bbt_dgemm_crt: d_C (M x N, column-major, ldc) = alpha A^T B + beta C for
 * column-major d_A (K x M, lda) and d_B (K x N, ldb), rounded to a double.
 * bbt_gram_dd: the upper triangle of G = X X^T for a row-major m x n d_X
 * (ldx), as a double-double d_Gh + d_Gl (column-major m x m) with 53-bit rows:
 * exact up to about 2^-100 of the largest entry. */
bbt_status bbt_dgemm_crt(bbt_ctx* ctx, int M, int N, long K, double alpha, const double* d_A, long lda,
                         const double* d_B, long ldb, double beta, double* d_C, long ldc, int bits);
bbt_status bbt_gram_dd(bbt_ctx* ctx, int m, long n, const double* d_X, long ldx, double* d_Gh, double* d_Gl);

/* ---- exact-Gram local QR (precision mode 2) --------------------------------
 * bbt_exact_local_qr: the R factor of A = X^T for a row-major m x local_n d_x
 * (local_n >= m; not modified) from the BF16x3 sketch's preconditioner R_p
 * and the exact Gram of X's 53-bit rows (bbt_gram_dd), preconditioned in
 * double-double: d_R (m x m, column-major, dgeqrf's row signs; with
 * local_n == m the last row's sign can differ, LAPACK's last reflector being
 * the identity there), d_W, d_Rp
 * (m x m column-major) and d_scale (m) describe Q = A_int R_p^-1 W, with
 * A_int X^T's rows rounded to 53-bit integers at the row scales d_scale.
 * bbt_exact_apply_q: d_C (rows x k column-major, ldc) = A_int R_p^-1 d_Z for
 * d_Z (m x k column-major), A_int(j, i) the integers of d_x[i ldx + j] --
 * with the outputs of bbt_exact_local_qr for the same d_x and Z = W Z',
 * d_C = Q Z' (R_p^-1 W Z' solved in double-double and multiplied exactly). */
bbt_status bbt_exact_local_qr(bbt_ctx* ctx, int m, size_t local_n, const double* d_x, double* d_R, double* d_W,
                              double* d_Rp, double* d_scale);
bbt_status bbt_exact_apply_q(bbt_ctx* ctx, int m, size_t rows, const double* d_x, long ldx, const double* d_scale,
                             const double* d_Rp, const double* d_Z, int k, double* d_C, long ldc);

/* ---- whole pipeline ------------------------------------------------------
 * DecentralizedClient::run() (client.cpp:447-1200) with opt_control 3, for P
 * participants held as separate device buffers on one GPU; the socket
 * all-reduce / all-gather become in-device reductions.  Both branches of the
 * reference:
 *   short-and-wide, m <= global_n (client.cpp:570-606, 680-800, 1174-1195):
 *     block c is X_c, row-major m x local_n[c]; local QR of blocks with
 *     local_n / m > 5, global QR of the masked blocks (none when
 *     m == global_n), Ralha of the m x m result;
 *   tall-and-skinny, m > global_n (client.cpp:543-568, 627-679, 1119-1169):
 *     block c is X_c^T, row-major local_n[c] x m (the reference's file layout
 *     in this branch); the masked blocks are repartitioned into column slabs
 *     of m_part[c] rows of X, slabs with m_part[c] > global_n are reduced by
 *     a local QR, and Ralha runs on the global_n x sum_c min(m_part[c],
 *     global_n) concatenation.
 * The global matrix is X = [X_0 | X_1 | ...] (m x global_n) in both. */
typedef struct {
  int participants;              /* P >= 1 */
  size_t m;                      /* rows of X (reference: m) */
  const size_t* local_n;         /* P column counts (reference: local_n) */
  unsigned public_seed;          /* shared mask seed (client.cpp:498) */
  const unsigned* private_seeds; /* P private mask seeds (client.cpp:531) */
  int top_k;                     /* <= 0: all singular values (client.cpp:971) */
  int svd_mode;                  /* client.cpp:186-192: 0 full SVD (the reference calls dbdsdc on the
                                    leading k x k bidiagonal; here bisection + twisted vectors on it),
                                    1 two-sided, 2 left vectors only (no FinalVT), 3 right vectors
                                    only (no FinalU), 4 linear regression (tall-and-skinny only, as in
                                    the reference, client.cpp:1023-1160): w = V diag(1/sigma) U^T y,
                                    the least-squares solution of X w = y, returned per participant
                                    in place of FinalVT; no FinalU */
  int precision;                 /* 0: plain FP64 (the reference's Householder local QR);
                                    1: mixed -- local QR by a BF16x3 tensor-core sketch
                                    and one FP64 Cholesky-QR refinement pass;
                                    2: exact Gram -- the sketch as preconditioner, the
                                    Gram of each block computed exactly from int8
                                    residues (CRT), the congruence in double-double, Q
                                    never formed and applied by exact products
                                    (bbt_exact_local_qr, bbt_exact_apply_q); the
                                    tall-and-skinny branch runs precision 2 as 1 */
  const double* labels;          /* svd_mode 4: y, m values (device memory for bbt_fedsvd_run, host
                                    memory for bbt_fedsvd_run_host; the reference's y.mat, held by
                                    the last participant); NULL otherwise */
} bbt_fedsvd_config;

/* Device-resident run.  d_blocks[c]: participant c's input in the branch's
 * layout (above), used as workspace (overwritten).  Outputs: d_sigma
 * (min(m, global_n) values), d_U = FinalU, row-major m x k (short-and-wide)
 * or k x m (tall-and-skinny, client.cpp:1071-1105); may be NULL in
 * svd_modes 3 and 4), d_VT[c] = FinalVT_c, row-major k x local_n[c] (d_VT may
 * be NULL in svd_mode 2), or in svd_mode 4 w_c (local_n[c] values);
 * *h_k is the number of singular values k.  Replaces client.cpp:543-1199. */
bbt_status bbt_fedsvd_run(bbt_ctx* ctx, const bbt_fedsvd_config* cfg, double* const* d_blocks,
                          double* d_sigma, double* d_U, double* const* d_VT, int* h_k);

/* Same with host buffers (pinned or pageable): copies in, runs, copies out;
 * inputs are not modified. */
bbt_status bbt_fedsvd_run_host(bbt_ctx* ctx, const bbt_fedsvd_config* cfg,
                               const double* const* h_blocks, double* h_sigma, double* h_U,
                               double* const* h_VT, int* h_k);

/* Same with the reference's on-disk input (client.cpp:210-213, 1028;
 * utils.cpp:237-252): participant c's block is read from
 * <dpath>/Client<c>.mat, raw float64 of m * local_n[c] values in the branch's
 * layout (row-major m x local_n[c], or local_n[c] x m when m > global_n, as the
 * reference's generate_data.cpp writes them), and in svd_mode 4 the labels
 * from <dpath>/y.mat (m values; cfg->labels is ignored).  Files are checked
 * before any work starts; a missing or wrongly sized file returns BBT_ERR_IO
 * with its name.  A host thread reads them through pinned staging while the
 * GPU works on the participants already read.  Outputs as
 * bbt_fedsvd_run_host. */
bbt_status bbt_fedsvd_run_files(bbt_ctx* ctx, const bbt_fedsvd_config* cfg, const char* dpath,
                                double* h_sigma, double* h_U, double* const* h_VT, int* h_k);

/* Autotuner of the batched local QR (the QR of every participant with
 * local_n / m > 5, client.cpp:572-589, issued on concurrent streams and
 * replayed as one CUDA graph): times every (streams, panel width) candidate
 * on synthetic blocks of cfg's shapes and keeps the fastest in ctx for later
 * bbt_fedsvd_run calls with the same shapes.  Outputs may be NULL. */
bbt_status bbt_fedsvd_tune(bbt_ctx* ctx, const bbt_fedsvd_config* cfg, int* streams, int* panel_width,
                           double* ms);

/* Per-stage wall time (ms, CUDA events) of the last bbt_fedsvd_run, in the
 * reference's phase order: local_qr, apply_mask, global_qr, bi_diag, bsvd,
 * combine_svd_remove_mask.  n must be >= 6. */
bbt_status bbt_fedsvd_stage_ms(const bbt_ctx* ctx, double* ms, int n);

#ifdef __cplusplus
}
#endif
#endif /* BBTSVD_B200_H */
