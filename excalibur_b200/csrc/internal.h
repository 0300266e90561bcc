// Internal declarations shared by the CUDA sources of libexcalibur_b200.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <functional>
#include <string>
#include <vector>

#include "../../include/bbtsvd_b200.h"

namespace bbt {

// Device workspace: one growing allocation per context, carved per call.
struct Arena {
  char* base = nullptr;
  size_t cap = 0;
  size_t top = 0;
  cudaError_t reserve(size_t bytes);   // grows (frees and reallocates) when needed
  void reset() { top = 0; }
  // A failed take leaves the arena exhausted, so every later take of the same
  // scope fails too and checking the last pointer of a group is enough.
  template <class T>
  T* take(size_t count) {
    size_t off = (top + 255) & ~size_t(255);
    size_t need = off + count * sizeof(T);
    if (need > cap) {
      top = cap;
      return nullptr;
    }
    top = need;
    return reinterpret_cast<T*>(base + off);
  }
  size_t room() const { return top < cap ? cap - top : 0; }
};

}  // namespace bbt

namespace bbt {
struct ProfRec {
  cudaEvent_t a, b;
  int cls;
  double work;
};
}  // namespace bbt

struct bbt_ctx {
  int device = 0;
  int num_sms = 0;
  cudaStream_t own = nullptr;
  cudaStream_t stream = nullptr;
  bbt::Arena ws;
  std::string err;
  uint64_t launches = 0;
  int* d_flag = nullptr;         // device error flag for bounded waits
  unsigned* d_barrier = nullptr; // grid-barrier state (count, generation)
  double stage_ms[8] = {0};
  bool prof = false;
  std::vector<bbt::ProfRec> recs;          // pending event pairs
  double prof_ms[16] = {0}, prof_work[16] = {0};
  uint64_t prof_n[16] = {0};
  bool allow_coop = true;        // false in the concurrent sub-streams of the batched QR
  // batched local QR: side streams, the captured graph and the tuned schedule
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> side_ev;
  cudaGraphExec_t qr_graph = nullptr;
  std::vector<size_t> qr_key;
  uint64_t qr_graph_nodes = 0;
  int tuned_streams = 0, tuned_nb = 0;   // 0: not tuned
  std::vector<size_t> tuned_key;
  // learned bisection brackets: MLP parameters (device copy, owned) and the
  // half-width multiplier; stats of the last bisection that used them
  double* bracket_theta = nullptr;
  double bracket_z = 3.0;
  long bisect_stats[4] = {0, 0, 0, 0};
  // host-buffer pipeline entry: staging arena, copy streams, and the events
  // that let participant c's work start as soon as its block has arrived and
  // FinalVT_c leave as soon as it is computed
  bbt::Arena io_ws;
  cudaStream_t copy_in = nullptr, copy_out = nullptr;
  bool io_on = false;
  std::vector<cudaEvent_t> in_ready, vt_done;
  std::vector<double*> vt_dst;
  // file entry: two pinned staging buffers and their copy events; the gate
  // blocks until participant c's input has been read and its copy enqueued
  void* io_pinned = nullptr;
  // pinned staging of the pipeline's prepared mask tables (grown on demand)
  void* mask_pinned = nullptr;
  size_t mask_pinned_cap = 0;
  cudaEvent_t io_stage_ev[2] = {nullptr, nullptr};
  bool (*io_gate)(void*, int) = nullptr;
  void* io_gate_arg = nullptr;
};

namespace bbt {

// Slots of ctx->d_flag (16 ints) besides slot 0, the grid-barrier timeout
// flag: the sketch pipeline's wait status and the Cholesky breakdown flag.
enum { FLAG_SKETCH = 4, FLAG_CHOL = 5 };

bbt_status fail(bbt_ctx* ctx, bbt_status s, const char* fmt, ...);
// Order ctx->stream after participant c's input (host-entry runs): passes the
// file gate first, then waits on ctx->in_ready[c] (hostio.cu).
bbt_status wait_input(bbt_ctx* ctx, int c);
bbt_status cuda_fail(bbt_ctx* ctx, cudaError_t e, const char* what);

#define BBT_CUDA(ctx, call)                                   \
  do {                                                        \
    cudaError_t e_ = (call);                                  \
    if (e_ != cudaSuccess) return bbt::cuda_fail(ctx, e_, #call); \
  } while (0)

#define BBT_LAUNCHED(ctx)                                        \
  do {                                                           \
    (ctx)->launches++;                                           \
    cudaError_t e_ = cudaGetLastError();                         \
    if (e_ != cudaSuccess) return bbt::cuda_fail(ctx, e_, "kernel launch"); \
  } while (0)

// Event-bracketed launch region for the profiler (no-op when profiling is off).
struct ProfScope {
  bbt_ctx* ctx;
  ProfRec r;
  bool on;
  ProfScope(bbt_ctx* c, int cls, double work) : ctx(c), on(c->prof) {
    if (!on) return;
    r.cls = cls;
    r.work = work;
    cudaEventCreate(&r.a);
    cudaEventCreate(&r.b);
    cudaEventRecord(r.a, c->stream);
  }
  ~ProfScope() {
    if (!on) return;
    cudaEventRecord(r.b, ctx->stream);
    ctx->recs.push_back(r);
  }
};

#define BBT_TRY(call)                       \
  do {                                      \
    bbt_status s_ = (call);                 \
    if (s_ != BBT_OK) return s_;            \
  } while (0)

// ---- kernels exposed across translation units (all stream-ordered) ----

// Sturm / bisection / twisted (sturm.cu, twisted.cu)
bbt_status sturm_counts(bbt_ctx* ctx, int n, const double* a, const double* b, const double* mu,
                        int nmu, int* counts);
// brackets (optional): [lo, hi] per j-th largest value (j < min(top_k, k)),
// snapped to the reference's tree, verified by Sturm counts, used to skip
// levels; stats (optional, 4): Sturm evaluations (verification included),
// rounds, jumps taken, Sturm evaluations spent on verification.
// Scratch of bisect for an order-n bidiagonal and top_k values (the node
// tree, the candidates of a round, the learned-bracket table).
size_t bisect_workspace_bytes(int n, int top_k);
bbt_status bisect(bbt_ctx* ctx, int n, const double* a, const double* b, double lo, double hi,
                  double tol, int top_k, double* sigma, int* count, const double* brackets = nullptr,
                  long* stats = nullptr);
bbt_status twisted(bbt_ctx* ctx, int n, int cnt, const double* sigma, const double* a,
                   const double* b, double* U, int ldu, double* V, bool sign_fix);
bbt_status bidiag_svd(bbt_ctx* ctx, int k, const double* a, const double* b, double* U, double* V,
                      double* sigma, int top_k, bool global_sign);
// twisted() on caller-provided scratch (scratch_doubles_twisted(n, cnt) doubles)
size_t scratch_doubles_twisted(int n, int cnt);
bbt_status twisted_scratch(bbt_ctx* ctx, int n, int cnt, const double* sigma, const double* a,
                           const double* b, double* U, int ldu, double* V, double* scratch);
// The reference's per-step helpers on device arrays (bbtsvd.cpp:54-136):
// LDL^T of B^T B (L n-1, D n), one inverse iteration (v[k ldv] = 1, backward
// with l, forward with u, normalised), one singular pair at *omega (device)
// from the given L, D: v contiguous (n), u with stride ldu; scratch holds
// twisted_pair_scratch_doubles(n) doubles.
bbt_status ldl_factor(bbt_ctx* ctx, int n, const double* a, const double* b, double* L, double* D);
bbt_status inverse_iteration_dev(bbt_ctx* ctx, int n, int k, const double* l, const double* u, double* v, long ldv);
size_t twisted_pair_scratch_doubles(int n);
bbt_status twisted_pair(bbt_ctx* ctx, int n, const double* omega, const double* L, const double* D, const double* a,
                        const double* b, double* v, double* u, int ldu, double* scratch);
// d_out[0] = ||a||^2 + ||b||^2 (the bisection bound, bbtsvd.cpp:936)
bbt_status bidiag_bound(bbt_ctx* ctx, int n, const double* a, const double* b, double* d_out);

// Givens masks (givens.cu)
// The random tables of one mask (bbtsvd.cpp:729-779): pairs and (c, s) per
// pass, drawn on the host with the reference's own calls (glibc rand(),
// std::default_random_engine, std::shuffle), and the same on the device.
struct GivensTables {
  size_t k = 0, passes = 0, ops = 0;
  int b1 = 0, b2 = 0;               // stages [0,b1), [b1,b2), [b2,ops)
  std::vector<int2> pairs;          // [pass][op]
  std::vector<double2> cs;          // (c, s) with s signed for the direction
};
struct GivensDev {
  size_t k = 0, passes = 0, ops = 0;
  int b1 = 0, b2 = 0;
  const int2* pairs = nullptr;
  const double2* cs = nullptr;
};
void draw_givens_tables(size_t k, size_t passes, bool mask, unsigned seed, GivensTables& T);
// The mask of a rotated length k <= 10000 (the direct path) with device tables.
bbt_status apply_givens(bbt_ctx* ctx, const GivensDev& T, size_t m, size_t n, double* x, bool is_left);
bbt_status givens_mask(bbt_ctx* ctx, size_t m, size_t n, size_t passes, double* x, bool mask,
                       bool is_left, unsigned seed);
bbt_status block_shift_mask(bbt_ctx* ctx, size_t m, size_t n, size_t passes, double* x, bool mask,
                            bool is_left, unsigned seed);
// Workspace block_shift_mask uses to process every vector in one batch (it
// splits the vectors into batches when less is free).
size_t mask_workspace_bytes(size_t m, size_t n, size_t passes, bool is_left);

// FP64 GEMM, column-major BLAS convention (dgemm.cu):
//   C = alpha * op(A) * op(B) + beta * C,  op(A) M x K, op(B) K x N.
// splits > 1 splits K; partial products are summed in a fixed order.  With
// upper, only the tiles that touch the upper triangle of C are computed (the
// rest of C is left undefined): for symmetric products.
bbt_status dgemm(bbt_ctx* ctx, bool ta, bool tb, int M, int N, long K, double alpha,
                 const double* A, long lda, const double* B, long ldb, double beta, double* C,
                 long ldc, int splits = 0, bool upper = false);
// Scratch the automatic split-K of dgemm takes from the workspace.
size_t dgemm_workspace_bytes(const bbt_ctx* ctx, int M, int N, long K);

// Householder QR, column-major A (rows x cols, lda), rows >= cols (qr.cu).
struct QrPlan {
  int nb = 128;    // outer panel width (compact-WY block of the trailing update)
  int leaf = 16;   // recursion leaf: columns factored one at a time
};
bbt_status geqrf(bbt_ctx* ctx, long rows, int cols, double* A, long lda, double* tau,
                 double* T /* ceil(cols/nb) * nb * nb */, const QrPlan& plan);
bbt_status orgqr(bbt_ctx* ctx, long rows, int cols, double* A, long lda, const double* tau,
                 const double* T, const QrPlan& plan);
// C (rows x ncols) <- H_0 H_1 ... H_{k-1} C.  Reflector j is column j of V
// from row j down (unit diagonal implied); V(r, c) is read at V[r*rs + c*cs].
// C is column-major (ld ldc) or, with c_rowmajor, row-major (ld ldc).
bbt_status ormqr_left_notrans(bbt_ctx* ctx, long rows, int k, const double* V, long rs, long cs,
                              const double* tau, double* C, long ldc, int ncols, bool c_rowmajor,
                              const QrPlan& plan);
size_t qr_workspace_bytes(long rows, int cols, int ncols_apply, const QrPlan& plan);

// Vectors of clusters of singular values (relative spacing < 1e-7) by block
// inverse iteration from the twisted vectors (clusters.cu).  U: n x k
// row-major, V: k x n row-major, both in place.
bbt_status refine_clusters(bbt_ctx* ctx, int n, int k, const double* a, const double* b, const double* sigma,
                           double* U, double* V, int* nclusters);

// Two-sided Householder bidiagonalisation A = Q B P^T of a column-major n x n
// A (LAPACK dgebrd storage), one cooperative kernel (gebrd.cu).
bbt_status gebrd(bbt_ctx* ctx, int n, double* A, double* d, double* e, double* tauq, double* taup);

// Ralha one-sided bidiagonalisation of W (m x n row-major, overwritten; the
// participants' column slabs side by side); V (m x n) receives the left
// vectors, house (m x m) the reflectors (ralha.cu).
bbt_status ralha(bbt_ctx* ctx, int m, int n, double* W, double* house, double* tau, double* alpha,
                 double* beta, double* V, double* cs);

// Small helpers (util.cu)
// Scratch cap (bytes) of the chunked passes over a long dimension (the
// sketch's bf16 pieces, the CRT residue planes, the Ozaki slices): dflt, or
// the environment's EXCALIBUR_B200_CHUNK_BYTES (at least 1 MiB) when set.
size_t long_chunk_bytes(size_t dflt);
bbt_status transpose(bbt_ctx* ctx, int rows, int cols, const double* src, long lds, double* dst,
                     long ldd);   // dst (cols x rows, row-major) = src^T
bbt_status copy2d(bbt_ctx* ctx, int rows, int cols, const double* src, long lds, double* dst,
                  long ldd);
bbt_status fill(bbt_ctx* ctx, double* p, size_t n, double v);
// RT (m x m row-major) = R^T, R = upper triangle of the top of column-major A
bbt_status r_transpose(bbt_ctx* ctx, int m, const double* A, long lda, double* RT);

// Split-precision sketch (sketch.cu): Y^T (m x N row-major FP64) = X S^T,
// X row-major m x n FP64, S (N x n bf16, row pitch sketch_pitch(n)) +-1.
long sketch_pitch(long n);
int sketch_rows(int m);   // N used by the mixed local QR: 2m rounded up to 128
size_t sketch_workspace_bytes(const bbt_ctx* ctx, int m, long n, int N);
bbt_status rademacher(bbt_ctx* ctx, int N, long n, void* S, uint64_t seed);
// rowmax (optional, zeroed by the caller): each row's max |X| as its FP64 bit
// pattern, from the same pass over X (the CRT row scales of X need them).
bbt_status sketch_bf16x3(bbt_ctx* ctx, int m, long n, const double* X, long ldx, int N, const void* S,
                         long spitch, double* Y, unsigned long long* rowmax = nullptr);

// FP64 Cholesky / triangular solve (chol.cu), column-major.
// A (rows x n) <- A R^{-1}, R upper n x n.
// oz: the updates of large row counts from exact int8 slices (ozaki.cu).
bbt_status trsm_right_upper(bbt_ctx* ctx, long rows, int n, const double* R, long ldr, double* A, long lda,
                            bool oz = false);
// G = R^T R in place (R upper, zeros below); a non-positive pivot sets *flag.
bbt_status potrf_upper(bbt_ctx* ctx, int n, double* G, long ld, int* flag);
bbt_status shift_diag(bbt_ctx* ctx, int n, double* G, long ld, double rel);
bbt_status identity(bbt_ctx* ctx, int n, double* W, long ld);
// Lower triangle of G (n x n column-major) <- upper triangle transposed.
bbt_status symmetrize_upper(bbt_ctx* ctx, int n, double* G, long ld);
// d (cols) <- the row signs of LAPACK's Householder R for the orthonormal
// matrix whose top block is A (rows x cols, rows >= cols; overwritten).
bbt_status householder_signs(bbt_ctx* ctx, int rows, int cols, double* A, long lda, double* d);
// R (m x m column-major) <- D R, W (optional) <- W D.
bbt_status apply_signs(bbt_ctx* ctx, int m, const double* d, double* R, double* W);

// FP64-accurate GEMM from exact int8 slices on the tensor cores (ozaki.cu):
// C (M x N column-major) = alpha A B^T + beta C, A(i,k) = A[i rsA + k csA],
// B(j,k) = B[j rsB + k csB]; each operand needs a unit stride in i or k.
// same: B is A (slices shared); upper: only tiles touching C's upper triangle;
// S (4..8): slices per operand -- error ~2^-(7S) of the row/column scales.
size_t oz_workspace_bytes(const bbt_ctx* ctx, int M, int N, long K, bool same);
bool oz_worthwhile(int M, int N, long K);
bbt_status gemm_oz(bbt_ctx* ctx, int M, int N, long K, double alpha, const double* A, long rsA, long csA,
                   const double* B, long rsB, long csB, double beta, double* C, long ldc, bool same, bool upper,
                   int S = 8);

// Exact integer products on the int8 tensor cores by the Chinese remainder
// theorem (crt.cu).  Operands are rounded per row to b-bit integers
// (t = rint(x 2^(b-1) / s_i), s_i a power of two above 2 max|x|) and given as
// residue planes [modulus][row][Kp] (bytes in [0, p)); the product's residues
// are bytes [split][modulus][N][M] that crt_combine turns back into
// C = alpha sa_i sb_j 2^-shift T + beta C (or a double-double).
long crt_pitch(long K);
int crt_moduli(int bits_a, int bits_b, long K);   // moduli for an exact product; -1 if too many
bbt_status crt_row_scales(bbt_ctx* ctx, int rows, long K, const double* X, long rs, double* scale);
// The same scales from row maxima already formed (max |x| as FP64 bit patterns).
bbt_status crt_scales_from_max(bbt_ctx* ctx, int rows, const unsigned long long* mx, double* scale);
bbt_status crt_residues_rows(bbt_ctx* ctx, int rows, long K, const double* X, long rs, const double* scale, int b,
                             int n, int8_t* planes, long Kp);
// X(i, k) = X[i + k cs] with the scale of K index k (the transposed layout of
// the same integers as crt_residues_rows on X^T)
bbt_status crt_residues_cols(bbt_ctx* ctx, int rows, long K, const double* X, long cs, const double* kscale, int b,
                             int n, int8_t* planes, long Kp);
bbt_status crt_residues_dd(bbt_ctx* ctx, int rows, long K, const double* Xh, const double* Xl, long rs,
                           const double* scale, int b, int n, int8_t* planes, long Kp);
size_t crt_product_bytes(const bbt_ctx* ctx, int M, int N, long K, int n, bool upper);
bbt_status crt_product(bbt_ctx* ctx, int M, int N, long K, int n, const int8_t* RA, const int8_t* RB, long Kp,
                       bool upper, uint8_t* R, int* splits);
// The same with A's planes MN-major: A(i, k) at RA[q][k lda + i] (lda >= M,
// a multiple of 16), e.g. the Gram's planes of X for products with X^T.
bbt_status crt_product_amn(bbt_ctx* ctx, int M, int N, long K, int n, const int8_t* RA, long lda, const int8_t* RB,
                           long Kp, uint8_t* R, int* splits_out);
// The product fused with its reconstruction (one K-split, 16..20 moduli):
// C (column-major, ldc) = alpha sb_j 2^-shift T, equal bit for bit to
// crt_product + crt_combine with no row scales and beta = 0.  A as for
// crt_product (lda = 0) or crt_product_amn (lda > 0).
bool crt_fused_supported(long K, int n);
bbt_status crt_product_fused(bbt_ctx* ctx, int M, int N, long K, int n, const int8_t* RA, long lda, const int8_t* RB,
                             long Kp, const double* sb, int shift, double alpha, double* C, long ldc);
bbt_status crt_combine(bbt_ctx* ctx, int M, int N, int n, int splits, const uint8_t* R, bool upper, const double* sa,
                       const double* sb, int shift, double alpha, double beta, double* C, long ldc);
bbt_status crt_combine_dd(bbt_ctx* ctx, int M, int N, int n, int splits, const uint8_t* R, bool upper,
                          const double* sa, const double* sb, int shift, double* Ch, double* Cl, long ldc);
size_t crt_gemm_workspace_bytes(const bbt_ctx* ctx, int M, int N, long K, int bits, bool same, bool upper);
bool crt_worthwhile(int M, int N, long K);
// C = alpha A B^T + beta C, operands contiguous along K (csA = csB = 1).
bbt_status gemm_crt(bbt_ctx* ctx, int M, int N, long K, double alpha, const double* A, long rsA, long csA,
                    const double* B, long rsB, long csB, double beta, double* C, long ldc, bool same, bool upper,
                    int bits);

// Double-double triangular solves with an FP64 upper-triangular R (ddsolve.cu):
// X (m x k column-major, hi + lo arrays) <- R^-T X (trans) or R^-1 X.
bbt_status dd_trsm_left(bbt_ctx* ctx, bool trans, int m, int k, const double* R, long ldr, double* Xh, double* Xl,
                        long ldx);
bbt_status dd_transpose(bbt_ctx* ctx, int m, const double* Ah, const double* Al, long lda, double* Th, double* Tl,
                        long ldt);
bbt_status dd_symmetrize_upper(bbt_ctx* ctx, int m, double* Gh, double* Gl, long ld);

// Exact-Gram local QR (exactqr.cu): X row-major m x n (= column-major A = X^T,
// kept), R (m x m column-major, dgeqrf's row signs), W = R_3^-1 D, the
// preconditioner Rp and the row scales of X's 53-bit integers; Q = A_int Rp^-1 W.
size_t exact_qr_workspace_bytes(const bbt_ctx* ctx, int m, long n);
// The residue planes of X_int that serve both the Gram and the later products
// with X_int^T (exact_apply_planes): their count and bytes for an m x n block.
int exact_keep_moduli(int m, long n);
size_t exact_keep_bytes(int m, long n);
// The exact Gram of X's 53-bit rows as a double-double (upper triangle, ld m),
// the row scales written to scale; keep: residue planes to fill and keep (or
// null: chunked scratch planes); rowmax: X's row maxima when already formed.
size_t exact_gram_workspace_bytes(const bbt_ctx* ctx, int m, long n);
bbt_status exact_gram_dd(bbt_ctx* ctx, int m, long n, const double* X, long ldx, double* scale, int8_t* keep,
                         double* Gh, double* Gl, const unsigned long long* rowmax = nullptr);
bbt_status exact_local_qr(bbt_ctx* ctx, int m, long n, const double* X, const void* S, long spitch, double* R,
                          double* W, double* Rp, double* scale,
                          int8_t* keep = nullptr);
// C (rows x k column-major) = A_int Rp^-1 Z for A_int(j, i) the integers of X[i ldx + j];
// the Z side can be prepared once (exact_operand, taken from the workspace)
// and applied to several row blocks of A_int (exact_apply_rows).
struct ExactOperand {
  int m = 0, k = 0, nm = 0;
  long Kp = 0;
  double* t = nullptr;
  int8_t* RB = nullptr;
};
size_t exact_operand_bytes(int m, int k);
bbt_status exact_operand(bbt_ctx* ctx, int m, const double* scale, const double* Rp, const double* Z, int k,
                         ExactOperand& op);
bbt_status exact_apply_rows(bbt_ctx* ctx, const ExactOperand& op, long rows, const double* X, long ldx,
                            const double* scale, double* C, long ldc);
// after(r0, R), when given, is called once the rows [r0, r0 + R) of C are
// issued on the context's stream (the caller can copy them out while the
// next rows are computed); chunk_rows (> 0) caps the rows per chunk.
bbt_status exact_apply_planes(bbt_ctx* ctx, const ExactOperand& op, long rows, const int8_t* planes, long pitch,
                              double* C, long ldc, const std::function<bbt_status(long, int)>* after = nullptr,
                              long chunk_rows = 0);
size_t exact_apply_workspace_bytes(const bbt_ctx* ctx, long rows, int m, int k);
bbt_status exact_apply_q(bbt_ctx* ctx, int m, long rows, const double* X, long ldx, const double* scale,
                         const double* Rp, const double* Z, int k, double* C, long ldc);

// Mixed-precision local QR (mixedqr.cu): X (row-major m x n = column-major
// A = X^T, n x m) -> Q_p in place, R (m x m column-major upper), W = R_3^{-1}
// (optional) with Q = Q_p W.  S: sketch_rows(m) x n Rademacher bf16 (row
// pitch spitch >= n, a multiple of 8).
size_t mixed_qr_workspace_bytes(const bbt_ctx* ctx, int m, long n);
bbt_status mixed_local_qr(bbt_ctx* ctx, int m, long n, double* X, const void* S, long spitch, double* R,
                          double* W);
// Clear / read (with a stream sync) the sketch and Cholesky flags.
bbt_status clear_tc_flags(bbt_ctx* ctx);
bbt_status check_tc_flags(bbt_ctx* ctx, const char* what);

// Learned brackets (mlp.cu).  MLP_PARAMS doubles of parameters.
enum { MLP_FEATURES = 10, MLP_HIDDEN = 32,
       MLP_PARAMS = MLP_HIDDEN * MLP_FEATURES + MLP_HIDDEN + MLP_HIDDEN * MLP_HIDDEN + MLP_HIDDEN +
                    2 * MLP_HIDDEN + 2 };
bbt_status mlp_summary(bbt_ctx* ctx, int k, const double* a, const double* b, double* s6);
bbt_status mlp_features(bbt_ctx* ctx, int k, int count, const double* s6, double* X);
bbt_status mlp_forward(bbt_ctx* ctx, int B, const double* X, const double* theta, double* out);
bbt_status mlp_grad(bbt_ctx* ctx, int B, const double* X, const double* y, const double* theta, double* grad,
                    double* loss);
bbt_status mlp_adam(bbt_ctx* ctx, double* theta, const double* grad, double* m, double* v, double lr, int t);
bbt_status mlp_brackets(bbt_ctx* ctx, int k, int count, const double* a, const double* b, const double* theta,
                        double z, double* br);

// Whole pipeline (fedsvd.cu)
bbt_status fedsvd(bbt_ctx* ctx, const bbt_fedsvd_config* cfg, double* const* blocks, double* sigma,
                  double* U, double* const* VT, int* k);
size_t fedsvd_workspace_bytes(const bbt_fedsvd_config* cfg);
bbt_status fedsvd_tune(bbt_ctx* ctx, const bbt_fedsvd_config* cfg, int* streams, int* nb, double* ms);
bbt_status svd_dense(bbt_ctx* ctx, int m, double* X, int top_k, double* sigma, double* U, double* VT, int* k);

}  // namespace bbt
