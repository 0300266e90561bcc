// Exact-Gram local QR (precision mode 2): the R factor of A = X^T without
// forming Q, and the products with the implicit Q, for the participant
// blocks (the replacement of client.cpp:417-445's dgeqrf/dorgqr and of the
// back-transform products with local_v, :1188-1195) and for the global QR
// (:705-794 and the products with its Q, :1179).
//
//   1. R_p = chol(Y^T Y + shift), Y = S A the BF16x3 sketch (sketch.cu) --
//      a preconditioner: A R_p^-1 is well conditioned;
//   2. G = X X^T exactly: every row of X rounded to a 53-bit integer relative
//      to a power-of-two row scale (exact for every entry whose exponent is
//      within 0..-1 of its row's largest, the rest to 2^-53 of that largest),
//      the integer product computed exactly from int8 residues on the tensor
//      cores (crt.cu) and kept as a double-double;
//   3. G_Q = R_p^-T G R_p^-1 in double-double (ddsolve.cu): the Gram of
//      Q_p = A_int R_p^-1 to ~2^-90 of its norm (compensated sums,
//      renormalised every 32 terms, growing with cond(R_p)), far below FP64
//      rounding; it is well conditioned, so R_3 = chol(G_Q) in FP64 is as
//      accurate as R_3 can be;
//   4. R = R_3 R_p, W = R_3^-1, Q = A_int R_p^-1 W (never formed), and
//      dgeqrf's row signs recovered from Q's top block as mixedqr.cu does.
//
// Products with Q (exact_apply_q) use the same integers A_int, so Q and R
// describe the same matrix: C = Q Z = A_int (R_p^-1 (W Z)) with R_p^-1 (W Z)
// solved in double-double, rounded to 80-bit integers per column and
// multiplied exactly by A_int (19 moduli at K = 1000).  No triangular solve
// over the long dimension of A is left.  The residue planes of A_int can be
// formed once, with every modulus both products need, and kept: the Gram
// reads them K-major, the products with Q MN-major (exact_apply_planes), and
// X itself is then read only by the sketch, the row maxima and that one pass.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>

#include "internal.h"

namespace bbt {
namespace {

constexpr int GRAM_BITS = 53;
constexpr int Z_BITS = 80;
// Scratch cap of one pass over the long dimension: the Gram's residue planes
// (when they are not kept) and the products with Q (residues of the rows and
// of the product) are formed in chunks of at most this many bytes, so a
// participant of any length needs bounded workspace (2 x 10^9-element blocks
// of 4 x 2000 x 10^6 included).
constexpr size_t LONG_CHUNK_DEFAULT = (size_t)6 << 30;

// K-chunk of the Gram's residue planes (nm planes of m rows): all of n when
// the planes fit the cap, else equal chunks, a multiple of 2^15 columns.
long gram_chunk(int m, long n, int nm) {
  const size_t cap = long_chunk_bytes(LONG_CHUNK_DEFAULT);
  const size_t full = (size_t)nm * m * crt_pitch(n);
  if (full <= cap) return n;
  long c = (long)(cap / ((size_t)nm * m)) / 32768 * 32768;
  c = std::max(c, 32768L);
  const long chunks = (n + c - 1) / c;
  return ((n + chunks - 1) / chunks + 32767) / 32768 * 32768;
}

// Products with Q: the two-pass CRT product (residues of the product in HBM,
// 256-column tiles) and reconstruction, or, with EXCALIBUR_B200_FUSED_APPLY=1,
// the product fused with its reconstruction (no residues in HBM, 128-column
// tiles; the same result bit for bit).  Measured at 2 x 500,000 x 1,000 the
// two-pass path is faster: the fused kernel's smaller tiles re-read the
// MN-major residue planes twice as often and its per-modulus reconstruction
// is as long as the MMAs at K = 1000.
bool apply_fused(int m, int nm) {
  const char* v = std::getenv("EXCALIBUR_B200_FUSED_APPLY");
  if (!v || v[0] != '1') return false;
  return crt_fused_supported(m, nm);
}

// Row chunk of a product with Q over `rows` rows: all rows when the residues
// of A and of the product fit the cap, else equal chunks (multiples of 128).
// fused: the product's residues are not stored.
long apply_chunk(long rows, int nm, long Kp, int k, bool fused) {
  const size_t cap = long_chunk_bytes(LONG_CHUNK_DEFAULT);
  const size_t per_row = (size_t)nm * (Kp + (fused ? 0 : k)) + 8;
  if ((size_t)rows * per_row <= cap) return rows;
  long c = (long)(cap / per_row) / 128 * 128;
  c = std::max(c, 128L);
  const long chunks = (rows + c - 1) / c;
  return ((rows + chunks - 1) / chunks + 127) / 128 * 128;
}

__global__ void dd_scale_rows_kernel(int m, int k, const double* __restrict__ s, double* __restrict__ Zh,
                                     double* __restrict__ Zl, long ld) {
  const long total = (long)m * k;
  for (long f = blockIdx.x * (long)blockDim.x + threadIdx.x; f < total; f += (long)gridDim.x * blockDim.x) {
    const int i = (int)(f % m);
    const long j = f / m;
    Zh[i + j * ld] *= s[i];   // powers of two: exact
    Zl[i + j * ld] *= s[i];
  }
}

__global__ void zero_kernel(double* __restrict__ p, long n) {
  for (long f = blockIdx.x * (long)blockDim.x + threadIdx.x; f < n; f += (long)gridDim.x * blockDim.x) p[f] = 0.0;
}

}  // namespace

// Product residues of the chunked Gram: every chunk's K-splits side by side.
size_t gram_product_bytes(const bbt_ctx* ctx, int m, long n, int nm, long kc, int* total_splits) {
  size_t b = 0;
  int sp = 0;
  for (long k0 = 0; k0 < n; k0 += kc) {
    const long K = std::min(kc, n - k0);
    const size_t one = crt_product_bytes(ctx, m, m, K, nm, true) - 4096;
    b += one;
    sp += (int)(one / ((size_t)nm * ((m + 3) & ~3) * m));
  }
  if (total_splits) *total_splits = sp;
  return b + 4096;
}

size_t exact_qr_workspace_bytes(const bbt_ctx* ctx, int m, long n) {
  const int N = sketch_rows(m);
  size_t s = sketch_workspace_bytes(ctx, m, n, N);
  s = std::max(s, dgemm_workspace_bytes(ctx, m, m, N));
  s = std::max(s, exact_gram_workspace_bytes(ctx, m, n));
  return s + ((size_t)N * m + 6 * (size_t)m * m + 3 * m) * 8 + 16384;
}

int exact_keep_moduli(int m, long n) {
  const int a = crt_moduli(GRAM_BITS, GRAM_BITS, n), b = crt_moduli(GRAM_BITS, Z_BITS, m);
  return (a < 1 || b < 1) ? -1 : std::max(a, b);
}

size_t exact_keep_bytes(int m, long n) {
  const int nk = exact_keep_moduli(m, n);
  return nk < 1 ? 0 : (size_t)nk * m * crt_pitch(n) + 256;
}

size_t exact_gram_workspace_bytes(const bbt_ctx* ctx, int m, long n) {
  const int nm = crt_moduli(GRAM_BITS, GRAM_BITS, n);
  if (nm < 1) return 0;
  const long kc = gram_chunk(m, n, nm);
  return (size_t)nm * m * crt_pitch(kc) + gram_product_bytes(ctx, m, n, nm, kc, nullptr) + (size_t)m * 8 + 4096;
}

// The upper triangle of G = X X^T for X's rows rounded to 53-bit integers at
// the row scales (written to scale), exactly, as a double-double (column-major,
// ld m).  Kept planes (every modulus the later products with X_int^T need)
// cover all of K at once; otherwise the planes are formed in K-chunks (the row
// scales over all of K first) whose products' K-splits sit side by side and
// are summed by one reconstruction.
bbt_status exact_gram_dd(bbt_ctx* ctx, int m, long n, const double* X, long ldx, double* scale, int8_t* keep,
                         double* Gh, double* Gl, const unsigned long long* rowmax) {
  const int nm = crt_moduli(GRAM_BITS, GRAM_BITS, n);
  if (nm < 1) return fail(ctx, BBT_ERR_ARG, "exact Gram: n=%ld too long", n);
  const size_t m2 = ctx->ws.top;
  const int nr = keep ? exact_keep_moduli(m, n) : nm;   // the Gram uses the first nm of the kept planes
  const long kc = keep ? n : gram_chunk(m, n, nm);
  const long Kp = crt_pitch(kc);
  int8_t* RX = keep ? keep : ctx->ws.take<int8_t>((size_t)nm * m * Kp);
  const size_t m3 = ctx->ws.top;
  if (rowmax)
    BBT_TRY(crt_scales_from_max(ctx, m, rowmax, scale));
  else
    BBT_TRY(crt_row_scales(ctx, m, n, X, ldx, scale));
  ctx->ws.top = m3;
  uint8_t* Rb = ctx->ws.take<uint8_t>(gram_product_bytes(ctx, m, n, nm, kc, nullptr));
  if (!Rb || !RX) return fail(ctx, BBT_ERR_NOMEM, "exact Gram: workspace");
  const size_t split_bytes = (size_t)nm * ((m + 3) & ~3) * m;
  int splits = 0;
  for (long k0 = 0; k0 < n; k0 += kc) {
    const long K = std::min(kc, n - k0);
    BBT_TRY(crt_residues_rows(ctx, m, K, X + k0, ldx, scale, GRAM_BITS, nr, RX, Kp));
    int sp = 1;
    BBT_TRY(crt_product(ctx, m, m, K, nm, RX, RX, Kp, true, Rb + (size_t)splits * split_bytes, &sp));
    splits += sp;
  }
  BBT_TRY(crt_combine_dd(ctx, m, m, nm, splits, Rb, true, scale, scale, 2 * (GRAM_BITS - 1), Gh, Gl, m));
  ctx->ws.top = m2;
  return BBT_OK;
}

bbt_status exact_local_qr(bbt_ctx* ctx, int m, long n, const double* X, const void* S, long spitch, double* R,
                          double* W, double* Rp, double* scale, int8_t* keep) {
  if (n < m) return fail(ctx, BBT_ERR_ARG, "exact local QR: n=%ld < m=%d", n, m);
  const int nm = crt_moduli(GRAM_BITS, GRAM_BITS, n);
  if (nm < 1) return fail(ctx, BBT_ERR_ARG, "exact local QR: n=%ld too long", n);
  const int N = sketch_rows(m);
  const size_t mark = ctx->ws.top;
  double* Y = ctx->ws.take<double>((size_t)N * m);
  double* Gh = ctx->ws.take<double>((size_t)m * m);
  double* Gl = ctx->ws.take<double>((size_t)m * m);
  double* Th = ctx->ws.take<double>((size_t)m * m);
  double* Tl = ctx->ws.take<double>((size_t)m * m);
  double* dsig = ctx->ws.take<double>(m);
  unsigned long long* rowmax = ctx->ws.take<unsigned long long>(m);
  if (!rowmax) return fail(ctx, BBT_ERR_NOMEM, "exact local QR: workspace");
  int* flag = ctx->d_flag + FLAG_CHOL;
  // 1. the preconditioner from the sketch (its pass over X also forms the row
  //    maxima of the Gram's scales)
  BBT_CUDA(ctx, cudaMemsetAsync(rowmax, 0, (size_t)m * 8, ctx->stream));
  BBT_TRY(sketch_bf16x3(ctx, m, n, X, n, N, S, spitch, Y, rowmax));
  BBT_TRY(dgemm(ctx, true, false, m, m, N, 1.0, Y, N, Y, N, 0.0, Rp, m, 0, true));
  BBT_TRY(symmetrize_upper(ctx, m, Rp, m));
  BBT_TRY(shift_diag(ctx, m, Rp, m, 1e-14));
  BBT_TRY(potrf_upper(ctx, m, Rp, m, flag));
  // 2. the exact Gram of the 53-bit rows of X, as a double-double
  BBT_TRY(exact_gram_dd(ctx, m, n, X, n, scale, keep, Gh, Gl, rowmax));
  BBT_TRY(dd_symmetrize_upper(ctx, m, Gh, Gl, m));
  // 3. G_Q = R_p^-T (R_p^-T G)^T in double-double (G symmetric)
  BBT_TRY(dd_trsm_left(ctx, true, m, m, Rp, m, Gh, Gl, m));
  BBT_TRY(dd_transpose(ctx, m, Gh, Gl, m, Th, Tl, m));
  BBT_TRY(dd_trsm_left(ctx, true, m, m, Rp, m, Th, Tl, m));
  // 4. R_3 = chol(G_Q), R = R_3 R_p, W = R_3^-1 (Gh is free again)
  BBT_TRY(potrf_upper(ctx, m, Th, m, flag));
  BBT_TRY(dgemm(ctx, false, false, m, m, m, 1.0, Th, m, Rp, m, 0.0, R, m));
  BBT_TRY(identity(ctx, m, W, m));
  BBT_TRY(trsm_right_upper(ctx, m, m, Th, m, W, m));
  // 5. dgeqrf's row signs from Q's top m x m block: A[:m] R_p^-1 W
  BBT_TRY(copy2d(ctx, m, m, X, n, Gh, m));   // column i of A[:m] = the first m entries of row i of X
  BBT_TRY(trsm_right_upper(ctx, m, m, Rp, m, Gh, m));
  BBT_TRY(dgemm(ctx, false, false, m, m, m, 1.0, Gh, m, W, m, 0.0, Tl, m));
  BBT_TRY(householder_signs(ctx, m, m, Tl, m, dsig));
  BBT_TRY(apply_signs(ctx, m, dsig, R, W));
  ctx->ws.top = mark;
  return BBT_OK;
}

size_t exact_apply_workspace_bytes(const bbt_ctx* ctx, long rows, int m, int k) {
  const int nm = crt_moduli(GRAM_BITS, Z_BITS, m);
  const long Kp = crt_pitch(m);
  const bool fused = apply_fused(m, nm);
  const long rc = apply_chunk(rows, nm, Kp, k, fused);
  return (size_t)nm * (rc + k) * Kp + (fused ? 0 : crt_product_bytes(ctx, (int)rc, k, m, nm, false)) +
         (4 * (size_t)m * k + 2 * (size_t)k) * 8 + 16384;
}

size_t exact_operand_bytes(int m, int k) {
  const int nm = crt_moduli(GRAM_BITS, Z_BITS, m);
  return (size_t)nm * k * crt_pitch(m) + (size_t)k * 8 + 512;
}

// The Z side of C = A_int R_p^-1 Z: Z2 = diag(scale) R_p^-1 Z solved in
// double-double (the row scales of X fold into Z's rows), then every column of
// Z2 rounded to an 80-bit integer at its own scale t (k) and reduced to the
// residue planes RB (exact_operand_bytes).  One operand serves every row block
// of A_int that shares R_p and the row scales.
bbt_status exact_operand(bbt_ctx* ctx, int m, const double* scale, const double* Rp, const double* Z, int k,
                         ExactOperand& op) {
  const int nm = crt_moduli(GRAM_BITS, Z_BITS, m);
  if (nm < 1) return fail(ctx, BBT_ERR_ARG, "exact apply: m=%d", m);
  op.m = m;
  op.k = k;
  op.nm = nm;
  op.Kp = crt_pitch(m);
  op.t = ctx->ws.take<double>(k);
  op.RB = ctx->ws.take<int8_t>((size_t)nm * k * op.Kp);
  const size_t mark = ctx->ws.top;
  double* Zh = ctx->ws.take<double>((size_t)m * k);
  double* Zl = ctx->ws.take<double>((size_t)m * k);
  if (!Zl) return fail(ctx, BBT_ERR_NOMEM, "exact apply: workspace");
  BBT_TRY(copy2d(ctx, k, m, Z, m, Zh, m));   // k columns of m entries (copy2d counts rows of its row-major view)
  zero_kernel<<<2 * ctx->num_sms, 256, 0, ctx->stream>>>(Zl, (long)m * k);
  BBT_LAUNCHED(ctx);
  BBT_TRY(dd_trsm_left(ctx, false, m, k, Rp, m, Zh, Zl, m));
  dd_scale_rows_kernel<<<2 * ctx->num_sms, 256, 0, ctx->stream>>>(m, k, scale, Zh, Zl, m);
  BBT_LAUNCHED(ctx);
  {
    const size_t m2 = ctx->ws.top;
    BBT_TRY(crt_row_scales(ctx, k, m, Zh, m, op.t));
    ctx->ws.top = m2;
  }
  BBT_TRY(crt_residues_dd(ctx, k, m, Zh, Zl, m, op.t, Z_BITS, nm, op.RB, op.Kp));
  ctx->ws.top = mark;   // Zh, Zl die here; t and RB stay with the caller's mark
  return BBT_OK;
}

// C (rows x k, column-major, ldc) = A_int R_p^-1 Z for a prepared Z operand,
// A_int(j, i) the 53-bit integers of X(i, j) = X[i ldx + j] (i < m, j < rows)
// at the row scales of X (those exact_local_qr used).
bbt_status exact_apply_rows(bbt_ctx* ctx, const ExactOperand& op, long rows, const double* X, long ldx,
                            const double* scale, double* C, long ldc) {
  if (rows > 0x7fffffffL) return fail(ctx, BBT_ERR_ARG, "exact apply: rows=%ld", rows);
  const int m = op.m, k = op.k, nm = op.nm;
  const size_t mark = ctx->ws.top;
  const bool fused = apply_fused(m, nm);
  const long rc = apply_chunk(rows, nm, op.Kp, k, fused);   // rows are independent: chunks bound the scratch
  int8_t* RA = ctx->ws.take<int8_t>((size_t)nm * rc * op.Kp);
  uint8_t* Rb = fused ? nullptr : ctx->ws.take<uint8_t>(crt_product_bytes(ctx, (int)rc, k, m, nm, false));
  if (!RA || (!fused && !Rb)) return fail(ctx, BBT_ERR_NOMEM, "exact apply: workspace");
  const int shift = (GRAM_BITS - 1) + (Z_BITS - 1);
  for (long r0 = 0; r0 < rows; r0 += rc) {
    const int R = (int)std::min(rc, rows - r0);
    BBT_TRY(crt_residues_cols(ctx, R, m, X + r0, ldx, scale, GRAM_BITS, nm, RA, op.Kp));
    if (fused) {
      BBT_TRY(crt_product_fused(ctx, R, k, m, nm, RA, 0, op.RB, op.Kp, op.t, shift, 1.0, C + r0, ldc));
      continue;
    }
    int splits = 1;
    BBT_TRY(crt_product(ctx, R, k, m, nm, RA, op.RB, op.Kp, false, Rb, &splits));
    BBT_TRY(crt_combine(ctx, R, k, nm, splits, Rb, false, nullptr, op.t, shift, 1.0, 0.0, C + r0, ldc));
  }
  ctx->ws.top = mark;
  return BBT_OK;
}

// The same from the planes exact_local_qr kept (A_int(j, i) = X_int(i, j),
// planes [q][m][pitch], pitch = crt_pitch(rows)): X_int^T as an MN-major
// operand, so the block is not read again.
bbt_status exact_apply_planes(bbt_ctx* ctx, const ExactOperand& op, long rows, const int8_t* planes, long pitch,
                              double* C, long ldc, const std::function<bbt_status(long, int)>* after,
                              long chunk_rows) {
  if (rows > 0x7fffffffL) return fail(ctx, BBT_ERR_ARG, "exact apply: rows=%ld", rows);
  const int m = op.m, k = op.k, nm = op.nm;
  const int shift = (GRAM_BITS - 1) + (Z_BITS - 1);
  if (apply_fused(m, nm)) {   // the kept planes in, FP64 out: no scratch at all
    BBT_TRY(crt_product_fused(ctx, (int)rows, k, m, nm, planes, pitch, op.RB, op.Kp, op.t, shift, 1.0, C, ldc));
    return after ? (*after)(0, (int)rows) : BBT_OK;
  }
  const size_t mark = ctx->ws.top;
  long rc = apply_chunk(rows, nm, 0, k, false);   // only the product's residues are scratch here
  if (chunk_rows > 0 && rc > chunk_rows) rc = std::max(128L, chunk_rows / 128 * 128);
  uint8_t* Rb = ctx->ws.take<uint8_t>(crt_product_bytes(ctx, (int)rc, k, m, nm, false));
  if (!Rb) return fail(ctx, BBT_ERR_NOMEM, "exact apply: workspace");
  for (long r0 = 0; r0 < rows; r0 += rc) {   // row chunks start at multiples of 128: 16-byte TMA offsets
    const int R = (int)std::min(rc, rows - r0);
    int splits = 1;
    BBT_TRY(crt_product_amn(ctx, R, k, m, nm, planes + r0, pitch, op.RB, op.Kp, Rb, &splits));
    BBT_TRY(crt_combine(ctx, R, k, nm, splits, Rb, false, nullptr, op.t, shift, 1.0, 0.0, C + r0, ldc));
    if (after) BBT_TRY((*after)(r0, R));
  }
  ctx->ws.top = mark;
  return BBT_OK;
}

// C (rows x k, column-major, ldc) = A_int R_p^-1 Z, Z (m x k, column-major, FP64).
bbt_status exact_apply_q(bbt_ctx* ctx, int m, long rows, const double* X, long ldx, const double* scale,
                         const double* Rp, const double* Z, int k, double* C, long ldc) {
  const size_t mark = ctx->ws.top;
  ExactOperand op;
  BBT_TRY(exact_operand(ctx, m, scale, Rp, Z, k, op));
  BBT_TRY(exact_apply_rows(ctx, op, rows, X, ldx, scale, C, ldc));
  ctx->ws.top = mark;
  return BBT_OK;
}

}  // namespace bbt
