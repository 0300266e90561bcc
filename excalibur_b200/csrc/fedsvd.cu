// DecentralizedClient::run() (Excalibur src/client.cpp:447-1200) for P
// participants held as separate device buffers on one GPU.
//
// Short-and-wide branch (m <= global_n), svd_mode 1, opt_control 3:
//   local QR of every wide block (local_n / m > 5)          client.cpp:572-589
//   public (row) then private (column) Givens masks          :593-596
//   repartition = the column concatenation M = [M_0 | ...]  :681-703
//   Householder QR of M^T, Q_g kept                          :705-794
//   Ralha bidiagonalisation of R_g                           :801-954
//   bisection + twisted vectors, sign convention            :963-995
//   FinalU = unmask_pub((V_b Vr)^T)                          :1002-1115
//   FinalVT_c = unmask_priv_c(U2^T Q_g[c]^T) Q_c^T           :1119-1195
// The ring all-reduce / all-gather of the reference become reductions
// inside the kernels (Ralha) or plain device-memory reads (U all-gather).
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "internal.h"

namespace bbt {
namespace {

constexpr int MASK_PASSES = 32;            // client.cpp:536
constexpr double LOCAL_QR_THRESHOLD = 5.0; // client.cpp:482

size_t reduced_width(size_t m, size_t n) {   // client.cpp:505,510,517 (integer ratio)
  return (double)(n / m) > LOCAL_QR_THRESHOLD ? std::min(m, n) : n;
}
bool has_local_qr(size_t m, size_t n) { return m < n && (double)(n / m) > LOCAL_QR_THRESHOLD; }

// W (m x m row-major) = upper triangle of R held in the top of column-major Mt (ld).
__global__ void r_rowmajor(int m, const double* __restrict__ Mt, long ld, double* __restrict__ W) {
  const long total = (long)m * m;
  for (long f = blockIdx.x * (long)blockDim.x + threadIdx.x; f < total; f += (long)gridDim.x * blockDim.x) {
    const int i = (int)(f / m), j = (int)(f % m);
    W[f] = (j >= i) ? Mt[i + (long)j * ld] : 0.0;
  }
}

// Undo the lower->upper rotations on the rows of U_b (m x k row-major),
// i = m-2 .. 0, drot(c, -s) (client.cpp:1127-1128).  One thread per column.
__global__ void rot_sweep(int m, int k, const double* __restrict__ cs, double* __restrict__ U) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= k) return;
  for (int i = m - 2; i >= 0; --i) {
    const double c = cs[2 * i], s = -cs[2 * i + 1];
    const double x = U[(long)i * k + j], y = U[(long)(i + 1) * k + j];
    U[(long)i * k + j] = c * x + s * y;
    U[(long)(i + 1) * k + j] = c * y - s * x;
  }
}

struct Layout {
  int P = 0;
  size_t m = 0, rg = 0;
  std::vector<size_t> n, r, rpos;
  std::vector<bool> qr;
};

bbt_status plan(bbt_ctx* ctx, const bbt_fedsvd_config* cfg, Layout& L) {
  if (!cfg || cfg->participants < 1 || !cfg->local_n || !cfg->private_seeds)
    return fail(ctx, BBT_ERR_ARG, "fedsvd: bad config");
  if (cfg->precision != 0) return fail(ctx, BBT_ERR_UNSUPPORTED, "fedsvd: precision mode %d", cfg->precision);
  L.P = cfg->participants;
  L.m = cfg->m;
  if (L.m < 3) return fail(ctx, BBT_ERR_UNSUPPORTED, "fedsvd: m=%zu (the reference needs m >= 3)", L.m);
  size_t gn = 0;
  L.rpos.push_back(0);
  for (int c = 0; c < L.P; ++c) {
    const size_t n = cfg->local_n[c];
    if (n < 1) return fail(ctx, BBT_ERR_ARG, "fedsvd: local_n[%d]=0", c);
    L.n.push_back(n);
    L.r.push_back(reduced_width(L.m, n));
    L.qr.push_back(has_local_qr(L.m, n));
    gn += n;
    L.rg += L.r.back();
    L.rpos.push_back(L.rg);
  }
  if (L.m > gn)
    return fail(ctx, BBT_ERR_UNSUPPORTED, "fedsvd: m=%zu > global_n=%zu (tall-and-skinny branch)", L.m, gn);
  if (L.rg <= L.m)
    return fail(ctx, BBT_ERR_UNSUPPORTED,
                "fedsvd: reduced_global_n=%zu <= m=%zu (the reference's V back-transform needs the global QR)",
                L.rg, L.m);
  if (L.m > (size_t)1 << 20) return fail(ctx, BBT_ERR_UNSUPPORTED, "fedsvd: m=%zu too large", L.m);
  return BBT_OK;
}

size_t scratch_bytes(const Layout& L) {
  QrPlan qp;
  size_t s = 0;
  for (int c = 0; c < L.P; ++c)
    if (L.qr[c]) s = std::max(s, qr_workspace_bytes((long)L.n[c], (int)L.m, (int)L.m, qp));
  s = std::max(s, qr_workspace_bytes((long)L.rg, (int)L.m, (int)L.m, qp));
  const size_t m = L.m;
  s = std::max(s, (7 * (m + 1) * m + 4 * m) * 8 + 4096);          // twisted
  s = std::max(s, (m + 2) * (1 + 8 + 1 + 7) * 48 + 4096);         // bisection nodes
  size_t mask = 0;
  for (int c = 0; c < L.P; ++c) mask = std::max(mask, (size_t)MASK_PASSES * (std::max(m, L.r[c]) + 1) * 24);
  s = std::max(s, mask + 4096);
  return s + (64u << 20);
}

size_t persistent_bytes(const Layout& L) {
  const size_t m = L.m;
  QrPlan qp;
  const size_t tq = ((m + qp.nb - 1) / qp.nb) * qp.nb * qp.nb;
  size_t b = 0;
  for (int c = 0; c < L.P; ++c) b += (m * m + m + tq) * 8 + 768;   // R^T, tau, T
  b += (m * L.rg + m + tq) * 8 + 768;                                // M, tau_g, T_g
  b += (4 * m * m + 6 * m) * 8 + 2048;                               // W, house, Vr, U_b(+V_b), alpha...
  b += m * m * 8 + 256;                                              // V_b
  b += m * std::max(m, L.rg) * 8 + 256;                              // tmp
  return b;
}

}  // namespace

size_t fedsvd_workspace_bytes(const bbt_fedsvd_config* cfg) {
  Layout L;
  bbt_ctx dummy;
  if (plan(&dummy, cfg, L) != BBT_OK) return 0;
  return persistent_bytes(L) + scratch_bytes(L);
}

bbt_status fedsvd(bbt_ctx* ctx, const bbt_fedsvd_config* cfg, double* const* X, double* sigma,
                  double* Uout, double* const* VT, int* kout) {
  Layout L;
  BBT_TRY(plan(ctx, cfg, L));
  const int P = L.P;
  const size_t m = L.m, rg = L.rg;
  const int mi = (int)m;
  BBT_CUDA(ctx, L.m ? cudaSuccess : cudaErrorInvalidValue);
  const size_t need = persistent_bytes(L) + scratch_bytes(L);
  if (ctx->ws.cap < need) BBT_CUDA(ctx, ctx->ws.reserve(need));
  ctx->ws.reset();
  QrPlan qp;
  const size_t tq = ((m + qp.nb - 1) / qp.nb) * qp.nb * qp.nb;
  std::vector<double*> RT(P), tauc(P), Tc(P);
  for (int c = 0; c < P; ++c) {
    RT[c] = ctx->ws.take<double>(m * m);
    tauc[c] = ctx->ws.take<double>(m);
    Tc[c] = ctx->ws.take<double>(tq);
  }
  double* M = ctx->ws.take<double>(m * rg);
  double* taug = ctx->ws.take<double>(m);
  double* Tg = ctx->ws.take<double>(tq);
  double* W = ctx->ws.take<double>(m * m);
  double* house = ctx->ws.take<double>(m * m);
  double* Vr = ctx->ws.take<double>(m * m);
  double* Ub = ctx->ws.take<double>(m * m);
  double* Vb = ctx->ws.take<double>(m * m);
  double* tauh = ctx->ws.take<double>(m);
  double* alpha = ctx->ws.take<double>(m);
  double* beta = ctx->ws.take<double>(m);
  double* cs = ctx->ws.take<double>(2 * m);
  double* scal = ctx->ws.take<double>(8);
  int* cnt = ctx->ws.take<int>(8);
  double* tmp = ctx->ws.take<double>(m * std::max(m, rg));
  if (!tmp) return fail(ctx, BBT_ERR_NOMEM, "fedsvd: workspace");

  cudaEvent_t ev[7];
  for (auto& e : ev) BBT_CUDA(ctx, cudaEventCreate(&e));
  struct EvGuard {
    cudaEvent_t* e;
    ~EvGuard() { for (int i = 0; i < 7; ++i) cudaEventDestroy(e[i]); }
  } guard{ev};
  BBT_CUDA(ctx, cudaEventRecord(ev[0], ctx->stream));

  // 1) local QR (client.cpp:572-589): A = X_c^T column-major n x m, in place
  std::vector<double*> masked(P);
  for (int c = 0; c < P; ++c) {
    if (L.qr[c]) {
      const long n = (long)L.n[c];
      BBT_TRY(geqrf(ctx, n, mi, X[c], n, tauc[c], Tc[c], qp));
      BBT_TRY(r_transpose(ctx, mi, X[c], n, RT[c]));
      BBT_TRY(orgqr(ctx, n, mi, X[c], n, tauc[c], Tc[c], qp));   // X_c <- Q (= local_v)
      masked[c] = RT[c];
    } else {
      masked[c] = X[c];
    }
  }
  BBT_CUDA(ctx, cudaEventRecord(ev[1], ctx->stream));
  // 2) masks (client.cpp:593-596)
  for (int c = 0; c < P; ++c) {
    BBT_TRY(block_shift_mask(ctx, m, L.r[c], MASK_PASSES, masked[c], true, true, cfg->public_seed));
    BBT_TRY(block_shift_mask(ctx, m, L.r[c], MASK_PASSES, masked[c], true, false, cfg->private_seeds[c]));
  }
  BBT_CUDA(ctx, cudaEventRecord(ev[2], ctx->stream));
  // 3) repartition + global QR of M^T (client.cpp:681-794)
  for (int c = 0; c < P; ++c)
    BBT_TRY(copy2d(ctx, mi, (int)L.r[c], masked[c], (long)L.r[c], M + L.rpos[c], (long)rg));
  BBT_TRY(geqrf(ctx, (long)rg, mi, M, (long)rg, taug, Tg, qp));
  r_rowmajor<<<4 * ctx->num_sms, 256, 0, ctx->stream>>>(mi, M, (long)rg, W);
  BBT_LAUNCHED(ctx);
  BBT_TRY(orgqr(ctx, (long)rg, mi, M, (long)rg, taug, Tg, qp));   // M <- Q_g (column-major rg x m)
  BBT_CUDA(ctx, cudaEventRecord(ev[3], ctx->stream));
  // 4) Ralha bidiagonalisation, lower -> upper (client.cpp:801-954)
  BBT_TRY(ralha(ctx, mi, W, house, tauh, alpha, beta, Vr, cs));
  BBT_CUDA(ctx, cudaEventRecord(ev[4], ctx->stream));
  // 5) singular values / vectors (client.cpp:963-995)
  BBT_TRY(bidiag_bound(ctx, mi, alpha, beta, scal));
  BBT_CUDA(ctx, cudaMemsetAsync(scal + 1, 0, sizeof(double), ctx->stream));
  BBT_TRY(sturm_counts(ctx, mi, alpha, beta, scal, 2, cnt));
  int hc[2];
  BBT_CUDA(ctx, cudaMemcpyAsync(hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, ctx->stream));
  BBT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  int k = hc[0] - hc[1];
  if (cfg->top_k > 0) k = std::min(k, cfg->top_k);
  if (k < 1) return fail(ctx, BBT_ERR_COUNT, "fedsvd: no singular values in (0, bound]");
  BBT_TRY(bidiag_svd(ctx, mi, alpha, beta, Ub, Vb, sigma, k, true));   // Ub m x k, Vb k x m
  BBT_CUDA(ctx, cudaEventRecord(ev[5], ctx->stream));
  // 6) U: FinalU (m x k row-major) = (V_b Vr)^T, unmasked (client.cpp:1018, 1071-1115)
  BBT_TRY(dgemm(ctx, true, true, k, mi, m, 1.0, Vb, (long)m, Vr, (long)m, 0.0, Uout, k));
  BBT_TRY(block_shift_mask(ctx, m, (size_t)k, MASK_PASSES, Uout, false, true, cfg->public_seed));
  //    V: U2 = H (G^T U_b) (client.cpp:1127-1176)
  rot_sweep<<<(k + 127) / 128, 128, 0, ctx->stream>>>(mi, k, cs, Ub);
  BBT_LAUNCHED(ctx);
  BBT_TRY(ormqr_left_notrans(ctx, (long)m, mi, house, (long)m, 1, tauh, Ub, k, k, true, qp));
  for (int c = 0; c < P; ++c) {   // :1179-1195
    const int rc = (int)L.r[c];
    // tmp (k x r_c row-major) = U2^T Q_g[rows_c, :]^T  ==  column-major r_c x k = Q_g[rows_c,:] U2
    BBT_TRY(dgemm(ctx, false, true, rc, k, m, 1.0, M + L.rpos[c], (long)rg, Ub, k, 0.0, tmp, rc));
    BBT_TRY(block_shift_mask(ctx, (size_t)k, (size_t)rc, MASK_PASSES, tmp, false, false, cfg->private_seeds[c]));
    const long n = (long)L.n[c];
    if (L.qr[c]) {   // FinalVT^T (n x k col-major) = Q_c (n x m) tmp^T (m x k)
      BBT_TRY(dgemm(ctx, false, false, (int)n, k, m, 1.0, X[c], n, tmp, rc, 0.0, VT[c], n));
    } else {
      BBT_CUDA(ctx, cudaMemcpyAsync(VT[c], tmp, (size_t)k * n * sizeof(double), cudaMemcpyDeviceToDevice,
                                    ctx->stream));
    }
  }
  BBT_CUDA(ctx, cudaEventRecord(ev[6], ctx->stream));
  BBT_CUDA(ctx, cudaEventSynchronize(ev[6]));
  for (int s = 0; s < 6; ++s) {
    float ms = 0;
    BBT_CUDA(ctx, cudaEventElapsedTime(&ms, ev[s], ev[s + 1]));
    ctx->stage_ms[s] = ms;
  }
  *kout = k;
  return BBT_OK;
}

}  // namespace bbt
