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

// Mode 0: place the leading kk x kk bidiagonal SVD into U_b (m x kk, rows >= kk
// zero) and V_b (kk x m, columns >= kk zero), as dbdsdc's outputs sit in the
// reference's zero-initialised buffers (client.cpp:973-978).
__global__ void embed_leading(int m, int kk, const double* __restrict__ Us, const double* __restrict__ Vs,
                              double* __restrict__ Ub, double* __restrict__ Vb) {
  const long total = (long)m * kk;
  for (long f = blockIdx.x * (long)blockDim.x + threadIdx.x; f < total; f += (long)gridDim.x * blockDim.x) {
    const int r = (int)(f / kk), c = (int)(f % kk);   // Ub (r, c)
    Ub[f] = r < kk ? Us[(long)r * kk + c] : 0.0;
    const int i = (int)(f / m), j = (int)(f % m);     // Vb (i, j)
    Vb[f] = j < kk ? Vs[(long)i * kk + j] : 0.0;
  }
}

struct Layout {
  int P = 0;
  int precision = 0;
  size_t m = 0, rg = 0, nmax = 0;
  std::vector<size_t> n, r, rpos;
  std::vector<bool> qr;
};

bbt_status plan(bbt_ctx* ctx, const bbt_fedsvd_config* cfg, Layout& L) {
  if (!cfg || cfg->participants < 1 || !cfg->local_n || !cfg->private_seeds)
    return fail(ctx, BBT_ERR_ARG, "fedsvd: bad config");
  if (cfg->precision != 0 && cfg->precision != 1)
    return fail(ctx, BBT_ERR_UNSUPPORTED, "fedsvd: precision mode %d (0 plain, 1 mixed)", cfg->precision);
  if (cfg->svd_mode < 0 || cfg->svd_mode > 3)
    return fail(ctx, BBT_ERR_UNSUPPORTED, "fedsvd: svd_mode %d (4, linear regression, is not built)", cfg->svd_mode);
  L.P = cfg->participants;
  L.m = cfg->m;
  L.precision = cfg->precision;
  if (L.m < 3) return fail(ctx, BBT_ERR_UNSUPPORTED, "fedsvd: m=%zu (the reference needs m >= 3)", L.m);
  size_t gn = 0;
  L.rpos.push_back(0);
  for (int c = 0; c < L.P; ++c) {
    const size_t n = cfg->local_n[c];
    if (n < 1) return fail(ctx, BBT_ERR_ARG, "fedsvd: local_n[%d]=0", c);
    L.n.push_back(n);
    L.nmax = std::max(L.nmax, n);
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

size_t qr_scratch(const bbt_ctx* ctx, const Layout& L, long rows, const QrPlan& qp) {
  if (L.precision == 1) return mixed_qr_workspace_bytes(ctx, (int)L.m, rows) + (8u << 20);
  return qr_workspace_bytes(rows, (int)L.m, (int)L.m, qp) + (8u << 20);
}

size_t scratch_bytes(const bbt_ctx* ctx, const Layout& L) {
  QrPlan qp;
  size_t s = 0;
  for (int c = 0; c < L.P; ++c)
    if (L.qr[c]) s = std::max(s, qr_scratch(ctx, L, (long)L.n[c], qp));
  if (L.precision == 1) {
    s = std::max(s, qr_scratch(ctx, L, (long)L.rg, qp));
    for (int c = 0; c < L.P; ++c)   // the V back-transform from int8 slices
      if (L.qr[c]) s = std::max(s, oz_workspace_bytes(ctx, (int)L.n[c], (int)L.m, (long)L.m, false) + (8u << 20));
  }
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
  if (L.precision == 1) {                                            // W_c, W_g, Z, R_g, the sketch S
    b += (size_t)(L.P + 3) * (m * m * 8 + 256);
    b += (size_t)sketch_rows((int)m) * sketch_pitch((long)std::max(L.nmax, L.rg)) * 2 + 256;
  }
  return b;
}

// ---- batched local QR (all participants, concurrent streams, CUDA graph) --

// What every participant's local QR needs besides its block: the precision
// mode, the shared sketch (mode 1) and the per-participant outputs.
struct QrJob {
  int precision = 0;
  const void* S = nullptr;
  long spitch = 0;
  std::vector<double*> RT, tau, T, W;
  bool compute_v = false;
};

// Participants needing a local QR, largest first, each to the stream with the
// least work so far (longest-processing-time order).
std::vector<std::vector<int>> schedule(const Layout& L, int streams) {
  std::vector<int> idx;
  for (int c = 0; c < L.P; ++c) if (L.qr[c]) idx.push_back(c);
  std::sort(idx.begin(), idx.end(), [&](int x, int y) { return L.n[x] > L.n[y]; });
  std::vector<std::vector<int>> out(streams);
  std::vector<double> load(streams, 0.0);
  for (int c : idx) {
    int s = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    out[s].push_back(c);
    load[s] += (double)L.n[c];
  }
  return out;
}

size_t batched_scratch(const bbt_ctx* ctx, const Layout& L, int streams, const QrPlan& qp) {
  if (streams <= 1) {
    size_t s = 0;
    for (int c = 0; c < L.P; ++c) if (L.qr[c]) s = std::max(s, qr_scratch(ctx, L, (long)L.n[c], qp));
    return s;
  }
  size_t tot = 0;
  for (auto& lst : schedule(L, streams)) {
    size_t s = 0;
    for (int c : lst) s = std::max(s, qr_scratch(ctx, L, (long)L.n[c], qp));
    tot += s + 4096;
  }
  return tot;
}

bbt_status qr_one(bbt_ctx* c, int mi, double* X, long n, int p, const QrJob& job, const QrPlan& qp) {
  if (job.precision == 1)   // R (column-major) is R^T row-major: the same bytes as r_transpose's output
    return mixed_local_qr(c, mi, n, X, job.S, job.spitch, job.RT[p], job.compute_v ? job.W[p] : nullptr);
  BBT_TRY(geqrf(c, n, mi, X, n, job.tau[p], job.T[p], qp));
  BBT_TRY(r_transpose(c, mi, X, n, job.RT[p]));
  if (job.compute_v) BBT_TRY(orgqr(c, n, mi, X, n, job.tau[p], job.T[p], qp));   // X_c <- Q (= local_v)
  return BBT_OK;
}

// Issue every participant's QR on its side stream (fork/join through events
// on ctx->stream).  Sub-contexts share the device arena in disjoint slices.
bbt_status issue_batched(bbt_ctx* ctx, const Layout& L, double* const* X, const QrJob& job, int streams,
                         const QrPlan& qp) {
  const int mi = (int)L.m;
  auto sched = schedule(L, streams);
  while ((int)ctx->side.size() < streams) {
    cudaStream_t st;
    BBT_CUDA(ctx, cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    ctx->side.push_back(st);
  }
  while ((int)ctx->side_ev.size() < streams + 1) {
    cudaEvent_t ev;
    BBT_CUDA(ctx, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    ctx->side_ev.push_back(ev);
  }
  BBT_CUDA(ctx, cudaEventRecord(ctx->side_ev[streams], ctx->stream));
  for (int s = 0; s < streams; ++s) {
    if (sched[s].empty()) continue;
    size_t slice = 0;
    for (int c : sched[s]) slice = std::max(slice, qr_scratch(ctx, L, (long)L.n[c], qp));
    char* base = ctx->ws.take<char>(slice);
    if (!base) return fail(ctx, BBT_ERR_NOMEM, "batched local QR: workspace slice");
    bbt_ctx sub;
    sub.device = ctx->device;
    sub.num_sms = ctx->num_sms;
    sub.stream = ctx->side[s];
    sub.ws.base = base;
    sub.ws.cap = slice;
    sub.allow_coop = false;
    sub.d_flag = ctx->d_flag;
    sub.d_barrier = ctx->d_barrier;
    BBT_CUDA(ctx, cudaStreamWaitEvent(sub.stream, ctx->side_ev[streams], 0));
    for (int c : sched[s]) {
      bbt_status st = qr_one(&sub, mi, X[c], (long)L.n[c], c, job, qp);
      if (st != BBT_OK) { ctx->err = sub.err; return st; }
    }
    ctx->launches += sub.launches;
    BBT_CUDA(ctx, cudaEventRecord(ctx->side_ev[s], sub.stream));
    BBT_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->side_ev[s], 0));
  }
  return BBT_OK;
}

bbt_status local_qr_stage(bbt_ctx* ctx, const Layout& L, double* const* X, const QrJob& job, int streams,
                          const QrPlan& qp, bool use_graph) {
  const int mi = (int)L.m;
  if (streams <= 1) {
    for (int c = 0; c < L.P; ++c)
      if (L.qr[c]) {
        if (ctx->io_on) BBT_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->in_ready[c], 0));
        BBT_TRY(qr_one(ctx, mi, X[c], (long)L.n[c], c, job, qp));
      }
    return BBT_OK;
  }
  if (ctx->io_on)   // the batched schedule (and its graph) starts once every block has arrived
    for (int c = 0; c < L.P; ++c) BBT_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->in_ready[c], 0));
  std::vector<size_t> key = {L.m, (size_t)job.compute_v, (size_t)streams, (size_t)qp.nb, (size_t)ctx->ws.base,
                             ctx->ws.cap, ctx->ws.top, (size_t)job.precision, (size_t)job.S};
  for (int c = 0; c < L.P; ++c) {
    key.push_back((size_t)X[c]);
    key.push_back(L.n[c]);
    key.push_back((size_t)job.RT[c]);
    key.push_back(job.W.empty() ? 0 : (size_t)job.W[c]);
  }
  if (!use_graph) return issue_batched(ctx, L, X, job, streams, qp);
  if (ctx->qr_graph && key == ctx->qr_key) {
    BBT_CUDA(ctx, cudaGraphLaunch(ctx->qr_graph, ctx->stream));
    ctx->launches += ctx->qr_graph_nodes;
    return BBT_OK;
  }
  if (ctx->qr_key != key) {   // first call with this shape: run eagerly (sets every kernel attribute)
    ctx->qr_key = key;
    if (ctx->qr_graph) { cudaGraphExecDestroy(ctx->qr_graph); ctx->qr_graph = nullptr; }
    return issue_batched(ctx, L, X, job, streams, qp);
  }
  // second call: capture the same schedule once, replay it from now on
  const uint64_t before = ctx->launches;
  const size_t top = ctx->ws.top;
  BBT_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed));
  bbt_status st = issue_batched(ctx, L, X, job, streams, qp);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
  if (st != BBT_OK) { if (g) cudaGraphDestroy(g); return st; }
  if (e != cudaSuccess) return cuda_fail(ctx, e, "batched local QR: capture");
  cudaGraphExec_t ex = nullptr;
  e = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "batched local QR: instantiate");
  ctx->qr_graph = ex;
  ctx->qr_graph_nodes = ctx->launches - before;
  ctx->ws.top = top;
  BBT_CUDA(ctx, cudaGraphLaunch(ctx->qr_graph, ctx->stream));
  return BBT_OK;
}

}  // namespace

size_t fedsvd_workspace_bytes(const bbt_fedsvd_config* cfg) {
  Layout L;
  bbt_ctx dummy;
  if (plan(&dummy, cfg, L) != BBT_OK) return 0;
  dummy.num_sms = 148;
  return persistent_bytes(L) + scratch_bytes(&dummy, L);
}

bbt_status fedsvd(bbt_ctx* ctx, const bbt_fedsvd_config* cfg, double* const* X, double* sigma,
                  double* Uout, double* const* VT, int* kout) {
  Layout L;
  BBT_TRY(plan(ctx, cfg, L));
  const int P = L.P;
  const size_t m = L.m, rg = L.rg;
  const int mi = (int)m;
  BBT_CUDA(ctx, L.m ? cudaSuccess : cudaErrorInvalidValue);
  QrPlan qp;
  int streams = 1;
  {
    int nqr = 0;
    for (int c = 0; c < P; ++c) nqr += L.qr[c];
    std::vector<size_t> skey = {L.m, (size_t)L.precision};
    for (int c = 0; c < P; ++c) skey.push_back(L.n[c]);
    if (ctx->tuned_streams > 0 && ctx->tuned_key == skey) {
      streams = ctx->tuned_streams;
      qp.nb = ctx->tuned_nb;
    } else if (nqr >= 8) {
      streams = 8;
    }
  }
  const size_t need =
      persistent_bytes(L) + std::max(scratch_bytes(ctx, L), batched_scratch(ctx, L, streams, qp) + (64u << 20));
  if (ctx->ws.cap < need) BBT_CUDA(ctx, ctx->ws.reserve(need));
  ctx->ws.reset();
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
  QrJob job;
  job.precision = L.precision;
  job.RT = RT;
  job.tau = tauc;
  job.T = Tc;
  double *Z = nullptr, *Wg = nullptr, *Rg = nullptr;
  void* S = nullptr;
  const long sk_cols = (long)std::max(L.nmax, L.rg);   // the sketch serves the local and the global QR
  if (L.precision == 1) {
    for (int c = 0; c < P; ++c) job.W.push_back(ctx->ws.take<double>(m * m));
    Z = ctx->ws.take<double>(m * m);
    Wg = ctx->ws.take<double>(m * m);
    Rg = ctx->ws.take<double>(m * m);
    S = ctx->ws.take<char>((size_t)sketch_rows(mi) * sketch_pitch(sk_cols) * 2);
    if (!S) return fail(ctx, BBT_ERR_NOMEM, "fedsvd: workspace (mixed precision)");
    job.S = S;
    job.spitch = sketch_pitch(sk_cols);
  }

  cudaEvent_t ev[7];
  for (auto& e : ev) BBT_CUDA(ctx, cudaEventCreate(&e));
  struct EvGuard {
    cudaEvent_t* e;
    ~EvGuard() { for (int i = 0; i < 7; ++i) cudaEventDestroy(e[i]); }
  } guard{ev};
  BBT_CUDA(ctx, cudaEventRecord(ev[0], ctx->stream));

  // 1) local QR (client.cpp:572-589): A = X_c^T column-major n x m, in place
  const bool compute_u = cfg->svd_mode != 3, compute_v = cfg->svd_mode != 2;   // client.cpp:491-492
  job.compute_v = compute_v;
  std::vector<double*> masked(P);
  for (int c = 0; c < P; ++c) masked[c] = L.qr[c] ? RT[c] : X[c];
  if (L.precision == 1) {
    BBT_TRY(rademacher(ctx, sketch_rows(mi), sk_cols, S, 0x5EED5EEDull));
    BBT_TRY(clear_tc_flags(ctx));
  }
  {
    const size_t mark = ctx->ws.top;
    BBT_TRY(local_qr_stage(ctx, L, X, job, streams, qp, true));
    ctx->ws.top = mark;
  }
  if (L.precision == 1) BBT_TRY(check_tc_flags(ctx, "fedsvd: mixed-precision local QR"));
  if (ctx->io_on)
    for (int c = 0; c < P; ++c) BBT_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->in_ready[c], 0));
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
  if (L.precision == 1) {   // M <- Q_p, Q_g = Q_p W_g, R_g with dgeqrf's signs (mixedqr.cu)
    const size_t mark = ctx->ws.top;
    BBT_TRY(mixed_local_qr(ctx, mi, (long)rg, M, S, job.spitch, Rg, compute_v ? Wg : nullptr));
    ctx->ws.top = mark;
    BBT_TRY(transpose(ctx, mi, mi, Rg, (long)m, W, (long)m));   // W (row-major) = R_g
    BBT_TRY(check_tc_flags(ctx, "fedsvd: mixed-precision global QR"));
  } else {
    BBT_TRY(geqrf(ctx, (long)rg, mi, M, (long)rg, taug, Tg, qp));
    r_rowmajor<<<4 * ctx->num_sms, 256, 0, ctx->stream>>>(mi, M, (long)rg, W);
    BBT_LAUNCHED(ctx);
    if (compute_v) BBT_TRY(orgqr(ctx, (long)rg, mi, M, (long)rg, taug, Tg, qp));   // M <- Q_g (rg x m)
  }
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
  if (cfg->svd_mode == 0 && k < mi) {
    // dbdsdc on the leading k x k bidiagonal (client.cpp:975-980)
    double* Us = tmp;   // k x k each; the Ralha input W is free by now
    double* Vs = W;
    BBT_TRY(bidiag_svd(ctx, k, alpha, beta, Us, Vs, sigma, k, true));
    embed_leading<<<4 * ctx->num_sms, 256, 0, ctx->stream>>>(mi, k, Us, Vs, Ub, Vb);
    BBT_LAUNCHED(ctx);
  } else {
    BBT_TRY(bidiag_svd(ctx, mi, alpha, beta, Ub, Vb, sigma, k, true));   // Ub m x k, Vb k x m
  }
  BBT_CUDA(ctx, cudaEventRecord(ev[5], ctx->stream));
  // 6) U: FinalU (m x k row-major) = (V_b Vr)^T, unmasked (client.cpp:1018, 1071-1115)
  if (compute_u) {
    BBT_TRY(dgemm(ctx, true, true, k, mi, m, 1.0, Vb, (long)m, Vr, (long)m, 0.0, Uout, k));
    BBT_TRY(block_shift_mask(ctx, m, (size_t)k, MASK_PASSES, Uout, false, true, cfg->public_seed));
  }
  //    V: U2 = H (G^T U_b) (client.cpp:1127-1176)
  if (compute_v) {
  rot_sweep<<<(k + 127) / 128, 128, 0, ctx->stream>>>(mi, k, cs, Ub);
  BBT_LAUNCHED(ctx);
  BBT_TRY(ormqr_left_notrans(ctx, (long)m, mi, house, (long)m, 1, tauh, Ub, k, k, true, qp));
  if (L.precision == 1)   // Q_g U2 = Q_p (W_g U2): Rg (free by now) <- W_g U2, m x k column-major
    BBT_TRY(dgemm(ctx, false, true, mi, k, m, 1.0, Wg, (long)m, Ub, k, 0.0, Rg, (long)m));
  for (int c = 0; c < P; ++c) {   // :1179-1195
    const int rc = (int)L.r[c];
    // tmp (k x r_c row-major) = U2^T Q_g[rows_c, :]^T  ==  column-major r_c x k = Q_g[rows_c,:] U2
    if (L.precision == 1)
      BBT_TRY(dgemm(ctx, false, false, rc, k, m, 1.0, M + L.rpos[c], (long)rg, Rg, (long)m, 0.0, tmp, rc));
    else
      BBT_TRY(dgemm(ctx, false, true, rc, k, m, 1.0, M + L.rpos[c], (long)rg, Ub, k, 0.0, tmp, rc));
    BBT_TRY(block_shift_mask(ctx, (size_t)k, (size_t)rc, MASK_PASSES, tmp, false, false, cfg->private_seeds[c]));
    const long n = (long)L.n[c];
    if (L.qr[c] && L.precision == 1) {   // Q_c = Q_p W_c: FinalVT^T = Q_p (W_c tmp^T)
      BBT_TRY(dgemm(ctx, false, false, mi, k, m, 1.0, job.W[c], (long)m, tmp, rc, 0.0, Z, (long)m));
      if (oz_worthwhile((int)n, k, (long)m))   // FinalVT^T (n x k) = Q_p Z from exact int8 slices; 6 slices
        BBT_TRY(gemm_oz(ctx, (int)n, k, (long)m, 1.0, X[c], 1, n, Z, (long)m, 1, 0.0, VT[c], n, false, false, 6));
      else
        BBT_TRY(dgemm(ctx, false, false, (int)n, k, m, 1.0, X[c], n, Z, (long)m, 0.0, VT[c], n));
    } else if (L.qr[c]) {   // FinalVT^T (n x k col-major) = Q_c (n x m) tmp^T (m x k)
      BBT_TRY(dgemm(ctx, false, false, (int)n, k, m, 1.0, X[c], n, tmp, rc, 0.0, VT[c], n));
    } else {
      BBT_CUDA(ctx, cudaMemcpyAsync(VT[c], tmp, (size_t)k * n * sizeof(double), cudaMemcpyDeviceToDevice,
                                    ctx->stream));
    }
    if (ctx->io_on && ctx->vt_dst[c]) {   // FinalVT_c leaves while the next participant is computed
      BBT_CUDA(ctx, cudaEventRecord(ctx->vt_done[c], ctx->stream));
      BBT_CUDA(ctx, cudaStreamWaitEvent(ctx->copy_out, ctx->vt_done[c], 0));
      BBT_CUDA(ctx, cudaMemcpyAsync(ctx->vt_dst[c], VT[c], (size_t)k * n * sizeof(double), cudaMemcpyDeviceToHost,
                                    ctx->copy_out));
    }
  }
  }
  BBT_CUDA(ctx, cudaEventRecord(ev[6], ctx->stream));
  BBT_CUDA(ctx, cudaEventSynchronize(ev[6]));
  if (L.precision == 1) BBT_TRY(check_tc_flags(ctx, "fedsvd: tensor-core back-transform"));
  for (int s = 0; s < 6; ++s) {
    float ms = 0;
    BBT_CUDA(ctx, cudaEventElapsedTime(&ms, ev[s], ev[s + 1]));
    ctx->stage_ms[s] = ms;
  }
  *kout = k;
  return BBT_OK;
}

namespace {
__global__ void fill_hash(double* __restrict__ x, size_t n, unsigned seed) {
  for (size_t f = blockIdx.x * (size_t)blockDim.x + threadIdx.x; f < n; f += (size_t)gridDim.x * blockDim.x) {
    unsigned h = (unsigned)f * 2654435761u ^ seed * 97u;
    h ^= h >> 13; h *= 0x5bd1e995u; h ^= h >> 15;
    x[f] = (double)(h & 0xffffff) / 16777216.0 - 0.5;
  }
}
}  // namespace

// Autotuner of the batched local QR: times every (streams, panel width)
// candidate on synthetic blocks of the configuration's shapes and keeps the
// fastest for later fedsvd calls with the same shapes.
bbt_status fedsvd_tune(bbt_ctx* ctx, const bbt_fedsvd_config* cfg, int* best_streams, int* best_nb, double* best_ms) {
  Layout L;
  BBT_TRY(plan(ctx, cfg, L));
  const int P = L.P, mi = (int)L.m;
  std::vector<double*> blocks(P, nullptr);
  struct Free {
    std::vector<double*>& b;
    ~Free() { for (auto p : b) if (p) cudaFree(p); }
  } fr{blocks};
  for (int c = 0; c < P; ++c)
    if (L.qr[c]) BBT_CUDA(ctx, cudaMalloc(&blocks[c], L.m * L.n[c] * sizeof(double)));
  const int cand_s[] = {1, 4, 8, 16};
  // the panel width only matters to the Householder (precision 0) path
  const std::vector<int> cand_nb = L.precision == 1 ? std::vector<int>{128} : std::vector<int>{64, 128};
  size_t need = 0;
  for (int nb : cand_nb)
    for (int st : cand_s) {
      QrPlan qp;
      qp.nb = nb;
      need = std::max(need, batched_scratch(ctx, L, st, qp));
    }
  const size_t tq = ((L.m + 63) / 64) * 128 * 128;
  const size_t sbytes = (size_t)sketch_rows(mi) * sketch_pitch((long)L.nmax) * 2;
  need += (size_t)P * (L.m * L.m + L.m + tq) * 8 + (size_t)P * 1024 + (64u << 20);
  if (L.precision == 1) need += (size_t)P * (L.m * L.m * 8 + 256) + sbytes + 256;
  if (ctx->ws.cap < need) BBT_CUDA(ctx, ctx->ws.reserve(need));
  ctx->ws.reset();
  QrJob job;
  job.precision = L.precision;
  job.compute_v = true;
  for (int c = 0; c < P; ++c) {
    job.RT.push_back(ctx->ws.take<double>(L.m * L.m));
    job.tau.push_back(ctx->ws.take<double>(L.m));
    job.T.push_back(ctx->ws.take<double>(tq));
    if (L.precision == 1) job.W.push_back(ctx->ws.take<double>(L.m * L.m));
  }
  if (L.precision == 1) {
    void* S = ctx->ws.take<char>(sbytes);
    if (!S) return fail(ctx, BBT_ERR_NOMEM, "tune: workspace");
    BBT_TRY(rademacher(ctx, sketch_rows(mi), (long)L.nmax, S, 0x5EED5EEDull));
    job.S = S;
    job.spitch = sketch_pitch((long)L.nmax);
  }
  cudaEvent_t e0, e1;
  BBT_CUDA(ctx, cudaEventCreate(&e0));
  BBT_CUDA(ctx, cudaEventCreate(&e1));
  double best = 1e300;
  int bs = 1, bnb = 128;
  for (int nb : cand_nb)
    for (int st : cand_s) {
      QrPlan qp;
      qp.nb = nb;
      for (int rep = 0; rep < 2; ++rep) {   // first repetition warms the kernels up
        for (int c = 0; c < P; ++c)
          if (blocks[c]) {
            fill_hash<<<4 * ctx->num_sms, 256, 0, ctx->stream>>>(blocks[c], L.m * L.n[c], (unsigned)c + 1);
            BBT_LAUNCHED(ctx);
          }
        const size_t mark = ctx->ws.top;
        BBT_CUDA(ctx, cudaEventRecord(e0, ctx->stream));
        BBT_TRY(local_qr_stage(ctx, L, blocks.data(), job, st, qp, false));
        BBT_CUDA(ctx, cudaEventRecord(e1, ctx->stream));
        BBT_CUDA(ctx, cudaEventSynchronize(e1));
        ctx->ws.top = mark;
        float ms = 0;
        BBT_CUDA(ctx, cudaEventElapsedTime(&ms, e0, e1));
        if (rep == 1 && ms < best) { best = ms; bs = st; bnb = nb; }
      }
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ctx->tuned_streams = bs;
  ctx->tuned_nb = bnb;
  ctx->tuned_key = {L.m, (size_t)L.precision};
  for (int c = 0; c < P; ++c) ctx->tuned_key.push_back(L.n[c]);
  (void)mi;
  if (best_streams) *best_streams = bs;
  if (best_nb) *best_nb = bnb;
  if (best_ms) *best_ms = best;
  return BBT_OK;
}

bbt_status svd_dense(bbt_ctx* ctx, int m, double* X, int top_k, double* sigma, double* Uout, double* VTout,
                     int* kout) {
  if (m < 3) return fail(ctx, BBT_ERR_UNSUPPORTED, "svd_dense: m=%d", m);
  const size_t mm = (size_t)m * m;
  QrPlan qp;
  size_t scratch = std::max(qr_workspace_bytes(m, m, m, qp), (7 * ((size_t)m + 1) * m + 4 * (size_t)m) * 8 + 4096);
  scratch = std::max(scratch, ((size_t)m + 2) * 17 * 48 + 4096) + (64u << 20);
  const size_t need = (2 * mm + 8 * (size_t)m + 64) * 8 + 4096 + scratch;
  if (ctx->ws.cap < need) BBT_CUDA(ctx, ctx->ws.reserve(need));
  ctx->ws.reset();
  double* Ub = ctx->ws.take<double>(mm);
  double* Vb = ctx->ws.take<double>(mm);
  double* d = ctx->ws.take<double>(m);
  double* e = ctx->ws.take<double>(m);
  double* tauq = ctx->ws.take<double>(m);
  double* taup = ctx->ws.take<double>(m);
  double* scal = ctx->ws.take<double>(8);
  int* cnt = ctx->ws.take<int>(8);
  if (!cnt) return fail(ctx, BBT_ERR_NOMEM, "svd_dense: workspace");
  // A = the buffer read column-major = X^T;  A = Q B P^T (two-sided Householder)
  double* A = X;
  BBT_TRY(gebrd(ctx, m, A, d, e, tauq, taup));
  BBT_TRY(bidiag_bound(ctx, m, d, e, scal));
  BBT_CUDA(ctx, cudaMemsetAsync(scal + 1, 0, sizeof(double), ctx->stream));
  BBT_TRY(sturm_counts(ctx, m, d, e, scal, 2, cnt));
  int hc[2];
  BBT_CUDA(ctx, cudaMemcpyAsync(hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, ctx->stream));
  BBT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  int k = hc[0] - hc[1];
  if (top_k > 0) k = std::min(k, top_k);
  if (k < 1) return fail(ctx, BBT_ERR_COUNT, "svd_dense: no singular values in (0, bound]");
  BBT_TRY(bidiag_svd(ctx, m, d, e, Ub, Vb, sigma, k, true));   // B = U_b S V_b^T
  int ncl = 0;
  BBT_TRY(refine_clusters(ctx, m, k, d, e, sigma, Ub, Vb, &ncl));   // vectors inside tight clusters
  // X = A^T = (P V_b^T) S (Q U_b)^T
  BBT_TRY(ormqr_left_notrans(ctx, (long)m, m, A, 1, (long)m, tauq, Ub, k, k, true, qp));   // Ub <- Q Ub
  BBT_TRY(ormqr_left_notrans(ctx, (long)m - 1, m - 1, A + m, (long)m, 1, taup, Vb + 1, (long)m, k, false,
                             qp));                                                        // V_b^T <- P V_b^T
  BBT_TRY(transpose(ctx, k, m, Vb, m, Uout, k));    // U (m x k) = P V_b^T
  BBT_TRY(transpose(ctx, m, k, Ub, k, VTout, m));   // VT (k x m) = (Q U_b)^T
  BBT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  *kout = k;
  return BBT_OK;
}

}  // namespace bbt
