// DecentralizedClient::run() (Excalibur src/client.cpp:447-1200) for P
// participants held as separate device buffers on one GPU.
//
// Short-and-wide branch (m <= global_n), opt_control 3:
//   local QR of every wide block (local_n / m > 5)          client.cpp:572-589
//   public (row) then private (column) Givens masks          :593-596
//   repartition = the column concatenation M = [M_0 | ...]  :681-703
//   Householder QR of M^T, Q_g kept (none if m == global_n)  :705-798
//   Ralha bidiagonalisation of R_g                           :801-954
//   bisection + twisted vectors, sign convention            :963-995
//   FinalU = unmask_pub((V_b Vr)^T)                          :1002-1115
//   FinalVT_c = unmask_priv_c(U2^T Q_g[c]^T) Q_c^T           :1174-1195
//     (m == global_n: unmask_priv_c(U2[rows of c]^T))        :1129-1169
// Tall-and-skinny branch (m > global_n): fedsvd_tall below.
// The ring all-reduce / all-gather of the reference become reductions
// inside the kernels (Ralha) or plain device-memory reads (U all-gather).
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <vector>

#include <cstring>
#include <thread>

#include "internal.h"

namespace bbt {
namespace {

// Host-side NVTX ranges, one per phase of a pipeline call, named as the
// reference's phase timers (client.hpp:83-84: local_qr, apply_mask,
// global_qr, bi_diag, bsvd, combine_svd_remove_mask), each opened where the
// phase's start event is recorded, so a trace lines up with the reference's
// log lines.  Without a tool attached NVTX calls do nothing.
struct PhaseRanges {
  bool open = false;
  void next(const char* name) {
    if (open) nvtxRangePop();
    nvtxRangePushA(name);
    open = true;
  }
  void close() {
    if (open) nvtxRangePop();
    open = false;
  }
  ~PhaseRanges() { close(); }
};

constexpr int MASK_PASSES = 32;            // client.cpp:536
constexpr size_t MASK_SCRATCH_CAP = (size_t)2 << 30;
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

// Scale each of k entries of x by 1/sigma (client.cpp:1045).
__global__ void div_sigma(int k, const double* __restrict__ sigma, double* __restrict__ x) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < k) x[j] = x[j] / sigma[j];
}

struct Layout {
  int P = 0;
  int precision = 0;
  size_t m = 0, rg = 0, nmax = 0;
  std::vector<size_t> n, r, rpos;
  std::vector<bool> qr;
  // tall-and-skinny branch (m > global_n): column slabs of X
  bool tall = false;
  size_t gn = 0, wn = 0;              // global_n; Ralha columns sum_c min(m_part[c], global_n)
  std::vector<size_t> npos;           // n_pos
  std::vector<size_t> part, ppos;     // m_part / m_part_pos (client.cpp:613-624)
  std::vector<size_t> wpos;           // slab c's first column in the Ralha matrix
};

// The slab QRs of the tall-and-skinny branch as a short-and-wide local-QR
// layout: slab c is global_n x m_part[c] row-major (= column-major A of
// m_part[c] x global_n, the shape local_qr_reduction(m_part, global_n) takes,
// client.cpp:661-667), reduced when m_part[c] > global_n.
Layout slab_layout(const Layout& L) {
  Layout q;
  q.P = L.P;
  q.precision = L.precision;
  q.m = L.gn;
  q.rpos.push_back(0);
  for (int c = 0; c < L.P; ++c) {
    q.n.push_back(L.part[c]);
    q.nmax = std::max(q.nmax, L.part[c]);
    q.qr.push_back(L.part[c] > L.gn);
    q.r.push_back(std::min(L.part[c], L.gn));
    q.rg += q.r.back();
    q.rpos.push_back(q.rg);
  }
  return q;
}

bbt_status plan(bbt_ctx* ctx, const bbt_fedsvd_config* cfg, Layout& L) {
  if (!cfg || cfg->participants < 1 || !cfg->local_n || !cfg->private_seeds)
    return fail(ctx, BBT_ERR_ARG, "fedsvd: bad config");
  if (cfg->precision < 0 || cfg->precision > 2)
    return fail(ctx, BBT_ERR_UNSUPPORTED, "fedsvd: precision mode %d (0 plain, 1 mixed, 2 exact Gram)",
                cfg->precision);
  if (cfg->svd_mode < 0 || cfg->svd_mode > 4)
    return fail(ctx, BBT_ERR_UNSUPPORTED, "fedsvd: svd_mode %d (0..4)", cfg->svd_mode);
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
  L.gn = gn;
  L.tall = L.m > gn;
  if (L.tall && L.precision == 2) L.precision = 1;   // the slab QRs of the tall branch run as mode 1
  L.npos.push_back(0);
  for (int c = 0; c < L.P; ++c) L.npos.push_back(L.npos.back() + L.n[c]);
  if (cfg->svd_mode == 4 && !L.tall)
    return fail(ctx, BBT_ERR_UNSUPPORTED,
                "fedsvd: svd_mode 4 (linear regression) needs m > global_n, the reference's vertical layout "
                "(client.cpp:1180)");
  if (cfg->svd_mode == 4 && !cfg->labels) return fail(ctx, BBT_ERR_ARG, "fedsvd: svd_mode 4 without labels");
  if (L.tall) {
    if (gn < 3) return fail(ctx, BBT_ERR_UNSUPPORTED, "fedsvd: global_n=%zu (the bidiagonal needs >= 3)", gn);
    if (gn > (size_t)1 << 16) return fail(ctx, BBT_ERR_UNSUPPORTED, "fedsvd: global_n=%zu too large", gn);
    if (L.m > ((size_t)1 << 31) - 1) return fail(ctx, BBT_ERR_UNSUPPORTED, "fedsvd: m=%zu too large", L.m);
    L.ppos.push_back(0);
    for (int c = 0; c < L.P; ++c) {   // row_split (client.cpp:613-624)
      L.part.push_back(L.m / L.P + ((size_t)c < L.m % L.P ? 1 : 0));
      L.ppos.push_back(L.ppos.back() + L.part.back());
      L.wpos.push_back(L.wn);
      L.wn += std::min(L.part.back(), gn);
    }
    for (int c = 0; c < L.P; ++c)
      if (L.part[c] < 1) return fail(ctx, BBT_ERR_UNSUPPORTED, "fedsvd: m=%zu < P=%d", L.m, L.P);
    return BBT_OK;
  }
  if (L.rg <= L.m && L.m < gn)
    return fail(ctx, BBT_ERR_UNSUPPORTED,
                "fedsvd: reduced_global_n=%zu <= m=%zu (the reference's V back-transform needs the global QR)",
                L.rg, L.m);
  if (L.rg == L.m) L.precision = 0;   // m == global_n: no QR anywhere, nothing to run in split precision
  if (L.m > (size_t)1 << 20) return fail(ctx, BBT_ERR_UNSUPPORTED, "fedsvd: m=%zu too large", L.m);
  return BBT_OK;
}

size_t qr_scratch(const bbt_ctx* ctx, const Layout& L, long rows, const QrPlan& qp) {
  if (L.precision == 1) return mixed_qr_workspace_bytes(ctx, (int)L.m, rows) + (8u << 20);
  if (L.precision == 2) return exact_qr_workspace_bytes(ctx, (int)L.m, rows) + (8u << 20);
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
  if (L.precision == 2) {   // the global QR and the exact products with the implicit Q's
    s = std::max(s, qr_scratch(ctx, L, (long)L.rg, qp));
    s += exact_operand_bytes((int)L.m, (int)L.m);   // the global chain's prepared operand stays taken
    for (int c = 0; c < L.P; ++c) {
      s = std::max(s, exact_apply_workspace_bytes(ctx, (long)L.r[c], (int)L.m, (int)L.m) + (8u << 20));
      if (L.qr[c]) s = std::max(s, exact_apply_workspace_bytes(ctx, (long)L.n[c], (int)L.m, (int)L.m) + (8u << 20));
    }
  }
  s = std::max(s, qr_workspace_bytes((long)L.rg, (int)L.m, (int)L.m, qp));
  const size_t m = L.m;
  s = std::max(s, (7 * (m + 1) * m + 4 * m) * 8 + 4096);          // twisted
  s = std::max(s, bisect_workspace_bytes((int)m, (int)m) + 16 * m);   // bisection nodes, brackets
  size_t mask = mask_workspace_bytes(m, m, MASK_PASSES, true);   // FinalU (m x k, k <= m)
  for (int c = 0; c < L.P; ++c)
    mask = std::max({mask, mask_workspace_bytes(m, L.r[c], MASK_PASSES, true),
                     mask_workspace_bytes(m, L.r[c], MASK_PASSES, false)});
  s = std::max(s, std::min(mask, MASK_SCRATCH_CAP) + 4096);   // larger masks run in batches of vectors
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
  if (L.precision >= 1) {                                            // W_c, W_g, Z, R_g, the sketch S
    b += (size_t)(L.P + 3) * (m * m * 8 + 256);
    b += (size_t)sketch_rows((int)m) * sketch_pitch((long)std::max(L.nmax, L.rg)) * 2 + 256;
  }
  if (L.precision == 2) b += (size_t)(L.P + 1) * ((m * m + m) * 8 + 512);   // R_p and the row scales
  return b;
}

// ---- the masks' random tables, drawn while the local QRs run -------------
// Every mask of a short-and-wide call is known from the shapes and seeds
// alone: the public row mask and each participant's private column mask
// (client.cpp:593-596) and their inverses (:1109, :1182).  Their tables are
// drawn with the reference's own calls (glibc rand() and
// std::default_random_engine, so bit for bit the tables the reference draws)
// on a host thread while the GPU runs the local QRs, then uploaded at once
// through pinned memory; each mask is then a single launch with no host work.
// Rotated lengths above 10000 (the virtual-matrix path) draw theirs in place.
struct MaskPrefetch {
  struct Key {
    size_t k;
    bool mask;
    unsigned seed;
  };
  std::vector<Key> keys;
  std::vector<GivensTables> tabs;
  std::vector<GivensDev> dev;
  std::thread th;
  bool failed = false;

  int find(size_t k, bool mask, unsigned seed) const {
    for (size_t i = 0; i < keys.size(); ++i)
      if (keys[i].k == k && keys[i].mask == mask && keys[i].seed == seed) return (int)i;
    return -1;
  }
  void add(size_t k, bool mask, unsigned seed) {
    if (k < 2 || k > 10000 || find(k, mask, seed) >= 0) return;
    keys.push_back({k, mask, seed});
  }
  static size_t ops(size_t k) { return (k + (k & 1)) / 2; }
  size_t bytes() const {
    size_t b = 0;
    for (const Key& key : keys) b += MASK_PASSES * ops(key.k) * (sizeof(int2) + sizeof(double2)) + 512;
    return b;
  }
  void start() {
    tabs.resize(keys.size());
    th = std::thread([this] {
      try {
        for (size_t i = 0; i < keys.size(); ++i)
          draw_givens_tables(keys[i].k, MASK_PASSES, keys[i].mask, keys[i].seed, tabs[i]);
      } catch (...) {
        failed = true;
      }
    });
  }
  // Joins the drawing thread and copies every table into the device slab.
  bbt_status upload(bbt_ctx* ctx, char* slab) {
    if (th.joinable()) th.join();
    if (failed) return fail(ctx, BBT_ERR_NOMEM, "fedsvd: mask tables");
    if (keys.empty()) return BBT_OK;
    const size_t total = bytes();
    if (ctx->mask_pinned_cap < total) {
      if (ctx->mask_pinned) cudaFreeHost(ctx->mask_pinned);
      ctx->mask_pinned = nullptr;
      ctx->mask_pinned_cap = 0;
      BBT_CUDA(ctx, cudaMallocHost(&ctx->mask_pinned, total));
      ctx->mask_pinned_cap = total;
    }
    char* h = static_cast<char*>(ctx->mask_pinned);
    size_t off = 0;
    dev.resize(keys.size());
    for (size_t i = 0; i < keys.size(); ++i) {
      const GivensTables& T = tabs[i];
      GivensDev& D = dev[i];
      D.k = T.k;
      D.passes = T.passes;
      D.ops = T.ops;
      D.b1 = T.b1;
      D.b2 = T.b2;
      off = (off + 255) & ~size_t(255);
      std::memcpy(h + off, T.pairs.data(), T.pairs.size() * sizeof(int2));
      D.pairs = reinterpret_cast<const int2*>(slab + off);
      off += T.pairs.size() * sizeof(int2);
      off = (off + 255) & ~size_t(255);
      std::memcpy(h + off, T.cs.data(), T.cs.size() * sizeof(double2));
      D.cs = reinterpret_cast<const double2*>(slab + off);
      off += T.cs.size() * sizeof(double2);
    }
    BBT_CUDA(ctx, cudaMemcpyAsync(slab, h, off, cudaMemcpyHostToDevice, ctx->stream));
    return BBT_OK;
  }
  ~MaskPrefetch() {
    if (th.joinable()) th.join();
  }
};

// A mask with its prefetched tables, or drawn in place.
bbt_status apply_mask(bbt_ctx* ctx, const MaskPrefetch& pf, size_t m, size_t n, double* x, bool mask, bool is_left,
                      unsigned seed) {
  const int i = pf.find(is_left ? m : n, mask, seed);
  if (i >= 0 && (size_t)i < pf.dev.size()) return apply_givens(ctx, pf.dev[i], m, n, x, is_left);
  return block_shift_mask(ctx, m, n, MASK_PASSES, x, mask, is_left, seed);
}

// ---- batched local QR (all participants, concurrent streams, CUDA graph) --

// What every participant's local QR needs besides its block: the precision
// mode, the shared sketch (mode 1) and the per-participant outputs.
struct QrJob {
  int precision = 0;
  const void* S = nullptr;
  long spitch = 0;
  std::vector<double*> RT, tau, T, W;
  std::vector<double*> Rp, scale;   // precision 2: the preconditioner and X's row scales
  std::vector<int8_t*> planes;      // precision 2: X_int's residue planes kept for the V back-transform (or null)
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
  if (job.precision == 2)   // X kept: Q = X_int^T Rp^-1 W is applied by exact products
    return exact_local_qr(c, mi, n, X, job.S, job.spitch, job.RT[p], job.W[p], job.Rp[p], job.scale[p],
                          job.planes.empty() ? nullptr : job.planes[p]);
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
        if (ctx->io_on) BBT_TRY(wait_input(ctx, c));
        BBT_TRY(qr_one(ctx, mi, X[c], (long)L.n[c], c, job, qp));
      }
    return BBT_OK;
  }
  if (ctx->io_on)   // the batched schedule (and its graph) starts once every block has arrived
    for (int c = 0; c < L.P; ++c) BBT_TRY(wait_input(ctx, c));
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

// ---- tall-and-skinny branch (m > global_n) --------------------------------

size_t tall_persistent_bytes(const Layout& L, const Layout& Q, int svd_mode) {
  const size_t g = L.gn, m = L.m;
  QrPlan qp;
  const size_t tq = ((g + qp.nb - 1) / qp.nb) * qp.nb * qp.nb;
  size_t b = 0;
  for (int c = 0; c < L.P; ++c)
    if (Q.qr[c]) {
      b += g * L.part[c] * 8 + 256;              // the slab, then its Q (or Q_p)
      b += (g * g + g + tq) * 8 + 768;           // R^T, tau, T
      if (L.precision == 1) b += g * g * 8 + 256;   // W_c
    }
  b += 2 * (g * L.wn * 8 + 256);                 // Ralha matrix, Vr
  b += 5 * (g * g * 8 + 256) + (6 * g + 16) * 8 + 2048;   // house, U_b, V_b, tmp, Z; tau, alpha, beta, cs
  if (L.precision == 1) b += (size_t)sketch_rows((int)g) * sketch_pitch((long)Q.nmax) * 2 + 256;
  if (svd_mode == 4) b += (m * g + m + 2 * g) * 8 + 1024;   // U (k x m), masked y, Sigma^-1 U^T y, w
  return b;
}

size_t tall_scratch_bytes(const bbt_ctx* ctx, const Layout& L, const Layout& Q) {
  QrPlan qp;
  const size_t g = L.gn;
  size_t s = 0;
  for (int c = 0; c < L.P; ++c)
    if (Q.qr[c]) {
      s = std::max(s, qr_scratch(ctx, Q, (long)L.part[c], qp));
      if (L.precision == 1)   // FinalU parts from int8 slices
        s = std::max(s, oz_workspace_bytes(ctx, (int)L.part[c], (int)g, (long)g, false) + (8u << 20));
    }
  s = std::max(s, qr_workspace_bytes((long)g, (int)g, (int)g, qp));   // the reflectors of Ralha on U_b
  s = std::max(s, (7 * (g + 1) * g + 4 * g) * 8 + 4096);              // twisted
  s = std::max(s, bisect_workspace_bytes((int)g, (int)g) + 16 * g);       // bisection nodes, brackets
  size_t mask = std::max(mask_workspace_bytes(g, L.m, MASK_PASSES, false),    // FinalU (k x m, k <= g)
                         mask_workspace_bytes(1, L.m, MASK_PASSES, false));   // y
  for (int c = 0; c < L.P; ++c)
    mask = std::max({mask, mask_workspace_bytes(L.n[c], L.m, MASK_PASSES, true),
                     mask_workspace_bytes(L.n[c], L.m, MASK_PASSES, false),
                     mask_workspace_bytes(g, L.n[c], MASK_PASSES, false)});
  s = std::max(s, std::min(mask, MASK_SCRATCH_CAP) + 4096);   // larger masks run in batches of vectors
  s = std::max(s, dgemm_workspace_bytes(ctx, (int)g, 1, (long)L.m));
  return s + (64u << 20);
}

// client.cpp:543-568 (masks), 627-679 (repartition into column slabs, local
// QR of slabs wider than global_n), 805-954 (Ralha, bidiagonal order
// global_n), 963-995 (bidiagonal SVD), 1002-1105 (FinalU, k x m), 1023-1048
// and 1136-1160 (svd_mode 4), 1119-1169 (FinalVT_c from rows of U2).
bbt_status fedsvd_tall(bbt_ctx* ctx, const bbt_fedsvd_config* cfg, const Layout& L, double* const* X,
                       double* sigma, double* Uout, double* const* VT, int* kout) {
  const int P = L.P, mode = cfg->svd_mode;
  const size_t m = L.m, g = L.gn, wn = L.wn;
  const int gi = (int)g;
  const Layout Q = slab_layout(L);
  QrPlan qp;
  int streams = 1;
  {
    int nqr = 0;
    for (int c = 0; c < P; ++c) nqr += Q.qr[c];
    std::vector<size_t> skey = {L.m, (size_t)L.precision};
    for (int c = 0; c < P; ++c) skey.push_back(L.n[c]);
    if (ctx->tuned_streams > 0 && ctx->tuned_key == skey) {
      streams = ctx->tuned_streams;
      qp.nb = ctx->tuned_nb;
    } else if (nqr >= 8) {
      streams = 8;
    }
  }
  const size_t need = tall_persistent_bytes(L, Q, mode) +
                      std::max(tall_scratch_bytes(ctx, L, Q), batched_scratch(ctx, Q, streams, qp) + (64u << 20));
  if (ctx->ws.cap < need) BBT_CUDA(ctx, ctx->ws.reserve(need));
  ctx->ws.reset();
  const size_t tq = ((g + qp.nb - 1) / qp.nb) * qp.nb * qp.nb;
  std::vector<double*> slab(P, nullptr), RT(P, nullptr), tauc(P, nullptr), Tc(P, nullptr);
  QrJob job;
  job.precision = L.precision;
  for (int c = 0; c < P; ++c)
    if (Q.qr[c]) {
      slab[c] = ctx->ws.take<double>(g * L.part[c]);
      RT[c] = ctx->ws.take<double>(g * g);
      tauc[c] = ctx->ws.take<double>(g);
      Tc[c] = ctx->ws.take<double>(tq);
    }
  double* W = ctx->ws.take<double>(g * wn);
  double* Vr = ctx->ws.take<double>(g * wn);
  double* house = ctx->ws.take<double>(g * g);
  double* Ub = ctx->ws.take<double>(g * g);
  double* Vb = ctx->ws.take<double>(g * g);
  double* tmp = ctx->ws.take<double>(g * g);
  double* Z = ctx->ws.take<double>(g * g);
  double* tauh = ctx->ws.take<double>(g);
  double* alpha = ctx->ws.take<double>(g);
  double* beta = ctx->ws.take<double>(g);
  double* cs = ctx->ws.take<double>(2 * g);
  double* scal = ctx->ws.take<double>(8);
  int* cnt = ctx->ws.take<int>(8);
  if (!cnt) return fail(ctx, BBT_ERR_NOMEM, "fedsvd: workspace");
  job.RT = RT;
  job.tau = tauc;
  job.T = Tc;
  void* S = nullptr;
  if (L.precision == 1) {
    job.W.assign(P, nullptr);
    for (int c = 0; c < P; ++c)
      if (Q.qr[c]) job.W[c] = ctx->ws.take<double>(g * g);
    S = ctx->ws.take<char>((size_t)sketch_rows(gi) * sketch_pitch((long)Q.nmax) * 2);
    if (!S) return fail(ctx, BBT_ERR_NOMEM, "fedsvd: workspace (mixed precision)");
    job.S = S;
    job.spitch = sketch_pitch((long)Q.nmax);
  }
  double *Ulr = nullptr, *ym = nullptr, *sut = nullptr, *wfull = nullptr;
  if (mode == 4) {
    Ulr = ctx->ws.take<double>(m * g);
    ym = ctx->ws.take<double>(m);
    sut = ctx->ws.take<double>(g);
    wfull = ctx->ws.take<double>(g);
    if (!wfull) return fail(ctx, BBT_ERR_NOMEM, "fedsvd: workspace (linear regression)");
  }
  const bool compute_u = mode != 3, compute_v = mode != 2;   // client.cpp:491-492
  job.compute_v = compute_u;   // the slab's Q enters FinalU (u_reduction_tall_and_skinny, :664-666)

  cudaEvent_t ev[7];
  for (auto& e : ev) BBT_CUDA(ctx, cudaEventCreate(&e));
  struct EvGuard {
    cudaEvent_t* e;
    ~EvGuard() { for (int i = 0; i < 7; ++i) cudaEventDestroy(e[i]); }
  } guard{ev};
  PhaseRanges phases;
  BBT_CUDA(ctx, cudaEventRecord(ev[0], ctx->stream));
  phases.next("apply_mask");
  // 1) masks: private on the left (rows of X_c^T), public on the right (:548-551)
  for (int c = 0; c < P; ++c) {
    if (ctx->io_on) BBT_TRY(wait_input(ctx, c));
    BBT_TRY(block_shift_mask(ctx, L.n[c], m, MASK_PASSES, X[c], true, true, cfg->private_seeds[c]));
    BBT_TRY(block_shift_mask(ctx, L.n[c], m, MASK_PASSES, X[c], true, false, cfg->public_seed));
  }
  BBT_CUDA(ctx, cudaEventRecord(ev[1], ctx->stream));
  phases.next("global_qr");
  // 2) repartition (:627-659): slab c = rows n_pos.. of every masked block,
  //    columns m_part_pos[c].., global_n x m_part[c]; a slab that is not
  //    reduced goes straight into its columns of the Ralha matrix
  for (int c = 0; c < P; ++c) {
    double* dst = Q.qr[c] ? slab[c] : W + L.wpos[c];
    const long ldd = Q.qr[c] ? (long)L.part[c] : (long)wn;
    for (int d = 0; d < P; ++d)
      BBT_TRY(copy2d(ctx, (int)L.n[d], (int)L.part[c], X[d] + L.ppos[c], (long)m, dst + L.npos[d] * ldd, ldd));
  }
  BBT_CUDA(ctx, cudaEventRecord(ev[2], ctx->stream));
  phases.next("local_qr");
  // 3) local QR of the slabs with m_part > global_n (:661-677): R^T replaces the slab
  if (L.precision == 1) {
    BBT_TRY(rademacher(ctx, sketch_rows(gi), (long)Q.nmax, S, 0x5EED5EEDull));
    BBT_TRY(clear_tc_flags(ctx));
  }
  {
    const size_t mark = ctx->ws.top;
    const bool io = ctx->io_on;
    ctx->io_on = false;   // every block has been waited for above
    bbt_status st = local_qr_stage(ctx, Q, slab.data(), job, streams, qp, true);
    ctx->io_on = io;
    BBT_TRY(st);
    ctx->ws.top = mark;
  }
  if (L.precision == 1) BBT_TRY(check_tc_flags(ctx, "fedsvd: mixed-precision slab QR"));
  for (int c = 0; c < P; ++c)
    if (Q.qr[c]) BBT_TRY(copy2d(ctx, gi, gi, RT[c], (long)g, W + L.wpos[c], (long)wn));
  BBT_CUDA(ctx, cudaEventRecord(ev[3], ctx->stream));
  phases.next("bi_diag");
  // 4) Ralha of the global_n x wn matrix (:805-954)
  BBT_TRY(ralha(ctx, gi, (int)wn, W, house, tauh, alpha, beta, Vr, cs));
  BBT_CUDA(ctx, cudaEventRecord(ev[4], ctx->stream));
  phases.next("bsvd");
  // 5) singular values / vectors (:963-995); svd_mode 4 takes dbdsdc's path as mode 0
  BBT_TRY(bidiag_bound(ctx, gi, alpha, beta, scal));
  BBT_CUDA(ctx, cudaMemsetAsync(scal + 1, 0, sizeof(double), ctx->stream));
  BBT_TRY(sturm_counts(ctx, gi, alpha, beta, scal, 2, cnt));
  int hc[2];
  BBT_CUDA(ctx, cudaMemcpyAsync(hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, ctx->stream));
  BBT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  int k = hc[0] - hc[1];
  if (cfg->top_k > 0) k = std::min(k, cfg->top_k);
  if (k < 1) return fail(ctx, BBT_ERR_COUNT, "fedsvd: no singular values in (0, bound]");
  int ncl = 0;   // dbdsdc (modes 0, 4) keeps the vectors of tight clusters orthogonal: refine_clusters
  if ((mode == 0 || mode == 4) && k < gi) {
    BBT_TRY(bidiag_svd(ctx, k, alpha, beta, tmp, W, sigma, k, true));   // leading k x k (W is free)
    BBT_TRY(refine_clusters(ctx, k, k, alpha, beta, sigma, tmp, W, &ncl));
    embed_leading<<<4 * ctx->num_sms, 256, 0, ctx->stream>>>(gi, k, tmp, W, Ub, Vb);
    BBT_LAUNCHED(ctx);
  } else {
    BBT_TRY(bidiag_svd(ctx, gi, alpha, beta, Ub, Vb, sigma, k, true));   // Ub g x k, Vb k x g
    if (mode == 0 || mode == 4) BBT_TRY(refine_clusters(ctx, gi, k, alpha, beta, sigma, Ub, Vb, &ncl));
  }
  BBT_CUDA(ctx, cudaEventRecord(ev[5], ctx->stream));
  phases.next("combine_svd_remove_mask");
  // 6) U (:1002-1015): part_c = V_b Vr_c (Q_c^T), k x m_part[c], at columns
  //    m_part_pos[c] of FinalU (k x m row-major = column-major m x k)
  if (compute_u) {
    double* U = mode == 4 ? Ulr : Uout;
    for (int c = 0; c < P; ++c) {
      const int pc = (int)L.part[c];
      double* dst = U + L.ppos[c];
      if (!Q.qr[c]) {   // column-major part_c^T = Vr_c^T V_b^T
        BBT_TRY(dgemm(ctx, false, false, pc, k, g, 1.0, Vr + L.wpos[c], (long)wn, Vb, (long)g, 0.0, dst, (long)m));
        continue;
      }
      BBT_TRY(dgemm(ctx, false, false, gi, k, g, 1.0, Vr + L.wpos[c], (long)wn, Vb, (long)g, 0.0, tmp, (long)g));
      if (L.precision == 1) {   // Q_c = Q_p W_c: part_c^T = Q_p (W_c tmp)
        BBT_TRY(dgemm(ctx, false, false, gi, k, g, 1.0, job.W[c], (long)g, tmp, (long)g, 0.0, Z, (long)g));
        if (oz_worthwhile(pc, k, (long)g))
          BBT_TRY(gemm_oz(ctx, pc, k, (long)g, 1.0, slab[c], 1, pc, Z, (long)g, 1, 0.0, dst, (long)m, false, false, 6));
        else
          BBT_TRY(dgemm(ctx, false, false, pc, k, g, 1.0, slab[c], pc, Z, (long)g, 0.0, dst, (long)m));
      } else {
        BBT_TRY(dgemm(ctx, false, false, pc, k, g, 1.0, slab[c], pc, tmp, (long)g, 0.0, dst, (long)m));
      }
    }
    if (mode == 4) {   // Sigma^-1 U^T y with the public mask on y (:1026-1045)
      BBT_CUDA(ctx, cudaMemcpyAsync(ym, cfg->labels, m * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
      BBT_TRY(block_shift_mask(ctx, 1, m, MASK_PASSES, ym, true, false, cfg->public_seed));
      BBT_TRY(dgemm(ctx, true, false, k, 1, (long)m, 1.0, Ulr, (long)m, ym, (long)m, 0.0, sut, k));
      div_sigma<<<(k + 127) / 128, 128, 0, ctx->stream>>>(k, sigma, sut);
      BBT_LAUNCHED(ctx);
    } else {   // the public unmask of FinalU (:1098-1105)
      BBT_TRY(block_shift_mask(ctx, (size_t)k, m, MASK_PASSES, Uout, false, false, cfg->public_seed));
    }
  }
  // 7) V (:1119-1169): U2 = H (G^T U_b), global_n x k; participant c owns rows n_pos[c]..
  if (compute_v) {
    rot_sweep<<<(k + 127) / 128, 128, 0, ctx->stream>>>(gi, k, cs, Ub);
    BBT_LAUNCHED(ctx);
    BBT_TRY(ormqr_left_notrans(ctx, (long)g, gi, house, (long)g, 1, tauh, Ub, k, k, true, qp));
    if (mode == 4)   // w = U2 Sigma^-1 U^T y (:1140)
      BBT_TRY(dgemm(ctx, true, false, gi, 1, k, 1.0, Ub, k, sut, k, 0.0, wfull, (long)g));
    for (int c = 0; c < P; ++c) {
      const int nc = (int)L.n[c];
      size_t bytes;
      if (mode == 4) {   // w_c, unmasked with the private seed (:1141-1153)
        BBT_CUDA(ctx, cudaMemcpyAsync(VT[c], wfull + L.npos[c], nc * sizeof(double), cudaMemcpyDeviceToDevice,
                                      ctx->stream));
        BBT_TRY(block_shift_mask(ctx, 1, (size_t)nc, MASK_PASSES, VT[c], false, false, cfg->private_seeds[c]));
        bytes = (size_t)nc * sizeof(double);
      } else {           // FinalVT_c = U2[rows of c]^T, unmasked (:1161-1166)
        BBT_TRY(transpose(ctx, nc, k, Ub + L.npos[c] * k, k, VT[c], nc));
        BBT_TRY(block_shift_mask(ctx, (size_t)k, (size_t)nc, MASK_PASSES, VT[c], false, false,
                                 cfg->private_seeds[c]));
        bytes = (size_t)k * nc * sizeof(double);
      }
      if (ctx->io_on && ctx->vt_dst[c]) {
        BBT_CUDA(ctx, cudaEventRecord(ctx->vt_done[c], ctx->stream));
        BBT_CUDA(ctx, cudaStreamWaitEvent(ctx->copy_out, ctx->vt_done[c], 0));
        BBT_CUDA(ctx, cudaMemcpyAsync(ctx->vt_dst[c], VT[c], bytes, cudaMemcpyDeviceToHost, ctx->copy_out));
      }
    }
  }
  BBT_CUDA(ctx, cudaEventRecord(ev[6], ctx->stream));
  phases.close();
  BBT_CUDA(ctx, cudaEventSynchronize(ev[6]));
  if (L.precision >= 1) BBT_TRY(check_tc_flags(ctx, "fedsvd: tensor-core back-transform"));
  // stage order of the reference's timers: local_qr, apply_mask, global_qr
  // (here the repartition gather; this branch has no global QR), bi_diag,
  // bsvd, combine_svd_remove_mask
  const int from[6] = {2, 0, 1, 3, 4, 5}, to[6] = {3, 1, 2, 4, 5, 6};
  for (int s = 0; s < 6; ++s) {
    float ms = 0;
    BBT_CUDA(ctx, cudaEventElapsedTime(&ms, ev[from[s]], ev[to[s]]));
    ctx->stage_ms[s] = ms;
  }
  *kout = k;
  return BBT_OK;
}

}  // namespace

size_t fedsvd_workspace_bytes(const bbt_fedsvd_config* cfg) {
  Layout L;
  bbt_ctx dummy;
  if (plan(&dummy, cfg, L) != BBT_OK) return 0;
  dummy.num_sms = 148;
  if (L.tall) {
    const Layout Q = slab_layout(L);
    return tall_persistent_bytes(L, Q, cfg->svd_mode) + tall_scratch_bytes(&dummy, L, Q);
  }
  return persistent_bytes(L) + scratch_bytes(&dummy, L);
}

bbt_status fedsvd(bbt_ctx* ctx, const bbt_fedsvd_config* cfg, double* const* X, double* sigma,
                  double* Uout, double* const* VT, int* kout) {
  Layout L;
  BBT_TRY(plan(ctx, cfg, L));
  if (L.tall) return fedsvd_tall(ctx, cfg, L, X, sigma, Uout, VT, kout);
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
  const bool compute_u = cfg->svd_mode != 3, compute_v = cfg->svd_mode != 2;   // client.cpp:491-492
  MaskPrefetch pf;
  for (int c = 0; c < P; ++c) {
    pf.add(m, true, cfg->public_seed);                  // row mask, client.cpp:594
    pf.add(L.r[c], true, cfg->private_seeds[c]);        // column mask, :595
    if (compute_v) pf.add(L.r[c], false, cfg->private_seeds[c]);   // its inverse on FinalVT_c, :1182
  }
  if (compute_u) pf.add(m, false, cfg->public_seed);    // the row mask's inverse on FinalU, :1109
  const size_t need = persistent_bytes(L) + pf.bytes() +
                      std::max(scratch_bytes(ctx, L), batched_scratch(ctx, L, streams, qp) + (64u << 20));
  // precision 2: X_int's residue planes serve the Gram and, kept, the V back-transform
  // (no second pass over the blocks), where the device has room for them
  size_t keep = 0;
  if (L.precision == 2 && cfg->svd_mode != 2) {
    for (int c = 0; c < P; ++c)
      if (L.qr[c]) keep += exact_keep_bytes(mi, (long)L.n[c]);
    size_t free_b = 0, total_b = 0;   // a larger arena replaces the current one: its bytes come back
    if (ctx->ws.cap < need + keep &&
        (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess || need + keep + ((size_t)4 << 30) > free_b + ctx->ws.cap))
      keep = 0;
  }
  if (ctx->ws.cap < need + keep) BBT_CUDA(ctx, ctx->ws.reserve(need + keep));
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
  char* mask_slab = ctx->ws.take<char>(pf.bytes());
  if (!tmp || !mask_slab) return fail(ctx, BBT_ERR_NOMEM, "fedsvd: workspace");
  pf.start();   // the mask tables are drawn on the host while the GPU runs the local QRs
  QrJob job;
  job.precision = L.precision;
  job.RT = RT;
  job.tau = tauc;
  job.T = Tc;
  double *Z = nullptr, *Wg = nullptr, *Rg = nullptr, *Rpg = nullptr, *scg = nullptr;
  void* S = nullptr;
  const long sk_cols = (long)std::max(L.nmax, L.rg);   // the sketch serves the local and the global QR
  if (L.precision >= 1) {
    for (int c = 0; c < P; ++c) job.W.push_back(ctx->ws.take<double>(m * m));
    Z = ctx->ws.take<double>(m * m);
    Wg = ctx->ws.take<double>(m * m);
    Rg = ctx->ws.take<double>(m * m);
    S = ctx->ws.take<char>((size_t)sketch_rows(mi) * sketch_pitch(sk_cols) * 2);
    if (!S) return fail(ctx, BBT_ERR_NOMEM, "fedsvd: workspace (mixed precision)");
    job.S = S;
    job.spitch = sketch_pitch(sk_cols);
  }
  if (L.precision == 2) {
    for (int c = 0; c < P; ++c) {
      job.Rp.push_back(ctx->ws.take<double>(m * m));
      job.scale.push_back(ctx->ws.take<double>(m));
    }
    Rpg = ctx->ws.take<double>(m * m);
    scg = ctx->ws.take<double>(m);
    if (!scg) return fail(ctx, BBT_ERR_NOMEM, "fedsvd: workspace (exact Gram)");
    if (keep) {
      job.planes.assign(P, nullptr);
      for (int c = 0; c < P; ++c)
        if (L.qr[c]) {
          job.planes[c] = ctx->ws.take<int8_t>(exact_keep_bytes(mi, (long)L.n[c]));
          if (!job.planes[c]) return fail(ctx, BBT_ERR_NOMEM, "fedsvd: workspace (residue planes)");
        }
    }
  }

  cudaEvent_t ev[7];
  for (auto& e : ev) BBT_CUDA(ctx, cudaEventCreate(&e));
  struct EvGuard {
    cudaEvent_t* e;
    ~EvGuard() { for (int i = 0; i < 7; ++i) cudaEventDestroy(e[i]); }
  } guard{ev};
  PhaseRanges phases;
  BBT_CUDA(ctx, cudaEventRecord(ev[0], ctx->stream));
  phases.next("local_qr");

  // 1) local QR (client.cpp:572-589): A = X_c^T column-major n x m, in place
  job.compute_v = compute_v;
  std::vector<double*> masked(P);
  for (int c = 0; c < P; ++c) masked[c] = L.qr[c] ? RT[c] : X[c];
  if (L.precision >= 1) {
    BBT_TRY(rademacher(ctx, sketch_rows(mi), sk_cols, S, 0x5EED5EEDull));
    BBT_TRY(clear_tc_flags(ctx));
  }
  {
    const size_t mark = ctx->ws.top;
    BBT_TRY(local_qr_stage(ctx, L, X, job, streams, qp, true));
    ctx->ws.top = mark;
  }
  if (L.precision >= 1) BBT_TRY(check_tc_flags(ctx, "fedsvd: mixed-precision local QR"));
  if (ctx->io_on)
    for (int c = 0; c < P; ++c) BBT_TRY(wait_input(ctx, c));
  BBT_CUDA(ctx, cudaEventRecord(ev[1], ctx->stream));
  phases.next("apply_mask");
  // 2) masks (client.cpp:593-596)
  BBT_TRY(pf.upload(ctx, mask_slab));
  for (int c = 0; c < P; ++c) {
    BBT_TRY(apply_mask(ctx, pf, m, L.r[c], masked[c], true, true, cfg->public_seed));
    BBT_TRY(apply_mask(ctx, pf, m, L.r[c], masked[c], true, false, cfg->private_seeds[c]));
  }
  BBT_CUDA(ctx, cudaEventRecord(ev[2], ctx->stream));
  phases.next("global_qr");
  // 3) repartition + global QR of M^T (client.cpp:681-794)
  for (int c = 0; c < P; ++c)
    BBT_TRY(copy2d(ctx, mi, (int)L.r[c], masked[c], (long)L.r[c], M + L.rpos[c], (long)rg));
  if (rg == m) {   // m == global_n: no global QR, Ralha takes M^T (the in-place transpose, client.cpp:795-798)
    BBT_TRY(transpose(ctx, mi, mi, M, (long)rg, W, (long)m));
  } else if (L.precision == 2) {   // M kept, Q_g = M_int^T Rp_g^-1 W_g (exactqr.cu)
    const size_t mark = ctx->ws.top;
    BBT_TRY(exact_local_qr(ctx, mi, (long)rg, M, S, job.spitch, Rg, Wg, Rpg, scg));
    ctx->ws.top = mark;
    BBT_TRY(transpose(ctx, mi, mi, Rg, (long)m, W, (long)m));   // W (row-major) = R_g
    BBT_TRY(check_tc_flags(ctx, "fedsvd: exact-Gram global QR"));
  } else if (L.precision == 1) {   // M <- Q_p, Q_g = Q_p W_g, R_g with dgeqrf's signs (mixedqr.cu)
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
  phases.next("bi_diag");
  // 4) Ralha bidiagonalisation, lower -> upper (client.cpp:801-954)
  BBT_TRY(ralha(ctx, mi, mi, W, house, tauh, alpha, beta, Vr, cs));
  BBT_CUDA(ctx, cudaEventRecord(ev[4], ctx->stream));
  phases.next("bsvd");
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
  // dbdsdc (mode 0) keeps the vectors of tight clusters orthogonal where the
  // twisted vectors collapse onto each other: refine_clusters after bidiag_svd
  int ncl = 0;
  if (cfg->svd_mode == 0 && k < mi) {
    // dbdsdc on the leading k x k bidiagonal (client.cpp:975-980)
    double* Us = tmp;   // k x k each; the Ralha input W is free by now
    double* Vs = W;
    BBT_TRY(bidiag_svd(ctx, k, alpha, beta, Us, Vs, sigma, k, true));
    BBT_TRY(refine_clusters(ctx, k, k, alpha, beta, sigma, Us, Vs, &ncl));
    embed_leading<<<4 * ctx->num_sms, 256, 0, ctx->stream>>>(mi, k, Us, Vs, Ub, Vb);
    BBT_LAUNCHED(ctx);
  } else {
    BBT_TRY(bidiag_svd(ctx, mi, alpha, beta, Ub, Vb, sigma, k, true));   // Ub m x k, Vb k x m
    if (cfg->svd_mode == 0) BBT_TRY(refine_clusters(ctx, mi, k, alpha, beta, sigma, Ub, Vb, &ncl));
  }
  BBT_CUDA(ctx, cudaEventRecord(ev[5], ctx->stream));
  phases.next("combine_svd_remove_mask");
  // 6) U: FinalU (m x k row-major) = (V_b Vr)^T, unmasked (client.cpp:1018, 1071-1115)
  if (compute_u) {
    BBT_TRY(dgemm(ctx, true, true, k, mi, m, 1.0, Vb, (long)m, Vr, (long)m, 0.0, Uout, k));
    BBT_TRY(apply_mask(ctx, pf, m, (size_t)k, Uout, false, true, cfg->public_seed));
  }
  //    V: U2 = H (G^T U_b) (client.cpp:1127-1176)
  if (compute_v) {
  rot_sweep<<<(k + 127) / 128, 128, 0, ctx->stream>>>(mi, k, cs, Ub);
  BBT_LAUNCHED(ctx);
  BBT_TRY(ormqr_left_notrans(ctx, (long)m, mi, house, (long)m, 1, tauh, Ub, k, k, true, qp));
  if (L.precision >= 1)   // Q_g U2 = Q_p (W_g U2): Rg (free by now) <- W_g U2, m x k column-major
    BBT_TRY(dgemm(ctx, false, true, mi, k, m, 1.0, Wg, (long)m, Ub, k, 0.0, Rg, (long)m));
  ExactOperand zg;   // precision 2: Rp_g^-1 (W_g U2) as residue planes, shared by every participant
  if (L.precision == 2 && rg > m) BBT_TRY(exact_operand(ctx, mi, scg, Rpg, Rg, k, zg));
  for (int c = 0; c < P; ++c) {   // :1179-1195
    const int rc = (int)L.r[c];
    if (rg == m) {   // m == global_n: FinalVT_c = U2[rows of c]^T, unmasked (client.cpp:1161-1166)
      BBT_TRY(transpose(ctx, rc, k, Ub + L.rpos[c] * k, k, VT[c], rc));
      BBT_TRY(apply_mask(ctx, pf, (size_t)k, (size_t)rc, VT[c], false, false, cfg->private_seeds[c]));
      if (ctx->io_on && ctx->vt_dst[c]) {
        BBT_CUDA(ctx, cudaEventRecord(ctx->vt_done[c], ctx->stream));
        BBT_CUDA(ctx, cudaStreamWaitEvent(ctx->copy_out, ctx->vt_done[c], 0));
        BBT_CUDA(ctx, cudaMemcpyAsync(ctx->vt_dst[c], VT[c], (size_t)k * rc * sizeof(double), cudaMemcpyDeviceToHost,
                                      ctx->copy_out));
      }
      continue;
    }
    // tmp (k x r_c row-major) = U2^T Q_g[rows_c, :]^T  ==  column-major r_c x k = Q_g[rows_c,:] U2
    if (L.precision == 2) {   // Q_g[rows_c,:] U2 = M_int^T[rows_c] Rp_g^-1 (W_g U2), exactly (exactqr.cu)
      BBT_TRY(exact_apply_rows(ctx, zg, rc, M + L.rpos[c], (long)rg, scg, tmp, rc));
    } else if (L.precision == 1)
      BBT_TRY(dgemm(ctx, false, false, rc, k, m, 1.0, M + L.rpos[c], (long)rg, Rg, (long)m, 0.0, tmp, rc));
    else
      BBT_TRY(dgemm(ctx, false, true, rc, k, m, 1.0, M + L.rpos[c], (long)rg, Ub, k, 0.0, tmp, rc));
    BBT_TRY(apply_mask(ctx, pf, (size_t)k, (size_t)rc, tmp, false, false, cfg->private_seeds[c]));
    const long n = (long)L.n[c];
    bool vt_sent = false;   // FinalVT_c already copied out chunk by chunk
    if (L.qr[c] && L.precision == 2) {   // Q_c = X_int^T Rp_c^-1 W_c: FinalVT^T = X_int^T Rp_c^-1 (W_c tmp^T)
      BBT_TRY(dgemm(ctx, false, false, mi, k, m, 1.0, job.W[c], (long)m, tmp, rc, 0.0, Z, (long)m));
      const size_t mark = ctx->ws.top;
      if (!job.planes.empty() && job.planes[c]) {   // from the planes the local QR kept
        ExactOperand op;
        BBT_TRY(exact_operand(ctx, mi, job.scale[c], job.Rp[c], Z, k, op));
        if (ctx->io_on && ctx->vt_dst[c]) {
          // host output: each chunk of rows leaves as soon as it is computed
          // (a 2D copy of its k row segments), eight chunks per participant
          double* dst = ctx->vt_dst[c];
          double* src = VT[c];
          const std::function<bbt_status(long, int)> out = [&](long r0, int R) -> bbt_status {
            cudaEvent_t ev;
            BBT_CUDA(ctx, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
            BBT_CUDA(ctx, cudaEventRecord(ev, ctx->stream));
            BBT_CUDA(ctx, cudaStreamWaitEvent(ctx->copy_out, ev, 0));
            BBT_CUDA(ctx, cudaEventDestroy(ev));
            BBT_CUDA(ctx, cudaMemcpy2DAsync(dst + r0, (size_t)n * sizeof(double), src + r0, (size_t)n * sizeof(double),
                                            (size_t)R * sizeof(double), (size_t)k, cudaMemcpyDeviceToHost,
                                            ctx->copy_out));
            return BBT_OK;
          };
          BBT_TRY(exact_apply_planes(ctx, op, n, job.planes[c], crt_pitch(n), VT[c], n, &out, (n + 7) / 8));
          vt_sent = true;
        } else {
          BBT_TRY(exact_apply_planes(ctx, op, n, job.planes[c], crt_pitch(n), VT[c], n));
        }
      } else {
        BBT_TRY(exact_apply_q(ctx, mi, n, X[c], n, job.scale[c], job.Rp[c], Z, k, VT[c], n));
      }
      ctx->ws.top = mark;
    } else if (L.qr[c] && L.precision == 1) {   // Q_c = Q_p W_c: FinalVT^T = Q_p (W_c tmp^T)
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
    if (ctx->io_on && ctx->vt_dst[c] && !vt_sent) {   // FinalVT_c leaves while the next participant is computed
      BBT_CUDA(ctx, cudaEventRecord(ctx->vt_done[c], ctx->stream));
      BBT_CUDA(ctx, cudaStreamWaitEvent(ctx->copy_out, ctx->vt_done[c], 0));
      BBT_CUDA(ctx, cudaMemcpyAsync(ctx->vt_dst[c], VT[c], (size_t)k * n * sizeof(double), cudaMemcpyDeviceToHost,
                                    ctx->copy_out));
    }
  }
  }
  BBT_CUDA(ctx, cudaEventRecord(ev[6], ctx->stream));
  phases.close();
  BBT_CUDA(ctx, cudaEventSynchronize(ev[6]));
  if (L.precision >= 1) BBT_TRY(check_tc_flags(ctx, "fedsvd: tensor-core back-transform"));
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
  bbt_fedsvd_config shape = *cfg;   // the QRs depend on the shapes only
  if (shape.svd_mode == 4) shape.svd_mode = 1;
  Layout L0;
  BBT_TRY(plan(ctx, &shape, L0));
  const Layout L = L0.tall ? slab_layout(L0) : L0;   // the QRs this configuration runs
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
  const std::vector<int> cand_nb = L.precision >= 1 ? std::vector<int>{128} : std::vector<int>{64, 128};
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
  if (L.precision >= 1) need += (size_t)P * (L.m * L.m * 8 + 256) + sbytes + 256;
  if (L.precision == 2) need += (size_t)P * ((L.m * L.m + L.m) * 8 + 512);
  if (ctx->ws.cap < need) BBT_CUDA(ctx, ctx->ws.reserve(need));
  ctx->ws.reset();
  QrJob job;
  job.precision = L.precision;
  job.compute_v = true;
  for (int c = 0; c < P; ++c) {
    job.RT.push_back(ctx->ws.take<double>(L.m * L.m));
    job.tau.push_back(ctx->ws.take<double>(L.m));
    job.T.push_back(ctx->ws.take<double>(tq));
    if (L.precision >= 1) job.W.push_back(ctx->ws.take<double>(L.m * L.m));
    if (L.precision == 2) {
      job.Rp.push_back(ctx->ws.take<double>(L.m * L.m));
      job.scale.push_back(ctx->ws.take<double>(L.m));
    }
  }
  if (L.precision >= 1) {
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
  ctx->tuned_key = {L0.m, (size_t)L0.precision};
  for (int c = 0; c < P; ++c) ctx->tuned_key.push_back(L0.n[c]);
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
  scratch = std::max(scratch, bisect_workspace_bytes(m, m) + 16 * (size_t)m) + (64u << 20);
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
