// Sturm counts and the reference's bisection tree on the GPU.
//
// Excalibur's negative_count (src/bbtsvd.cpp:7-17) is a stationary-qd
// Sturm count of B^T B - mu^2 I; bisection_singular_values (:19-52) walks a
// binary tree over [lo, hi] depth first, upper half first, and stops a
// branch when the midpoint no longer splits it (or the width is <= tol),
// emitting that midpoint.  Every value is therefore fixed by the tree, not
// by the traversal order, so the tree can be walked breadth first: all live
// intervals of a level in parallel.  Each round resolves DEPTH levels at
// once ("multisection"): the 2^DEPTH - 1 midpoints below a live interval are
// counted by separate threads, then one thread per interval replays the
// reference's rules over that subtree.  Intervals are kept in descending
// order, terminal ones included, so the final list is already the
// reference's output order and top_k is a truncation.
//
// Arithmetic: every product, quotient and sum is rounded on its own
// (__dmul_rn / __ddiv_rn / __dadd_rn: no FMA contraction), as in the
// reference's build, so counts and singular values match it bit for bit.
#include <cuda_runtime.h>

#include <algorithm>

#include "internal.h"

namespace bbt {
namespace {

constexpr int DEPTH = 5;                 // tree levels resolved per round
constexpr int NPTS = (1 << DEPTH) - 1;   // midpoints counted per live interval
constexpr int FAN = 1 << DEPTH;          // max intervals one interval becomes
constexpr int SMEM_PAIRS_MAX = 12288;    // stage (beta^2, alpha^2) in SMEM up to this n

// (b2[i-1], a2[i]) with b2[-1] unused; squares rounded once, as pow(x,2)
// folded to x*x in the reference's -O3 build.
__global__ void squares_kernel(int n, const double* __restrict__ a, const double* __restrict__ b,
                               double2* __restrict__ q) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    double ai = a[i];
    double bi = (i > 0) ? b[i - 1] : 0.0;
    q[i] = make_double2(__dmul_rn(bi, bi), __dmul_rn(ai, ai));
  }
}

// One Sturm count, q in SMEM or global.  Follows bbtsvd.cpp:9-15 exactly.
__device__ __forceinline__ int sturm(int n, const double2* q, double mu) {
  const double mu2 = __dmul_rn(mu, mu);
  double t = -mu2;
  double d = __dadd_rn(q[0].y, t);
  int neg = d < 0.0;
  for (int i = 1; i < n; ++i) {
    const double2 qi = q[i];
    const double r = __ddiv_rn(qi.x, d);
    t = __dsub_rn(__dmul_rn(t, r), mu2);
    d = __dadd_rn(qi.y, t);
    neg += d < 0.0;
  }
  return neg;
}

__device__ __forceinline__ void stage_pairs(int n, const double2* __restrict__ q, double2* sq) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) sq[i] = q[i];
  __syncthreads();
}

__global__ void counts_kernel(int n, const double2* __restrict__ q, const double* __restrict__ mu,
                              int nmu, int* __restrict__ out, int use_smem) {
  extern __shared__ double2 sq[];
  const double2* src = q;
  if (use_smem) { stage_pairs(n, q, sq); src = sq; }
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nmu; j += gridDim.x * blockDim.x)
    out[j] = sturm(n, src, mu[j]);
}

struct Node {
  double lo, hi;
  int clo, chi;
  int done;   // 1: terminal (value = lo), 0: live
  int pad;
};

__device__ __forceinline__ double midpoint(double lo, double hi) {
  return __dmul_rn(__dadd_rn(lo, hi), 0.5);   // (lo + hi) / 2, the sum rounded once
}

// Counts at the 2^DEPTH - 1 midpoints of the subtree under every live node.
__global__ void expand_kernel(int n, const double2* __restrict__ q, const Node* __restrict__ nodes,
                              int nnodes, int* __restrict__ cnt, int use_smem) {
  extern __shared__ double2 sq[];
  const double2* src = q;
  if (use_smem) { stage_pairs(n, q, sq); src = sq; }
  const long total = (long)nnodes * NPTS;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total;
       t += (long)gridDim.x * blockDim.x) {
    const int u = (int)(t / NPTS);
    const int h = (int)(t % NPTS) + 1;       // heap index in the subtree
    const Node nd = nodes[u];
    if (nd.done) continue;
    double lo = nd.lo, hi = nd.hi;
    const int depth = 31 - __clz(h);
    for (int bit = depth - 1; bit >= 0; --bit) {
      const double mid = midpoint(lo, hi);
      if ((h >> bit) & 1) lo = mid; else hi = mid;
    }
    cnt[(long)u * NPTS + h - 1] = sturm(n, src, midpoint(lo, hi));
  }
}

// One thread per node: replay the reference's pop/emit/push rules over the
// node's subtree (upper child first) and write the resulting intervals in
// descending order.
__global__ void resolve_kernel(const Node* __restrict__ nodes, int nnodes, const int* __restrict__ cnt,
                               double tol, Node* __restrict__ out, int* __restrict__ nout) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= nnodes) return;
  Node nd = nodes[u];
  Node* o = out + (long)u * FAN;
  if (nd.done) { o[0] = nd; nout[u] = 1; return; }
  struct Item { double lo, hi; int clo, chi, h; };
  Item st[DEPTH + 2];
  int sp = 0, k = 0;
  st[sp++] = {nd.lo, nd.hi, nd.clo, nd.chi, 1};
  while (sp > 0) {
    const Item it = st[--sp];
    const double mid = midpoint(it.lo, it.hi);
    if (__dsub_rn(it.hi, it.lo) <= tol || mid == it.lo || mid == it.hi) {
      o[k++] = {mid, mid, it.clo, it.chi, 1, 0};
      continue;
    }
    if (it.h > NPTS) {                        // below this round's subtree: live next round
      o[k++] = {it.lo, it.hi, it.clo, it.chi, 0, 0};
      continue;
    }
    const int cm = cnt[(long)u * NPTS + it.h - 1];
    if (cm > it.clo) st[sp++] = {it.lo, mid, it.clo, cm, 2 * it.h};       // lower, popped last
    if (it.chi > cm) st[sp++] = {mid, it.hi, cm, it.chi, 2 * it.h + 1};   // upper, popped first
  }
  nout[u] = k;
}

// Single block: exclusive scan of nout, scatter into the next node list
// (truncated to top_k), report (count, live count).
__global__ void compact_kernel(const Node* __restrict__ cand, const int* __restrict__ nout, int nnodes,
                               int top_k, Node* __restrict__ next, int* __restrict__ stats) {
  __shared__ int warp_sums[32];
  __shared__ int carry;
  __shared__ int live_total;
  if (threadIdx.x == 0) { carry = 0; live_total = 0; }
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int base = 0; base < nnodes; base += blockDim.x) {
    const int u = base + threadIdx.x;
    const int v = (u < nnodes) ? nout[u] : 0;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    if (wid == 0) {
      int w = (lane < nw) ? warp_sums[lane] : 0;
      for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      if (lane < nw) warp_sums[lane] = w;
    }
    __syncthreads();
    const int excl = carry + (wid > 0 ? warp_sums[wid - 1] : 0) + x - v;
    int live = 0;
    for (int j = 0; j < v; ++j) {
      const int dst = excl + j;
      if (dst < top_k) {
        const Node c = cand[(long)u * FAN + j];
        next[dst] = c;
        live += !c.done;
      }
    }
    if (live) atomicAdd(&live_total, live);
    __syncthreads();
    if (threadIdx.x == 0) carry += warp_sums[nw - 1];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    stats[0] = carry < top_k ? carry : top_k;
    stats[1] = live_total;
  }
}

__global__ void emit_kernel(const Node* __restrict__ nodes, int n, double* __restrict__ sigma) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) sigma[i] = nodes[i].lo;
}

__global__ void root_kernel(double lo, double hi, const int* __restrict__ c, Node* nodes) {
  nodes[0] = {lo, hi, c[0], c[1], 0, 0};
}

int smem_bytes(int n) { return n <= SMEM_PAIRS_MAX ? n * (int)sizeof(double2) : 0; }

// ---- learned brackets (proposed by the MLP of mlp.cu) ----------------------
// Each bracket [L, U] of the j-th largest value is snapped to the deepest node
// of the reference's tree that contains it: descend from the root by the same
// midpoint arithmetic as resolve_kernel, stopping at a terminal node or where
// the bracket straddles the midpoint.  Entry t of the table belongs to the
// value of ascending rank rbase + t, i.e. j = chi_root - 1 - (rbase + t);
// pad = 1 marks a candidate, 0 one that can no longer help, -1 one rejected.
__global__ void snap_kernel(int count, const double* __restrict__ br, double rlo, double rhi, double tol, int cb,
                            int rbase, Node* __restrict__ table) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= count) return;
  const double L = br[2 * j], U = br[2 * j + 1];
  double lo = rlo, hi = rhi;
  for (int d = 0; d < 4096; ++d) {
    const double mid = midpoint(lo, hi);
    if (__dsub_rn(hi, lo) <= tol || mid == lo || mid == hi) break;
    if (U < mid) hi = mid;
    else if (L >= mid) lo = mid;
    else break;
  }
  table[(cb - 1 - j) - rbase] = {lo, hi, 0, 0, 0, (L <= U) ? 1 : 0};
}

// A live interval holding one value and strictly containing that value's
// snapped node is checked against that node by two exact Sturm counts (lazily: only
// when such a jump is possible).  With the same count range, every level in
// between holds exactly the same values, so the reference's walk through
// them ends in that node: the interval becomes the node.  Otherwise the
// entry is rejected and plain bisection goes on.
__global__ void jump_kernel(int n, const double2* __restrict__ q, Node* __restrict__ nodes, int N,
                            Node* __restrict__ table, int tcount, int rbase, int* __restrict__ stat) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= N) return;
  const Node nd = nodes[u];
  if (nd.done || nd.chi - nd.clo != 1) return;   // single-value intervals only
  const int t = nd.clo - rbase;
  if (t < 0 || t >= tcount) return;
  const Node tb = table[t];
  if (tb.pad != 1) return;
  if (!(tb.lo >= nd.lo && tb.hi <= nd.hi)) return;
  if (!(__dsub_rn(tb.hi, tb.lo) < __dsub_rn(nd.hi, nd.lo))) {   // not deeper (yet): try again next round
    return;
  }
  const int clo = sturm(n, q, tb.lo), chi = sturm(n, q, tb.hi);
  atomicAdd(stat, 2);
  if (clo == nd.clo && chi == nd.chi) {
    nodes[u].lo = tb.lo;
    nodes[u].hi = tb.hi;
    atomicAdd(stat + 1, 1);
  }
  table[t].pad = -1;   // used or rejected: never tried again
}

}  // namespace

bbt_status sturm_counts(bbt_ctx* ctx, int n, const double* a, const double* b, const double* mu,
                        int nmu, int* counts) {
  if (n < 1 || nmu < 0) return fail(ctx, BBT_ERR_ARG, "sturm_counts: n=%d nmu=%d", n, nmu);
  if (nmu == 0) return BBT_OK;
  size_t mark = ctx->ws.top;
  double2* q = ctx->ws.take<double2>(n);
  if (!q) return fail(ctx, BBT_ERR_NOMEM, "sturm_counts: workspace");
  squares_kernel<<<(n + 255) / 256, 256, 0, ctx->stream>>>(n, a, b, q);
  BBT_LAUNCHED(ctx);
  const int sm = smem_bytes(n);
  if (sm > 48 * 1024)
    BBT_CUDA(ctx, cudaFuncSetAttribute(counts_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  const int threads = 128;
  int blocks = (nmu + threads - 1) / threads;
  counts_kernel<<<blocks, threads, sm, ctx->stream>>>(n, q, mu, nmu, counts, sm > 0);
  BBT_LAUNCHED(ctx);
  ctx->ws.top = mark;
  return BBT_OK;
}

size_t bisect_workspace_bytes(int n, int top_k) {
  const size_t cap = (size_t)std::max(n, 0) + 2;
  const size_t tk = (size_t)std::max(top_k, 0);
  return 16 * cap + cap * (sizeof(Node) * (1 + FAN) + sizeof(int) * (1 + NPTS)) + tk * sizeof(Node) + 16 * 256 + 4096;
}

bbt_status bisect(bbt_ctx* ctx, int n, const double* a, const double* b, double lo, double hi,
                  double tol, int top_k, double* sigma, int* count, const double* brackets, long* stats_out) {
  *count = 0;
  if (stats_out) for (int i = 0; i < 4; ++i) stats_out[i] = 0;
  if (n < 1) return fail(ctx, BBT_ERR_ARG, "bisection: n=%d", n);
  if (top_k <= 0) return BBT_OK;
  size_t mark = ctx->ws.top;
  double2* q = ctx->ws.take<double2>(n);
  double* ends = ctx->ws.take<double>(2);
  int* c2 = ctx->ws.take<int>(2);
  const int cap = n + 2;                    // live + terminal intervals never exceed the count range
  Node* nodes = ctx->ws.take<Node>(cap);
  Node* cand = ctx->ws.take<Node>((size_t)cap * FAN);
  int* nout = ctx->ws.take<int>(cap);
  int* cnt = ctx->ws.take<int>((size_t)cap * NPTS);
  int* stats = ctx->ws.take<int>(4);
  if (!stats) return fail(ctx, BBT_ERR_NOMEM, "bisection: workspace");
  squares_kernel<<<(n + 255) / 256, 256, 0, ctx->stream>>>(n, a, b, q);
  BBT_LAUNCHED(ctx);
  const int sm = smem_bytes(n);
  if (sm > 48 * 1024) {
    BBT_CUDA(ctx, cudaFuncSetAttribute(counts_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    BBT_CUDA(ctx, cudaFuncSetAttribute(expand_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  }
  double hend[2] = {lo, hi};
  BBT_CUDA(ctx, cudaMemcpyAsync(ends, hend, sizeof(hend), cudaMemcpyHostToDevice, ctx->stream));
  counts_kernel<<<1, 32, sm, ctx->stream>>>(n, q, ends, 2, c2, sm > 0);
  BBT_LAUNCHED(ctx);
  int hc[2];
  BBT_CUDA(ctx, cudaMemcpyAsync(hc, c2, sizeof(hc), cudaMemcpyDeviceToHost, ctx->stream));
  BBT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (!(hc[0] <= hc[1])) { ctx->ws.top = mark; return BBT_OK; }   // bbtsvd.cpp:26
  root_kernel<<<1, 1, 0, ctx->stream>>>(lo, hi, c2, nodes);
  BBT_LAUNCHED(ctx);
  int N = 1, live = 1;
  const int limit = top_k < cap ? top_k : cap;
  ProfScope prof(ctx, BBT_PROF_BISECT, 0.0);
  long evals = 2;
  // learned brackets: snapped to the tree, verified lazily in jump_kernel
  Node* table = nullptr;
  int tcount = 0, rbase = 0;
  int* jstat = stats + 2;   // [Sturm evaluations of verification, jumps]
  BBT_CUDA(ctx, cudaMemsetAsync(stats, 0, 4 * sizeof(int), ctx->stream));
  if (brackets) {
    tcount = std::min(hc[1] - hc[0], limit);
    rbase = hc[1] - tcount;
    if (tcount > 0) {
      table = ctx->ws.take<Node>(tcount);
      if (!table) return fail(ctx, BBT_ERR_NOMEM, "bisection: bracket table");
      snap_kernel<<<(tcount + 127) / 128, 128, 0, ctx->stream>>>(tcount, brackets, lo, hi, tol, hc[1], rbase, table);
      BBT_LAUNCHED(ctx);
    }
  }
  for (int round = 0; live > 0; ++round) {
    if (round > 4096) return fail(ctx, BBT_ERR_TIMEOUT, "bisection: no convergence");
    if (table) {
      jump_kernel<<<(N + 127) / 128, 128, 0, ctx->stream>>>(n, q, nodes, N, table, tcount, rbase, jstat);
      BBT_LAUNCHED(ctx);
    }
    evals += (long)live * NPTS;
    const long work = (long)N * NPTS;
    int threads = 128;
    long blocks = (work + threads - 1) / threads;
    if (blocks > 65535) blocks = 65535;
    expand_kernel<<<(int)blocks, threads, sm, ctx->stream>>>(n, q, nodes, N, cnt, sm > 0);
    BBT_LAUNCHED(ctx);
    resolve_kernel<<<(N + 127) / 128, 128, 0, ctx->stream>>>(nodes, N, cnt, tol, cand, nout);
    BBT_LAUNCHED(ctx);
    compact_kernel<<<1, 1024, 0, ctx->stream>>>(cand, nout, N, limit, nodes, stats);
    BBT_LAUNCHED(ctx);
    int hs[2];
    BBT_CUDA(ctx, cudaMemcpyAsync(hs, stats, sizeof(hs), cudaMemcpyDeviceToHost, ctx->stream));
    BBT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    N = hs[0];
    live = hs[1];
    if (stats_out) stats_out[1] = round + 1;
  }
  if (N > 0) {
    emit_kernel<<<(N + 255) / 256, 256, 0, ctx->stream>>>(nodes, N, sigma);
    BBT_LAUNCHED(ctx);
  }
  if (stats_out) {   // [Sturm evaluations, rounds, jumps taken, verification evaluations]
    int hs[4];
    BBT_CUDA(ctx, cudaMemcpyAsync(hs, stats, sizeof(hs), cudaMemcpyDeviceToHost, ctx->stream));
    BBT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    stats_out[0] = evals + hs[2];
    stats_out[2] = hs[3];
    stats_out[3] = hs[2];
  }
  *count = N;
  ctx->ws.top = mark;
  return BBT_OK;
}

}  // namespace bbt
