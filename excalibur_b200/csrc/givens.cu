// Random Givens-rotation data masks (Excalibur src/bbtsvd.cpp:533-876).
//
// A mask is `passes` sweeps; each sweep rotates disjoint random pairs of
// one dimension of a row-major m x n block (rows when is_left, columns
// otherwise).  Every vector along the other dimension sees the same
// rotations, so a CTA stages a strip of w vectors in shared memory as a
// [k][w+1] tile (k = rotated length, +1 pad against bank conflicts), applies
// all sweeps there, and writes the strip back once: 16 bytes of HBM traffic
// per element for 6 * passes flops.  Within a sweep all pairs are disjoint
// except, for odd k, the pair with the extra partner; it is applied on its
// own, before or after the others exactly where the reference applies it.
//
// The random tables are drawn on the host with the reference's own calls
// (srand, std::default_random_engine, std::shuffle, rand), and the
// rotation rounds each product and each sum (no FMA) like the reference's
// AVX2 code, so the masked block equals the reference's bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <random>
#include <vector>

#include "internal.h"

namespace bbt {
namespace {

using Tables = GivensTables;

// bbtsvd.cpp:729-779.  Leaves glibc's rand() state exactly as the reference.
void draw_tables(size_t k, size_t passes, bool mask, unsigned seed, Tables& T) {
  srand(seed);
  std::default_random_engine eng(seed);
  T.k = k;
  T.passes = passes;
  T.ops = (k + (k & 1)) / 2;
  if (k <= 1) { T.ops = 0; return; }
  const size_t ops = T.ops;
  std::vector<std::vector<size_t>> perm(passes);
  for (size_t t = 0; t < passes; ++t) {
    std::vector<size_t> v(k);
    for (size_t j = 0; j < k; ++j) v[j] = j;
    std::shuffle(v.begin(), v.end(), eng);
    if (k & 1) {   // odd k: one extra partner drawn with rand()
      v.push_back(rand() % k);
      while (v[k] == v[k - 1]) v[k] = rand() % k;
    }
    if (!mask) std::reverse(v.begin(), v.end());
    for (size_t j = 0; j < 2 * ops; j += 2)
      if (v[j] > v[j + 1]) std::swap(v[j], v[j + 1]);
    perm[t].swap(v);
  }
  if (!mask) std::reverse(perm.begin(), perm.end());
  std::vector<std::vector<double>> c(passes), s(passes);
  for (size_t t = 0; t < passes; ++t) {
    c[t].resize(ops);
    s[t].resize(ops);
    for (size_t j = 0; j < ops; ++j) {
      c[t][j] = (rand() / (double)RAND_MAX) * 2.0 + -1.0;   // random_value(-1, 1)
      s[t][j] = (rand() / (double)RAND_MAX) * 2.0 + -1.0;
      const double r = pow(c[t][j] * c[t][j] + s[t][j] * s[t][j], 0.5);
      c[t][j] /= r;
      s[t][j] /= r;
    }
    if (!mask) {
      std::reverse(c[t].begin(), c[t].end());
      std::reverse(s[t].begin(), s[t].end());
    }
  }
  if (!mask) {
    std::reverse(c.begin(), c.end());
    std::reverse(s.begin(), s.end());
  }
  T.pairs.resize(passes * ops);
  T.cs.resize(passes * ops);
  const double sg = mask ? 1.0 : -1.0;
  for (size_t t = 0; t < passes; ++t)
    for (size_t j = 0; j < ops; ++j) {
      T.pairs[t * ops + j] = make_int2((int)perm[t][2 * j], (int)perm[t][2 * j + 1]);
      T.cs[t * ops + j] = make_double2(c[t][j], sg * s[t][j]);
    }
  if (k & 1) {
    if (mask) { T.b1 = 0; T.b2 = (int)ops - 1; }   // extra pair applied last
    else { T.b1 = 1; T.b2 = (int)ops; }            // ... and first when undoing
  } else {
    T.b1 = 0;
    T.b2 = (int)ops;
  }
}

// Vector v, element i of the block: LEFT -> x[i*ld + v], else x[v*ld + i].
template <bool LEFT>
__global__ void __launch_bounds__(512) givens_kernel(double* __restrict__ x, long ld, int k, long nvec,
                                                     int w, int passes, int ops, int b1, int b2,
                                                     const int2* __restrict__ pairs,
                                                     const double2* __restrict__ cs) {
  extern __shared__ double tile[];   // [k][w+1]
  const int wp = w + 1;
  const long v0 = (long)blockIdx.x * w;
  const int wv = (int)min((long)w, nvec - v0);
  const int nt = blockDim.x, tid = threadIdx.x;
  if (LEFT) {
    for (long f = tid; f < (long)k * w; f += nt) {
      const int i = (int)(f / w), l = (int)(f % w);
      if (l < wv) tile[i * wp + l] = x[(long)i * ld + v0 + l];
    }
  } else {
    for (long f = tid; f < (long)k * w; f += nt) {
      const int l = (int)(f / k), i = (int)(f % k);
      if (l < wv) tile[i * wp + l] = x[(v0 + l) * ld + i];
    }
  }
  __syncthreads();
  for (int t = 0; t < passes; ++t) {
    const int2* pr = pairs + (long)t * ops;
    const double2* cc = cs + (long)t * ops;
    const int lo_[3] = {0, b1, b2}, hi_[3] = {b1, b2, ops};
    for (int st = 0; st < 3; ++st) {
      const int len = hi_[st] - lo_[st];
      if (len <= 0) continue;
      for (int f = tid; f < len * w; f += nt) {
        const int j = lo_[st] + f / w, l = f % w;
        const int2 p = pr[j];
        const double2 r = cc[j];
        double* a = tile + p.x * wp + l;
        double* b = tile + p.y * wp + l;
        const double x1 = *a, x2 = *b;
        *a = __dadd_rn(__dmul_rn(x1, r.x), __dmul_rn(x2, r.y));
        *b = __dadd_rn(__dmul_rn(x1, -r.y), __dmul_rn(x2, r.x));
      }
      __syncthreads();
    }
  }
  if (LEFT) {
    for (long f = tid; f < (long)k * w; f += nt) {
      const int i = (int)(f / w), l = (int)(f % w);
      if (l < wv) x[(long)i * ld + v0 + l] = tile[i * wp + l];
    }
  } else {
    for (long f = tid; f < (long)k * w; f += nt) {
      const int l = (int)(f / k), i = (int)(f % k);
      if (l < wv) x[(v0 + l) * ld + i] = tile[i * wp + l];
    }
  }
}

constexpr size_t SMEM_CAP = 200 * 1024;

// The strip kernel for one block with the tables already on the device.
bbt_status launch_tables(bbt_ctx* ctx, const GivensDev& T, size_t m, size_t n, double* x, bool is_left);

bbt_status apply_tables(bbt_ctx* ctx, const Tables& T, size_t m, size_t n, double* x, bool is_left) {
  if (T.ops == 0) return BBT_OK;
  const long nvec = (long)(is_left ? n : m);
  if (nvec == 0) return BBT_OK;
  size_t mark = ctx->ws.top;
  int2* dp = ctx->ws.take<int2>(T.pairs.size());
  double2* dc = ctx->ws.take<double2>(T.cs.size());
  if (!dc) return fail(ctx, BBT_ERR_NOMEM, "givens mask: workspace");
  BBT_CUDA(ctx, cudaMemcpyAsync(dp, T.pairs.data(), T.pairs.size() * sizeof(int2),
                                cudaMemcpyHostToDevice, ctx->stream));
  BBT_CUDA(ctx, cudaMemcpyAsync(dc, T.cs.data(), T.cs.size() * sizeof(double2),
                                cudaMemcpyHostToDevice, ctx->stream));
  GivensDev D{T.k, T.passes, T.ops, T.b1, T.b2, dp, dc};
  BBT_TRY(launch_tables(ctx, D, m, n, x, is_left));
  ctx->ws.top = mark;   // stream order protects the tables until the kernel has run
  return BBT_OK;
}

bbt_status launch_tables(bbt_ctx* ctx, const GivensDev& T, size_t m, size_t n, double* x, bool is_left) {
  if (T.ops == 0) return BBT_OK;
  const size_t k = T.k;
  const long nvec = (long)(is_left ? n : m);
  if (nvec == 0) return BBT_OK;
  if (k * 2 * 8 > SMEM_CAP) return fail(ctx, BBT_ERR_UNSUPPORTED, "givens mask: rotated length %zu too long", k);
  // strip width: coalesced rows for LEFT (>= 16 doubles) when the strip fits,
  // and enough CTAs to cover the SMs
  int w = 32;
  while (w > 1 && k * (size_t)(w + 1) * 8 > SMEM_CAP) w >>= 1;
  const int want_ctas = 2 * ctx->num_sms;
  while (w > (is_left ? 16 : 2) && (nvec + w - 1) / w < want_ctas) w >>= 1;
  if ((long)w > nvec) {
    int w2 = 1;
    while (w2 * 2 <= nvec) w2 <<= 1;
    w = w2;
  }
  const size_t smem = k * (size_t)(w + 1) * 8;
  const int2* dp = T.pairs;
  const double2* dc = T.cs;
  const int blocks = (int)((nvec + w - 1) / w);
  const int threads = 512;
  ProfScope prof(ctx, BBT_PROF_MASK, 16.0 * (double)k * (double)nvec);
  if (is_left) {
    BBT_CUDA(ctx, cudaFuncSetAttribute(givens_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    givens_kernel<true><<<blocks, threads, smem, ctx->stream>>>(x, (long)n, (int)k, nvec, w, (int)T.passes,
                                                                (int)T.ops, T.b1, T.b2, dp, dc);
  } else {
    BBT_CUDA(ctx, cudaFuncSetAttribute(givens_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    givens_kernel<false><<<blocks, threads, smem, ctx->stream>>>(x, (long)n, (int)k, nvec, w, (int)T.passes,
                                                                 (int)T.ops, T.b1, T.b2, dp, dc);
  }
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

// ---- near-square virtual-matrix path (k > 10000) -------------------------
// Z holds every vector's body as a vm x vn matrix, laid out [r][vector][q],
// so a row rotation of all virtual matrices is one LEFT mask of the
// vm x (nvec*vn) matrix Z and a column rotation is one right mask of the
// (vm*nvec) x vn matrix Z.  Rb holds each vector's remainder strip
// (first column of its virtual matrix, then the k - vm*vn tail), nvec x (vm+rem).

// Vector v element i lives at x[v*vs + i*es].
__global__ void gather_body(const double* __restrict__ x, long vs, long es, long nvec, int vm, int vn,
                            double* __restrict__ Z) {
  const long total = nvec * vm * (long)vn;
  for (long f = blockIdx.x * (long)blockDim.x + threadIdx.x; f < total; f += (long)gridDim.x * blockDim.x) {
    const int q = (int)(f % vn);
    const long rv = f / vn;
    const long v = rv % nvec;
    const int r = (int)(rv / nvec);
    Z[f] = x[v * vs + ((long)r * vn + q) * es];
  }
}
__global__ void scatter_body(double* __restrict__ x, long vs, long es, long nvec, int vm, int vn,
                             const double* __restrict__ Z) {
  const long total = nvec * vm * (long)vn;
  for (long f = blockIdx.x * (long)blockDim.x + threadIdx.x; f < total; f += (long)gridDim.x * blockDim.x) {
    const int q = (int)(f % vn);
    const long rv = f / vn;
    const long v = rv % nvec;
    const int r = (int)(rv / nvec);
    x[v * vs + ((long)r * vn + q) * es] = Z[f];
  }
}
// Rb[v][0..vm) <-> Z[r][v][0];  Rb[v][vm..vm+rem) <-> x tail.
__global__ void strip_io(double* __restrict__ x, long vs, long es, long nvec, int vm, int vn, int rem,
                         double* __restrict__ Z, double* __restrict__ Rb, int to_rb, int with_tail) {
  const int width = vm + rem;
  const long total = nvec * (long)width;
  const long body = (long)vm * vn;
  for (long f = blockIdx.x * (long)blockDim.x + threadIdx.x; f < total; f += (long)gridDim.x * blockDim.x) {
    const long v = f / width;
    const int j = (int)(f % width);
    if (j < vm) {
      double* z = Z + ((long)j * nvec + v) * vn;
      if (to_rb) Rb[f] = *z; else *z = Rb[f];
    } else if (with_tail) {
      double* t = x + v * vs + (body + (j - vm)) * es;
      if (to_rb) Rb[f] = *t; else *t = Rb[f];
    }
  }
}
// forward: S[r][v][q] = Z[r][v][(q - r) mod vn];  back: Z[r][v][q] = S[r][v][(q + r) mod vn]
__global__ void shift_rows(const double* __restrict__ src, double* __restrict__ dst, long nvec, int vm,
                           int vn, int forward) {
  const long total = nvec * vm * (long)vn;
  for (long f = blockIdx.x * (long)blockDim.x + threadIdx.x; f < total; f += (long)gridDim.x * blockDim.x) {
    const int q = (int)(f % vn);
    const long rv = f / vn;
    const int r = (int)(rv / nvec);
    long s = forward ? ((long)q - r) % vn : ((long)q + r) % vn;
    if (s < 0) s += vn;
    dst[f] = src[rv * vn + s];
  }
}

// bbtsvd.cpp:166-188: k - remain = rows * cols, rows < 10000, 1 < cols,
// aspect ratio < 2, most square; remain grows until one exists.
void square_convert(size_t k, size_t* rows, size_t* cols, size_t* remain) {
  const size_t lim = 10000;
  for (size_t rem = 0;; ++rem) {
    const size_t kk = k - rem;
    size_t bm = kk, bn = 1;
    for (size_t i = lim; i > 1; --i) {
      if (kk % i) continue;
      const size_t q = kk / i;
      if (i > q && q < lim && q > 1 && (i - q) < (bm - bn) && ((double)i / (double)q) < 2) { bm = i; bn = q; }
    }
    if (bm < lim) { *rows = bm; *cols = bn; *remain = rem; return; }
  }
}

}  // namespace

void draw_givens_tables(size_t k, size_t passes, bool mask, unsigned seed, GivensTables& T) {
  draw_tables(k, passes, mask, seed, T);
}

bbt_status apply_givens(bbt_ctx* ctx, const GivensDev& T, size_t m, size_t n, double* x, bool is_left) {
  if (T.k > 10000) return fail(ctx, BBT_ERR_ARG, "givens mask: prepared tables of the direct path only");
  return launch_tables(ctx, T, m, n, x, is_left);
}

bbt_status givens_mask(bbt_ctx* ctx, size_t m, size_t n, size_t passes, double* x, bool mask,
                       bool is_left, unsigned seed) {
  const size_t k = is_left ? m : n;
  Tables T;
  draw_tables(k, passes, mask, seed, T);
  if (k <= 1 || passes == 0) return BBT_OK;
  return apply_tables(ctx, T, m, n, x, is_left);
}

size_t mask_workspace_bytes(size_t m, size_t n, size_t passes, bool is_left) {
  const size_t k = is_left ? m : n, nvec = is_left ? n : m;
  if (k <= 10000) return passes * (k + 2) * 24 + 1024;
  size_t vm, vn, rem;
  square_convert(k, &vm, &vn, &rem);
  const size_t tables = passes * (std::max(vm + rem, vn) + 2) * 24 + 1024;
  return nvec * (2 * vm * vn + vm + rem) * 8 + 3 * 256 + tables;
}

// The vectors of x (columns for is_left, rows otherwise) are masked
// independently with the same rotation tables, so the virtual-matrix path
// processes them in batches sized to the free workspace.
bbt_status block_shift_mask(bbt_ctx* ctx, size_t m, size_t n, size_t passes, double* x, bool mask,
                            bool is_left, unsigned seed) {
  srand(seed);
  const size_t k = is_left ? m : n;
  if (k <= 10000) return givens_mask(ctx, m, n, passes, x, mask, is_left, seed);
  size_t vm, vn, rem;
  square_convert(k, &vm, &vn, &rem);
  const long nv_all = (long)(is_left ? n : m);
  const long vs = is_left ? 1 : (long)n, es = is_left ? (long)n : 1;
  const size_t per_vec = (2 * vm * vn + vm + rem) * 8;
  const size_t fixed = 3 * 256 + passes * (std::max(vm + rem, vn) + 2) * 24 + 2048;
  const size_t room = ctx->ws.room();
  const long batch = room > fixed ? (long)std::min<size_t>((size_t)nv_all, (room - fixed) / per_vec) : 0;
  if (batch < 1)
    return fail(ctx, BBT_ERR_NOMEM, "block_shift_mask: workspace (%zu bytes per vector of %zu)", per_vec, k);
  const size_t mark = ctx->ws.top;
  double* Z = ctx->ws.take<double>((size_t)batch * vm * vn);
  double* S = ctx->ws.take<double>((size_t)batch * vm * vn);
  double* Rb = ctx->ws.take<double>((size_t)batch * (vm + rem));
  if (!Z || !S || !Rb) return fail(ctx, BBT_ERR_NOMEM, "block_shift_mask: workspace");
  const int thr = 256;
  const int grid = 4 * ctx->num_sms;
  const unsigned s1 = seed + 1000, s2 = seed + 2000, s3 = seed + 3000, s4 = seed + 4000, s5 = seed + 5000;
  for (long v0 = 0; v0 < nv_all; v0 += batch) {
    const long nvec = std::min(batch, nv_all - v0);
    double* xb = x + v0 * vs;
    const size_t zr = (size_t)vm, zc = (size_t)nvec * vn;    // Z as LEFT target: vm x (nvec*vn)
    const size_t yr = (size_t)vm * nvec, yc = vn;            // Z as right target: (vm*nvec) x vn
    const size_t rw = vm + rem;
    gather_body<<<grid, thr, 0, ctx->stream>>>(xb, vs, es, nvec, (int)vm, (int)vn, mask ? Z : S);
    BBT_LAUNCHED(ctx);
    if (mask) {   // bbtsvd.cpp:560-613
      if (rem) {
        strip_io<<<grid, thr, 0, ctx->stream>>>(xb, vs, es, nvec, (int)vm, (int)vn, (int)rem, Z, Rb, 1, 1);
        BBT_LAUNCHED(ctx);
        BBT_TRY(givens_mask(ctx, nvec, rw, passes, Rb, true, false, s1));
        strip_io<<<grid, thr, 0, ctx->stream>>>(xb, vs, es, nvec, (int)vm, (int)vn, (int)rem, Z, Rb, 0, 0);
        BBT_LAUNCHED(ctx);
      }
      BBT_TRY(givens_mask(ctx, zr, zc, passes, Z, true, true, s2));
      shift_rows<<<grid, thr, 0, ctx->stream>>>(Z, S, nvec, (int)vm, (int)vn, 1);
      BBT_LAUNCHED(ctx);
      BBT_TRY(givens_mask(ctx, zr, zc, passes, S, true, true, s3));
      BBT_TRY(givens_mask(ctx, yr, yc, passes, S, true, false, s4));
      if (rem) {
        strip_io<<<grid, thr, 0, ctx->stream>>>(xb, vs, es, nvec, (int)vm, (int)vn, (int)rem, S, Rb, 1, 0);
        BBT_LAUNCHED(ctx);
        BBT_TRY(givens_mask(ctx, nvec, rw, passes, Rb, true, false, s5));
        strip_io<<<grid, thr, 0, ctx->stream>>>(xb, vs, es, nvec, (int)vm, (int)vn, (int)rem, S, Rb, 0, 1);
        BBT_LAUNCHED(ctx);
      }
      scatter_body<<<grid, thr, 0, ctx->stream>>>(xb, vs, es, nvec, (int)vm, (int)vn, S);
      BBT_LAUNCHED(ctx);
    } else {      // bbtsvd.cpp:615-663
      if (rem) {
        strip_io<<<grid, thr, 0, ctx->stream>>>(xb, vs, es, nvec, (int)vm, (int)vn, (int)rem, S, Rb, 1, 1);
        BBT_LAUNCHED(ctx);
        BBT_TRY(givens_mask(ctx, nvec, rw, passes, Rb, false, false, s5));
        strip_io<<<grid, thr, 0, ctx->stream>>>(xb, vs, es, nvec, (int)vm, (int)vn, (int)rem, S, Rb, 0, 0);
        BBT_LAUNCHED(ctx);
      }
      BBT_TRY(givens_mask(ctx, zr, zc, passes, S, false, true, s3));
      BBT_TRY(givens_mask(ctx, yr, yc, passes, S, false, false, s4));
      shift_rows<<<grid, thr, 0, ctx->stream>>>(S, Z, nvec, (int)vm, (int)vn, 0);
      BBT_LAUNCHED(ctx);
      BBT_TRY(givens_mask(ctx, zr, zc, passes, Z, false, true, s2));
      if (rem) {
        strip_io<<<grid, thr, 0, ctx->stream>>>(xb, vs, es, nvec, (int)vm, (int)vn, (int)rem, Z, Rb, 1, 0);
        BBT_LAUNCHED(ctx);
        BBT_TRY(givens_mask(ctx, nvec, rw, passes, Rb, false, false, s1));
        strip_io<<<grid, thr, 0, ctx->stream>>>(xb, vs, es, nvec, (int)vm, (int)vn, (int)rem, Z, Rb, 0, 1);
        BBT_LAUNCHED(ctx);
      }
      scatter_body<<<grid, thr, 0, ctx->stream>>>(xb, vs, es, nvec, (int)vm, (int)vn, Z);
      BBT_LAUNCHED(ctx);
    }
  }
  ctx->ws.top = mark;
  return BBT_OK;
}

}  // namespace bbt
