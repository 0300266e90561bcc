// Ralha one-sided bidiagonalisation (Excalibur src/client.cpp:801-958,
// overlapped variant :829-910) as ONE persistent cooperative kernel.
//
// The reference runs m-2 steps; each needs the Gram row g = W[i+1:] w_i
// plus four dot products, one ring all-reduce of m+3-i doubles across the
// participants, a Householder reflector (dlarfg), its application to rows
// i+1.. (dgemv + dger), and a Gram-Schmidt update of row i.  Here the
// participants' column slabs sit side by side in one m x m row-major
// matrix (m rows, n columns: n = m after the global QR of the short-and-wide
// branch, n = sum_c min(m_part[c], global_n) in the tall-and-skinny branch,
// client.cpp:805-814), so the all-reduce is the in-device reduction of each
// dot product,
// and a step is two grid-wide phases separated by bounded grid barriers:
//
//   B1 (column-partitioned, one CTA per SM, 8 columns x 32 row phases per
//      pass): every CTA forms the reflector from g and the step's extra
//      dots from the CTAs' partial sums (the same sums in the same order in
//      every CTA), writes its share of the Householder store, vt = sum_t
//      h_t W[i+1+t] for its columns, the next row i+1 after the update, row
//      i of V (w_i - beta v_{i-1}) / alpha_i, and its columns' share of the
//      next step's extra dots (w_{i+1}.v_i, v_i.v_i, w_{i+1}.w_{i+1}).
//   B2 (row-partitioned, one warp per row): W[r] += (-tau vt) h_r for
//      r > i, and, in the same pass, the next step's Gram row
//      g'[r] = W[r] . W[i+1].
// The passes over W keep eight loads in flight per thread; B2 reads the two
// vectors every row needs (-tau vt and the updated row i+1) from shared
// memory, staged once per CTA and step.
//
// Barriers spin a bounded number of times; on a timeout every CTA stops and
// the host reports BBT_ERR_TIMEOUT.
#include <algorithm>
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "internal.h"
#include "sync.cuh"

namespace bbt {
namespace {

constexpr int RT = 256;                 // threads per CTA
constexpr int RW = RT / 32;             // warps per CTA
constexpr int CB = 8;                   // columns per pass of B1
constexpr int RB = 8;                   // loads in flight per thread in the passes over W
constexpr size_t RALHA_STAGE_MAX = 200 * 1024;   // shared bytes for the staged vectors (n <= 12800)

struct RalhaArgs {
  int m, n;
  double* W;       // m x n row-major, rows are the vectors
  double* house;   // m x m row-major, zero on entry
  double* tau;     // m, zero on entry
  double* alpha;   // m
  double* beta;    // m-1 (lower bidiagonal)
  double* V;       // m x n row-major, left vectors, zero on entry
  double* g;       // 2 x m: Gram rows, ping-pong between steps
  double* part;    // 2 x grid x 4: per-CTA partial extra dots, ping-pong between steps
  double* vt;      // n
  double* tv;      // n: -tau * vt
  double* nextw;   // n: row i+1 after the update
  unsigned* bar;   // grid barrier
  int* err;
  int stage;       // 1: B2 reads tv and nextw from shared memory (2n doubles)
};

__device__ double block_sum(double v, double* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double s = 0.0;
  for (int k = 0; k < RW; ++k) s += sh[k];
  __syncthreads();
  return s;
}

// Four block-wide sums in one pass (two barriers).
__device__ void block_sum4(double (&v)[4], double (*sh)[4]) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 4; ++q)
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < 4; ++q) sh[w][q] = v[q];
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    double t = 0.0;
    for (int k = 0; k < RW; ++k) t += sh[k][q];
    v[q] = t;
  }
  __syncthreads();
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Gram row for step i from rows r >= i+1 against row `piv`, into out.
__device__ void gram_rows(const RalhaArgs& A, int i, const double* piv, double* out) {
  const int m = A.m, n = A.n;
  const int gw = blockIdx.x * RW + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  const int nw = gridDim.x * RW;
  for (int r = i + 1 + gw; r < m; r += nw) {
    const double* row = A.W + (long)r * n;
    double s = 0.0;
    for (int c = lane; c < n; c += 32) s += row[c] * piv[c];
    s = warp_sum(s);
    if (lane == 0) out[r - i - 1] = s;
  }
}

__global__ void __launch_bounds__(RT, 1) ralha_kernel(RalhaArgs A) {
  extern __shared__ double st_dyn[];
  __shared__ double sh[RW];
  __shared__ double sh4[RW][4];
  __shared__ double scal[6];   // beta_{i-1}, alpha_i, tau, scale, 1/alpha_i
  __shared__ double red[RT / CB][CB + 1];
  const int m = A.m, n = A.n;
  const int tid = threadIdx.x;
  const bool stage = A.stage != 0;   // tv and nextw copied to shared memory for B2
  double* st_tv = st_dyn;
  double* st_nw = st_dyn + n;
  // ---- step 0 set-up: alpha_0, v_0 (CTA 0); Gram row of w_0 (all)
  if (blockIdx.x == 0) {
    double s = 0.0;
    for (int c = tid; c < n; c += RT) s += A.W[c] * A.W[c];
    s = block_sum(s, sh);
    const double a0 = sqrt(s);
    if (tid == 0) A.alpha[0] = a0;
    const double inv = 1.0 / a0;
    for (int c = tid; c < n; c += RT) A.V[c] = inv * A.W[c];
    if (tid == 0) A.house[0] = 1.0;
  }
  gram_rows(A, 0, A.W, A.g);
  if (!grid_sync(A.bar, A.err)) return;

  // columns owned in B1
  const int cw = (n + gridDim.x - 1) / gridDim.x;
  const int c0 = blockIdx.x * cw;
  const int c1 = min(n, c0 + cw);

  for (int i = 0; i + 2 < m; ++i) {
    const int len = m - 1 - i;   // g[0..len)
    const double* g = A.g + (long)(i & 1) * m;
    double* gn = A.g + (long)((i + 1) & 1) * m;
    const double* pin = A.part + (long)(i & 1) * gridDim.x * 4;
    double* pout = A.part + (long)((i + 1) & 1) * gridDim.x * 4;
    // ---- scalars (identical in every CTA: the same sums in the same order)
    {
      double v4[4] = {0.0, 0.0, 0.0, 0.0};
      for (int t = 1 + tid; t < len; t += RT) v4[0] += g[t] * g[t];
      if (i > 0)   // the extra dots of this step: the CTAs' partial sums from the previous B1
        for (int q = tid; q < gridDim.x; q += RT) {
          v4[1] += pin[4 * q];
          v4[2] += pin[4 * q + 1];
          v4[3] += pin[4 * q + 2];
        }
      block_sum4(v4, sh4);
      const double s = v4[0];
      if (tid == 0) {
        const double al = g[0];
        double be = al, ta = 0.0, scl = 0.0;
        if (s != 0.0) {   // dlarfg
          const double h = hypot(al, sqrt(s));
          be = -copysign(h, al);
          ta = (be - al) / be;
          scl = 1.0 / (al - be);
        }
        scal[2] = ta;
        scal[3] = scl;
        if (i > 0) {   // w_i.v_{i-1}, v_{i-1}.v_{i-1}, w_i.w_i
          const double b = v4[1];
          const double vv = v4[2], ww = v4[3], vw = v4[1];
          const double a = sqrt(vv * (b * b) + ww - 2 * b * vw);
          scal[0] = b;
          scal[1] = a;
          scal[4] = 1.0 / a;
          if (blockIdx.x == 0) { A.beta[i - 1] = b; A.alpha[i] = a; }
        }
        if (blockIdx.x == 0) A.tau[i + 1] = ta;
      }
      __syncthreads();
    }
    const double ta = scal[2], scl = scal[3];
    // ---- B1: Householder store, vt, next row, V row i (my columns)
    // house column i+1 from row i+1: (1, g[1:] * scale); rows split across CTAs
    for (int t = blockIdx.x * RT + tid; t < len; t += gridDim.x * RT)
      A.house[(long)(i + 1 + t) * m + (i + 1)] = (t == 0) ? 1.0 : g[t] * scl;
    {
      // vt[c] = sum_t h_t W[i+1+t][c] with h_0 = 1, h_t = g[t]*scale: CB columns per
      // pass, RT / CB row phases (a warp reads 64-byte row segments of 4 rows)
      const int ncol = c1 - c0;
      for (int cb = 0; cb < ncol; cb += CB) {
        const int c = c0 + cb + (tid % CB);
        double s = 0.0;
        if (c < c1) {
          constexpr int PH = RT / CB;
          const double* wc = A.W + (long)(i + 1) * n + c;
          double s1 = 0.0;
          int t = tid / CB;
          if (t == 0) {
            s = wc[0];   // h_0 = 1
            t += PH;
          }
          for (; t + (RB - 1) * PH < len; t += RB * PH) {   // RB rows' loads in flight
            double w[RB], hh[RB];
#pragma unroll
            for (int e = 0; e < RB; ++e) {
              w[e] = wc[(long)(t + e * PH) * n];
              hh[e] = g[t + e * PH];
            }
#pragma unroll
            for (int e = 0; e < RB; e += 2) {
              s += (hh[e] * scl) * w[e];
              s1 += (hh[e + 1] * scl) * w[e + 1];
            }
          }
          for (; t < len; t += PH) s += (g[t] * scl) * wc[(long)t * n];
          s += s1;
        }
        red[tid / CB][tid % CB] = s;
        __syncthreads();
        if (tid < CB && c0 + cb + tid < c1) {
          const int cc = c0 + cb + tid;
          double v = 0.0;
          for (int k = 0; k < RT / CB; ++k) v += red[k][tid];
          A.vt[cc] = v;
          const double tvv = -ta * v;
          A.tv[cc] = tvv;
          A.nextw[cc] = A.W[(long)(i + 1) * n + cc] + tvv;   // h_0 = 1
        }
        __syncthreads();
      }
      if (i > 0) {
        const double b = scal[0], inva = scal[4];
        for (int c = c0 + tid; c < c1; c += RT) {
          const double w = A.W[(long)i * n + c] + (-b) * A.V[(long)(i - 1) * n + c];
          A.W[(long)i * n + c] = w;
          A.V[(long)i * n + c] = inva * w;
        }
      }
      // this CTA's share of the next step's extra dots: w_{i+1}.v_i, v_i.v_i, w_{i+1}.w_{i+1}
      __syncthreads();
      if (tid < 32) {
        double p0 = 0.0, p1 = 0.0, p2 = 0.0;
        const double* v = A.V + (long)i * n;
        for (int c = c0 + tid; c < c1; c += 32) {
          const double w = A.nextw[c], vc = v[c];
          p0 += w * vc;
          p1 += vc * vc;
          p2 += w * w;
        }
        p0 = warp_sum(p0);
        p1 = warp_sum(p1);
        p2 = warp_sum(p2);
        if (tid == 0) {
          pout[4 * blockIdx.x] = p0;
          pout[4 * blockIdx.x + 1] = p1;
          pout[4 * blockIdx.x + 2] = p2;
        }
      }
    }
    if (!grid_sync(A.bar, A.err)) return;
    // ---- B2: rank-1 update of rows i+1.., next Gram row
    {
      // -tau vt and row i+1 after the update, read by every row: staged once per CTA
      const double* tv = A.tv;
      const double* nw_ = A.nextw;
      if (stage) {
        for (int c = tid; c < n; c += RT) {
          st_tv[c] = A.tv[c];
          st_nw[c] = A.nextw[c];
        }
        __syncthreads();
        tv = st_tv;
        nw_ = st_nw;
      }
      const int gw = blockIdx.x * RW + (tid >> 5), lane = tid & 31;
      const int nw = gridDim.x * RW;
      for (int r = i + 1 + gw; r < m; r += nw) {
        const int t = r - i - 1;
        const double h = (t == 0) ? 1.0 : g[t] * scl;
        double* row = A.W + (long)r * n;
        double s = 0.0, s1 = 0.0;
        // batches of RB segments: all loads of a batch issued before its stores
        int c = lane;
        for (; c + (RB - 1) * 32 < n; c += RB * 32) {
          double w[RB];
#pragma unroll
          for (int e = 0; e < RB; ++e) w[e] = row[c + 32 * e];
#pragma unroll
          for (int e = 0; e < RB; ++e) {
            w[e] = fma(tv[c + 32 * e], h, w[e]);
            if (e & 1) s1 = fma(w[e], nw_[c + 32 * e], s1);
            else s = fma(w[e], nw_[c + 32 * e], s);
          }
#pragma unroll
          for (int e = 0; e < RB; ++e) row[c + 32 * e] = w[e];
        }
        {
          double w[RB];
#pragma unroll
          for (int e = 0; e < RB; ++e) w[e] = (c + 32 * e < n) ? row[c + 32 * e] : 0.0;
#pragma unroll
          for (int e = 0; e < RB; ++e)
            if (c + 32 * e < n) {
              w[e] = fma(tv[c + 32 * e], h, w[e]);
              s = fma(w[e], nw_[c + 32 * e], s);
              row[c + 32 * e] = w[e];
            }
        }
        s = warp_sum(s + s1);
        // g for step i+1 has entries for rows >= i+2
        if (lane == 0 && r >= i + 2) gn[r - i - 2] = s;
      }
    }
    if (!grid_sync(A.bar, A.err)) return;
  }
  // ---- tail steps i = m-2, m-1 (client.cpp:897-905), CTA 0
  if (blockIdx.x != 0) return;
  for (int i = (m >= 3 ? m - 2 : 1); i < m; ++i) {
    const double* vp = A.V + (long)(i - 1) * n;
    double* wi = A.W + (long)i * n;
    double s = 0.0;
    for (int c = tid; c < n; c += RT) s += wi[c] * vp[c];
    const double b = block_sum(s, sh);
    double q = 0.0;
    for (int c = tid; c < n; c += RT) {
      const double w = wi[c] + (-b) * vp[c];
      wi[c] = w;
      q += w * w;
    }
    q = block_sum(q, sh);
    const double a = sqrt(q);
    const double inv = 1.0 / a;
    for (int c = tid; c < n; c += RT) A.V[(long)i * n + c] = inv * wi[c];
    if (tid == 0) { A.beta[i - 1] = b; A.alpha[i] = a; }
    __syncthreads();
  }
}

// Lower -> upper bidiagonal with drotg (client.cpp:947-954); one thread.
__device__ void drotg_ref(double& a, double& b, double& c, double& s) {
  const double roe = fabs(a) > fabs(b) ? a : b;
  const double scale = fabs(a) + fabs(b);
  double r;
  if (scale == 0.0) {
    c = 1.0; s = 0.0; r = 0.0;
  } else {
    const double as = a / scale, bs = b / scale;
    r = scale * sqrt(as * as + bs * bs);
    r = copysign(1.0, roe) * r;
    c = a / r;
    s = b / r;
  }
  a = r;
}

__global__ void lower_to_upper_kernel(int m, double* __restrict__ alpha, double* __restrict__ beta,
                                      double* __restrict__ cs) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int i = 0; i + 1 < m; ++i) {
    double a = alpha[i], b = beta[i], c, s;
    drotg_ref(a, b, c, s);
    alpha[i] = a;
    cs[2 * i] = c;
    cs[2 * i + 1] = s;
    beta[i] = s * alpha[i + 1];
    alpha[i + 1] = c * alpha[i + 1];
  }
}

}  // namespace

bbt_status ralha(bbt_ctx* ctx, int m, int n, double* W, double* house, double* tau, double* alpha,
                 double* beta, double* V, double* cs) {
  if (m < 3) return fail(ctx, BBT_ERR_UNSUPPORTED, "ralha: m=%d (the reference needs m >= 3)", m);
  if (n < 1) return fail(ctx, BBT_ERR_ARG, "ralha: n=%d", n);
  size_t mark = ctx->ws.top;
  RalhaArgs A;
  A.m = m;
  A.n = n;
  A.W = W;
  A.house = house;
  A.tau = tau;
  A.alpha = alpha;
  A.beta = beta;
  A.V = V;
  A.g = ctx->ws.take<double>(2 * (size_t)m);
  A.part = ctx->ws.take<double>(8 * (size_t)std::max(ctx->num_sms, 1));
  A.vt = ctx->ws.take<double>(n);
  A.tv = ctx->ws.take<double>(n);
  A.nextw = ctx->ws.take<double>(n);
  if (!A.nextw) return fail(ctx, BBT_ERR_NOMEM, "ralha: workspace");
  A.bar = ctx->d_barrier;
  A.err = ctx->d_flag;
  const size_t smem = 2 * (size_t)n * sizeof(double);
  A.stage = smem <= RALHA_STAGE_MAX;
  static bool attr = false;
  if (A.stage && !attr) {
    BBT_CUDA(ctx, cudaFuncSetAttribute(ralha_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)RALHA_STAGE_MAX));
    attr = true;
  }
  const size_t dsmem = A.stage ? smem : 0;
  BBT_CUDA(ctx, cudaMemsetAsync(house, 0, (size_t)m * m * sizeof(double), ctx->stream));
  BBT_CUDA(ctx, cudaMemsetAsync(V, 0, (size_t)m * n * sizeof(double), ctx->stream));
  BBT_CUDA(ctx, cudaMemsetAsync(tau, 0, (size_t)m * sizeof(double), ctx->stream));
  BBT_CUDA(ctx, cudaMemsetAsync(ctx->d_barrier, 0, 2 * sizeof(unsigned), ctx->stream));
  BBT_CUDA(ctx, cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), ctx->stream));
  int per_sm = 0;
  BBT_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ralha_kernel, RT, dsmem));
  if (per_sm < 1) return fail(ctx, BBT_ERR_CUDA, "ralha: kernel does not fit an SM");
  int grid = (n + CB - 1) / CB;             // at least CB columns per CTA in B1, one CTA per SM
  if (grid > ctx->num_sms * per_sm) grid = ctx->num_sms * per_sm;
  if (grid > ctx->num_sms) grid = ctx->num_sms;
  if (grid < 1) grid = 1;
  void* args[] = {&A};
  ProfScope prof(ctx, BBT_PROF_RALHA, 16.0 * (double)m * m * n / 3.0);
  BBT_CUDA(ctx, cudaLaunchCooperativeKernel((void*)ralha_kernel, dim3(grid), dim3(RT), args, dsmem, ctx->stream));
  BBT_LAUNCHED(ctx);
  lower_to_upper_kernel<<<1, 1, 0, ctx->stream>>>(m, alpha, beta, cs);
  BBT_LAUNCHED(ctx);
  int herr = 0;
  BBT_CUDA(ctx, cudaMemcpyAsync(&herr, ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  BBT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->ws.top = mark;
  if (herr) return fail(ctx, BBT_ERR_TIMEOUT, "ralha: grid barrier timed out");
  return BBT_OK;
}

}  // namespace bbt
