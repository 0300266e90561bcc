// Double-double (about 106-bit) triangular solves with an FP64 triangular
// factor, for the preconditioned exact Gram of the mixed-precision local QR:
//
//   solve R^T X = B  (trans)   or   R X = B,   R upper m x m (column-major, FP64),
//   X, B m x k column-major double-doubles (hi + lo arrays), in place.
//
// Every column of X is an independent solve, so one CTA takes a group of up
// to 8 columns (one warp each) and solves them start to finish with the
// columns held in shared memory: one launch, no CTA waits for another.
// Left-looking in 32-row blocks: the block's rows first gather the terms of
// every row already solved (products of an FP64 and a double-double summed
// as compensated dot products over rows of R staged through shared memory,
// four independent chains per thread), then the 32 x 32 diagonal block is
// solved in registers, one row per lane, broadcasting each solved row by
// warp shuffles.  Columns too long for shared memory take a blocked
// multi-launch path instead (a leaf kernel per diagonal block, an update
// kernel for the rows still to solve).  The double-double operations are the
// classical error-free transformations (Knuth's two-sum, the FMA
// two-product) with the usual renormalisations.
#include <cuda_runtime.h>

#include <algorithm>

#include "internal.h"

namespace bbt {
namespace {

constexpr int NB = 32;

struct dd {
  double hi, lo;
};

// The error-free transformations need every sum and product rounded on its
// own: the _rn intrinsics are never merged into a fused multiply-add.
__device__ __forceinline__ dd two_sum(double a, double b) {
  const double s = __dadd_rn(a, b);
  const double bb = __dsub_rn(s, a);
  return {s, __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb))};
}
__device__ __forceinline__ dd quick_two_sum(double a, double b) {   // |a| >= |b|
  const double s = __dadd_rn(a, b);
  return {s, __dsub_rn(b, __dsub_rn(s, a))};
}
__device__ __forceinline__ dd dd_add(dd x, dd y) {
  dd s = two_sum(x.hi, y.hi);
  const dd t = two_sum(x.lo, y.lo);
  s.lo += t.hi;
  s = quick_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return quick_two_sum(s.hi, s.lo);
}
// a (double) times x (double-double)
__device__ __forceinline__ dd dd_mul_d(dd x, double a) {
  const double p = __dmul_rn(x.hi, a);
  const double e = fma(x.hi, a, -p) + x.lo * a;
  return quick_two_sum(p, e);
}
// x / a given ia = 1/a rounded: q1 = x.hi ia, the remainder x - q1 a
// exactly, then its quotient (q1's error is a few ulps, the correction
// restores double-double accuracy without a division instruction)
__device__ __forceinline__ dd dd_div_d(dd x, double a, double ia) {
  const double q1 = x.hi * ia;
  const double p = __dmul_rn(q1, a);
  const double pe = fma(q1, a, -p);
  const dd r = dd_add(x, {-p, -pe});
  const double q2 = r.hi * ia;
  return quick_two_sum(q1, q2);
}

// Compensated accumulation of sum_t a_t x_t (a_t doubles, x_t double-doubles):
// the running sum s with the exact error terms of its products and additions
// gathered in c (TwoProduct / TwoSum), renormalised once at the end.
struct dot2 {
  double s = 0.0, c = 0.0;
  __device__ __forceinline__ void add(double a, dd x) {
    const double p = __dmul_rn(a, x.hi);
    const double pe = fma(a, x.hi, -p);
    const double t = __dadd_rn(s, p);
    const double bb = __dsub_rn(t, s);
    c += (__dsub_rn(s, __dsub_rn(t, bb)) + __dsub_rn(p, bb)) + pe + a * x.lo;
    s = t;
  }
  __device__ __forceinline__ dd value() const { return quick_two_sum(s, c); }
};

// Diagonal block [j0, j0 + nb) of R: X[j0.., c] <- R_jj^{-T} X (trans) or R_jj^{-1} X.
// Right-looking and fully unrolled: after x_r is known, every remaining
// accumulator takes its term, so the updates of a step are independent.
// Rows past nb are padded with an identity block and a zero right-hand side.
__global__ void leaf_kernel(int trans, int nb, int j0, int k, const double* __restrict__ R, long ldr,
                            double* __restrict__ Xh, double* __restrict__ Xl, long ldx) {
  __shared__ double Rs[NB][NB + 1];   // Rs[r][c] = R(j0 + r, j0 + c)
  __shared__ double Ri[NB];           // 1 / R(j0 + r, j0 + r)
  for (int f = threadIdx.x; f < NB * NB; f += blockDim.x) {
    const int r = f % NB, c = f / NB;
    Rs[r][c] = (r < nb && c < nb) ? R[(j0 + r) + (long)(j0 + c) * ldr] : (r == c ? 1.0 : 0.0);
  }
  __syncthreads();
  for (int r = threadIdx.x; r < NB; r += blockDim.x) Ri[r] = 1.0 / Rs[r][r];
  __syncthreads();
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= k) return;
  double* xh = Xh + (long)col * ldx + j0;
  double* xl = Xl + (long)col * ldx + j0;
  dd x[NB];
#pragma unroll
  for (int r = 0; r < NB; ++r) x[r] = (r < nb) ? dd{xh[r], xl[r]} : dd{0.0, 0.0};
  if (trans) {   // forward with R^T (lower): x_r, then rows t > r lose R(r, t) x_r
#pragma unroll
    for (int r = 0; r < NB; ++r) {
      x[r] = dd_div_d(x[r], Rs[r][r], Ri[r]);
#pragma unroll
      for (int t = r + 1; t < NB; ++t) x[t] = dd_add(x[t], dd_mul_d(x[r], -Rs[r][t]));
    }
  } else {       // backward with the upper R: rows t < r lose R(t, r) x_r
#pragma unroll
    for (int r = NB - 1; r >= 0; --r) {
      x[r] = dd_div_d(x[r], Rs[r][r], Ri[r]);
#pragma unroll
      for (int t = 0; t < r; ++t) x[t] = dd_add(x[t], dd_mul_d(x[r], -Rs[t][r]));
    }
  }
#pragma unroll
  for (int r = 0; r < NB; ++r)
    if (r < nb) {
      xh[r] = x[r].hi;
      xl[r] = x[r].lo;
    }
}

// X[i, c] -= sum_t A(i, t) X[j0 + t, c] for rows i in [r0, r1), A(i, t) =
// R(j0 + t, i) (trans) or R(i, j0 + t); four columns per thread (independent
// accumulation chains sharing the loads of A).
constexpr int UC = 4;
__global__ void update_kernel(int trans, int nb, int j0, int r0, int r1, int k, const double* __restrict__ R,
                              long ldr, double* __restrict__ Xh, double* __restrict__ Xl, long ldx) {
  const int i = r0 + blockIdx.x * blockDim.x + threadIdx.x;
  const int c0 = blockIdx.y * UC;
  if (i >= r1) return;
  dot2 s[UC];
  for (int t = 0; t < nb; ++t) {
    const double a = trans ? R[(j0 + t) + (long)i * ldr] : R[i + (long)(j0 + t) * ldr];
#pragma unroll
    for (int u = 0; u < UC; ++u)
      if (c0 + u < k) {
        const long o = (long)(c0 + u) * ldx + j0 + t;
        s[u].add(a, {Xh[o], Xl[o]});
      }
  }
#pragma unroll
  for (int u = 0; u < UC; ++u)
    if (c0 + u < k) {
      const long o = (long)(c0 + u) * ldx + i;
      const dd v = s[u].value();
      const dd x = dd_add({Xh[o], Xl[o]}, {-v.hi, -v.lo});
      Xh[o] = x.hi;
      Xl[o] = x.lo;
    }
}

// The single-launch solve (header).  Shared memory: the CTA's columns as
// (hi, lo) pairs, column-major xs[c][mp] (mp = m + 4 rounded to even, zero
// past m); two 32 x VT tiles of R with a row per output row (row stride VT + 2,
// so a lane's 16-byte loads hit distinct banks) and two 32 x 32 diagonal
// blocks, double-buffered: the next copy is in flight while the current one
// is used; the diagonal's reciprocals.
constexpr int VC = 8;     // columns per CTA at most (one warp each)
constexpr int VT = 128;   // solved rows per staged tile
constexpr int VS = VT + 2;
constexpr size_t VFIXED = (size_t)2 * NB * VS * sizeof(double) + (size_t)2 * NB * (NB + 1) * sizeof(double) +
                          NB * sizeof(double);
constexpr size_t VSMEM_MAX = 227 * 1024;

__host__ __device__ inline int cols_mp(int m) { return (m + 5) & ~1; }
size_t cols_smem(int m, int C) { return (size_t)cols_mp(m) * C * sizeof(double2) + VFIXED; }

// 8-byte asynchronous global -> shared copy; zero-fills when !valid (no read).
__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 8 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// The loads of the solve form one fixed sequence of jobs, independent of X:
// for each 32-row block (in solve order) its update tiles of VT solved rows,
// then its diagonal block.  Job j's copy is issued while job j - 1 is used.
// Update tiles start at multiples of 32 (16-byte aligned rows of xs).
struct ColsJob {
  int diag, b, r0, nb, t0, tl, buf;
};

template <bool TRANS>
__device__ __forceinline__ bool next_job(int m, int nblk, int& s, int& t0, ColsJob& J) {
  // (s, t0): block s of the solve order and the start of its next update tile
  if (s >= nblk) return false;
  const int b = TRANS ? s : nblk - 1 - s;
  const int r0 = b * NB, nb = min(NB, m - r0);
  const int tb = TRANS ? r0 : m;
  J.b = b;
  J.r0 = r0;
  J.nb = nb;
  if (t0 < tb) {
    J.diag = 0;
    J.t0 = t0;
    J.tl = min(VT, tb - t0);
    t0 += VT;
  } else {
    J.diag = 1;
    if (++s < nblk) {
      const int b2 = TRANS ? s : nblk - 1 - s;
      t0 = TRANS ? 0 : b2 * NB + min(NB, m - b2 * NB);
    }
  }
  return true;
}

template <bool TRANS>
__global__ void __launch_bounds__(256, 1) cols_kernel(int m, int k, int C, const double* __restrict__ R, long ldr,
                                                      double* __restrict__ Xh, double* __restrict__ Xl, long ldx) {
  extern __shared__ double4 sm4[];
  const int mp = cols_mp(m);
  double2* xs = reinterpret_cast<double2*>(sm4);                        // [C][mp]
  double* Rs = reinterpret_cast<double*>(xs + (size_t)mp * C);          // [2][NB][VS]
  double(*Rd)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(Rs + 2 * NB * VS);   // [2][NB]
  double* Ri = reinterpret_cast<double*>(Rd + 2 * NB);
  const int c0 = blockIdx.x * C, w = threadIdx.x >> 5, lane = threadIdx.x & 31, nt = blockDim.x;
  const int nblk = (m + NB - 1) / NB;
  int nu = 0;   // update tiles issued so far: they alternate between the two buffers
  auto issue = [&](ColsJob& J) {
    if (J.diag) {   // Rd[i][j] = R(r0 + i, r0 + j), upper triangle; zero elsewhere (diagonal padding fixed later)
      double(*D)[NB + 1] = Rd + (J.b & 1) * NB;
      for (int f = threadIdx.x; f < NB * NB; f += nt) {
        const int i = f % NB, j = f / NB;
        const bool ok = i < J.nb && j < J.nb && i <= j;
        cp_async8(&D[i][j], ok ? R + (J.r0 + i) + (long)(J.r0 + j) * ldr : R, ok);
      }
    } else {        // T[rr][tt] = coefficient of x[t0 + tt] in row r0 + rr: R(t, r) (TRANS) or R(r, t)
      J.buf = nu++ & 1;
      double* T = Rs + (size_t)J.buf * NB * VS;
      for (int f = threadIdx.x; f < VT * NB; f += nt) {
        const int tt = TRANS ? f % VT : f / NB, rr = TRANS ? f / VT : f % NB;
        const bool ok = tt < J.tl && rr < J.nb;
        const double* src = TRANS ? R + (J.t0 + tt) + (long)(J.r0 + rr) * ldr : R + (J.r0 + rr) + (long)(J.t0 + tt) * ldr;
        cp_async8(T + rr * VS + tt, ok ? src : R, ok);
      }
    }
    cp_async_commit();
  };

  int s = 0, tn = TRANS ? 0 : m;
  ColsJob cur, nxt;
  next_job<TRANS>(m, nblk, s, tn, cur);
  issue(cur);
  for (int f = threadIdx.x; f < mp * C; f += nt) {   // column index fastest: 32-byte runs per column
    const int c = f % C, t = f / C, col = c0 + c;
    const bool ok = t < m && col < k;
    xs[(size_t)c * mp + t] = ok ? make_double2(Xh[(long)col * ldx + t], Xl[(long)col * ldx + t]) : make_double2(0.0, 0.0);
  }
  double2* xw = xs + (size_t)w * mp;   // this warp's column
  dd acc[4] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
  bool more = true;
  while (more) {
    more = next_job<TRANS>(m, nblk, s, tn, nxt);
    if (more) {
      issue(nxt);
      cp_async_wait_1();
    } else {
      cp_async_wait_0();
    }
    __syncthreads();
    if (!cur.diag) {
      const double* arow = Rs + (size_t)cur.buf * NB * VS + lane * VS;
      const double2* xv = xw + cur.t0;
      dot2 p[4];
      // zero past the tile, so the 4-way unrolled loop needs no guard (rows up to m + 2 < mp)
      for (int tt = 0; tt < cur.tl; tt += 4) {
        const double2 a01 = *reinterpret_cast<const double2*>(arow + tt);
        const double2 a23 = *reinterpret_cast<const double2*>(arow + tt + 2);
        const double2 x0 = xv[tt], x1 = xv[tt + 1], x2 = xv[tt + 2], x3 = xv[tt + 3];
        p[0].add(a01.x, {x0.x, x0.y});
        p[1].add(a01.y, {x1.x, x1.y});
        p[2].add(a23.x, {x2.x, x2.y});
        p[3].add(a23.y, {x3.x, x3.y});
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) acc[u] = dd_add(acc[u], p[u].value());
    } else {
      double(*D)[NB + 1] = Rd + (cur.b & 1) * NB;
      if (threadIdx.x < NB) {
        if (threadIdx.x >= cur.nb) D[threadIdx.x][threadIdx.x] = 1.0;   // identity past the block
        Ri[threadIdx.x] = 1.0 / D[threadIdx.x][threadIdx.x];
      }
      __syncthreads();
      const int r0 = cur.r0, nb = cur.nb;
      const dd v = dd_add(dd_add(acc[0], acc[1]), dd_add(acc[2], acc[3]));
      dd x = {0.0, 0.0};
      if (lane < nb) {
        const double2 b = xw[r0 + lane];
        x = dd_add({b.x, b.y}, {-v.hi, -v.lo});
      }
      if (TRANS) {   // forward with R^T: x_r, then rows t > r lose R(r, t) x_r
        for (int r = 0; r < nb; ++r) {
          if (lane == r) x = dd_div_d(x, D[r][r], Ri[r]);
          const dd xr = {__shfl_sync(0xffffffffu, x.hi, r), __shfl_sync(0xffffffffu, x.lo, r)};
          if (lane > r) x = dd_add(x, dd_mul_d(xr, -D[r][lane]));
        }
      } else {       // backward with R: rows t < r lose R(t, r) x_r
        for (int r = nb - 1; r >= 0; --r) {
          if (lane == r) x = dd_div_d(x, D[r][r], Ri[r]);
          const dd xr = {__shfl_sync(0xffffffffu, x.hi, r), __shfl_sync(0xffffffffu, x.lo, r)};
          if (lane < r) x = dd_add(x, dd_mul_d(xr, -D[lane][r]));
        }
      }
      if (lane < nb) xw[r0 + lane] = make_double2(x.hi, x.lo);
#pragma unroll
      for (int u = 0; u < 4; ++u) acc[u] = {0.0, 0.0};
    }
    __syncthreads();
    cur = nxt;
  }
  for (int f = threadIdx.x; f < m * C; f += nt) {
    const int c = f % C, t = f / C, col = c0 + c;
    if (col < k) {
      const double2 v = xs[(size_t)c * mp + t];
      Xh[(long)col * ldx + t] = v.x;
      Xl[(long)col * ldx + t] = v.y;
    }
  }
}

template <bool TRANS>
cudaError_t launch_cols(bbt_ctx* ctx, int m, int k, int C, const double* R, long ldr, double* Xh, double* Xl,
                        long ldx) {
  static bool attr = false;
  if (!attr) {
    const cudaError_t e =
        cudaFuncSetAttribute(cols_kernel<TRANS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)VSMEM_MAX);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  cols_kernel<TRANS><<<(k + C - 1) / C, 32 * C, cols_smem(m, C), ctx->stream>>>(m, k, C, R, ldr, Xh, Xl, ldx);
  return cudaGetLastError();
}

__global__ void dd_transpose_kernel(int m, const double* __restrict__ Ah, const double* __restrict__ Al, long lda,
                                    double* __restrict__ Th, double* __restrict__ Tl, long ldt) {
  __shared__ double th[32][33], tl[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = bx + threadIdx.x, j = by + r;
    if (i < m && j < m) {
      th[r][threadIdx.x] = Ah[i + (long)j * lda];
      tl[r][threadIdx.x] = Al[i + (long)j * lda];
    }
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = by + threadIdx.x, j = bx + r;
    if (i < m && j < m) {
      Th[i + (long)j * ldt] = th[threadIdx.x][r];
      Tl[i + (long)j * ldt] = tl[threadIdx.x][r];
    }
  }
}

__global__ void dd_symmetrize_kernel(int m, double* __restrict__ Gh, double* __restrict__ Gl, long ld) {
  const long total = (long)m * m;
  for (long f = blockIdx.x * (long)blockDim.x + threadIdx.x; f < total; f += (long)gridDim.x * blockDim.x) {
    const int i = (int)(f % m), j = (int)(f / m);
    if (i > j) {
      Gh[i + (long)j * ld] = Gh[j + (long)i * ld];
      Gl[i + (long)j * ld] = Gl[j + (long)i * ld];
    }
  }
}

}  // namespace

bbt_status dd_trsm_left(bbt_ctx* ctx, bool trans, int m, int k, const double* R, long ldr, double* Xh, double* Xl,
                        long ldx) {
  if (m < 1 || k < 1) return BBT_OK;
  ProfScope prof(ctx, BBT_PROF_DD, (double)m * m * k);
  // about one CTA per SM; fewer columns per CTA where long columns fill shared memory
  int C = std::min(VC, std::max(1, (k + ctx->num_sms - 1) / std::max(ctx->num_sms, 1)));
  while (C > 1 && cols_smem(m, C) > VSMEM_MAX) --C;
  if (cols_smem(m, C) <= VSMEM_MAX) {
    BBT_CUDA(ctx, trans ? launch_cols<true>(ctx, m, k, C, R, ldr, Xh, Xl, ldx)
                        : launch_cols<false>(ctx, m, k, C, R, ldr, Xh, Xl, ldx));
    return BBT_OK;
  }
  const int nblk = (m + NB - 1) / NB;
  for (int s = 0; s < nblk; ++s) {
    const int b = trans ? s : nblk - 1 - s;
    const int j0 = b * NB, nb = (j0 + NB <= m) ? NB : m - j0;
    leaf_kernel<<<(k + 31) / 32, 32, 0, ctx->stream>>>(trans ? 1 : 0, nb, j0, k, R, ldr, Xh, Xl, ldx);
    BBT_LAUNCHED(ctx);
    const int r0 = trans ? j0 + nb : 0, r1 = trans ? m : j0;   // rows still to solve
    if (r1 > r0) {
      const int gy = (k + UC - 1) / UC;
      if (gy > 65535) return fail(ctx, BBT_ERR_ARG, "dd_trsm: k=%d", k);
      update_kernel<<<dim3((unsigned)((r1 - r0 + 127) / 128), (unsigned)gy), 128, 0, ctx->stream>>>(
          trans ? 1 : 0, nb, j0, r0, r1, k, R, ldr, Xh, Xl, ldx);
      BBT_LAUNCHED(ctx);
    }
  }
  return BBT_OK;
}

bbt_status dd_transpose(bbt_ctx* ctx, int m, const double* Ah, const double* Al, long lda, double* Th, double* Tl,
                        long ldt) {
  dim3 b(32, 8), g((m + 31) / 32, (m + 31) / 32);
  dd_transpose_kernel<<<g, b, 0, ctx->stream>>>(m, Ah, Al, lda, Th, Tl, ldt);
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

bbt_status dd_symmetrize_upper(bbt_ctx* ctx, int m, double* Gh, double* Gl, long ld) {
  dd_symmetrize_kernel<<<2 * ctx->num_sms, 256, 0, ctx->stream>>>(m, Gh, Gl, ld);
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

}  // namespace bbt
