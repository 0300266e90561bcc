// FP64 Cholesky factorisation, triangular solves and the sign-recovery
// elimination of the mixed-precision and exact-Gram local QRs (mixedqr.cu,
// exactqr.cu), whose R factors are built from Gram matrices.
//
// Square operands (m x m, m up to a few thousand) take single launches: a
// cooperative blocked Cholesky and sign-recovery LU with bounded grid
// barriers, and triangular solves of independent rows or columns held in
// shared memory.  Tall operands (the mixed mode's A R_p^-1 over the long
// dimension), and the concurrent streams of the batched QR where cooperative
// launches are not used, take the recursive forms: the diagonal leaves as
// small SIMT kernels, everything above them as FP64 tensor-core GEMMs
// (dgemm.cu).
#include <cuda_runtime.h>

#include <algorithm>

#include "internal.h"
#include "sync.cuh"

namespace bbt {
namespace {

constexpr int PB = 32;   // Cholesky leaf (one warp)
constexpr int TB = 32;   // triangular-solve leaf
constexpr int LB = 16;   // sign-recovery LU leaf

// Upper Cholesky G = R^T R of an n x n (n <= PB) diagonal block, in place:
// R in the upper triangle, zeros below.  One warp: lane k owns column k in
// shared memory, so the n sequential steps synchronise with __syncwarp only.
// A pivot that is not positive sets *flag and is replaced by 1 so the
// factorisation still completes.
__global__ void __launch_bounds__(32) potrf_leaf(int n, double* __restrict__ G, long ld, int* flag) {
  __shared__ double a[PB][PB + 1];
  const int k = threadIdx.x;
  for (int i = 0; i < PB; ++i) a[i][k] = (i <= k && k < n) ? G[i + (long)k * ld] : 0.0;
  __syncwarp();
  for (int j = 0; j < n; ++j) {
    double d = a[j][j];
    if (!(d > 0.0) || !isfinite(d)) {
      if (k == 0) atomicExch(flag, 1);
      d = 1.0;
    }
    const double r = sqrt(d);
    __syncwarp();
    if (k >= j && k < n) a[j][k] = (k == j) ? r : a[j][k] / r;
    __syncwarp();
    if (k > j && k < n) {
      const double ajk = a[j][k];
      for (int i = j + 1; i <= k; ++i) a[i][k] -= a[j][i] * ajk;
    }
    __syncwarp();
  }
  if (k < n)
    for (int i = 0; i < n; ++i) G[i + (long)k * ld] = (i <= k) ? a[i][k] : 0.0;
}

// A (rows x n, column-major) <- A R^{-1}, R upper n x n (n <= NB): one thread
// per row, forward substitution along the row.  Columns past n are zero in
// shared memory (unit diagonal), so the unrolled loops need no guards.
template <int NB>
__global__ void __launch_bounds__(128) trsm_leaf(long rows, int n, const double* __restrict__ R, long ldr,
                                                 double* __restrict__ A, long lda) {
  __shared__ double r[NB][NB + 1];
  __shared__ double rinv[NB];
  for (int f = threadIdx.x; f < NB * NB; f += blockDim.x) {
    const int i = f % NB, j = f / NB;
    r[i][j] = (i < n && j < n) ? (i <= j ? R[i + (long)j * ldr] : 0.0) : (i == j ? 1.0 : 0.0);
  }
  __syncthreads();
  if (threadIdx.x < NB) rinv[threadIdx.x] = 1.0 / r[threadIdx.x][threadIdx.x];
  __syncthreads();
  // one row per thread (no row loop: the shared-memory reads of R must not be
  // hoisted into registers across rows)
  const long row = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (row >= rows) return;
  double x[NB];
#pragma unroll
  for (int j = 0; j < NB; ++j) x[j] = (j < n) ? A[row + (long)j * lda] : 0.0;
#pragma unroll
  for (int j = 0; j < NB; ++j) {
    double s = x[j];
#pragma unroll
    for (int i = 0; i < j; ++i) s -= x[i] * r[i][j];
    x[j] = s * rinv[j];
  }
#pragma unroll
  for (int j = 0; j < NB; ++j)
    if (j < n) A[row + (long)j * lda] = x[j];
}

// Triangular solves of independent vectors, one launch: vector v of X is
// x_j = X[v vs + j es] (a row of a column-major X: vs = 1, es = ld; a column:
// vs = ld, es = 1), solved in place forward (FWD, j = 0, 1, ..) or backward
// against the coefficients A(j, t) = T(t, j) (TRANS) or T(j, t):
//   x_j <- (x_j - sum_{t solved} A(j, t) x_t) / A(j, j)   (no division if UNIT).
// One CTA per group of up to 8 vectors (one warp each), held in shared
// memory, so no CTA waits for another.  Left-looking in 32-element blocks:
// the block first gathers the solved terms through VT x 32 tiles of A staged
// in shared memory (four FMA chains per thread), then solves its diagonal
// block in registers, one element per lane, broadcasting by warp shuffles.
// The tiles and diagonal blocks are one fixed sequence of copies,
// independent of X, double-buffered so that the next copy is in flight
// while the current one is used.  For square and short operands (rows up to
// a few thousand), where the recursive form spends its time in launches.
constexpr int VC = 8, VT = 128, VS = VT + 2;   // VS: row stride of a staged tile (16-byte loads, distinct banks)
constexpr size_t VFIXED = (size_t)2 * TB * VS * sizeof(double) + (size_t)2 * TB * (TB + 1) * sizeof(double) +
                          TB * sizeof(double);
constexpr size_t VSMEM_MAX = 227 * 1024;

__host__ __device__ inline int vec_np(int n) { return (n + 5) & ~1; }
size_t vec_smem(int n, int C) { return (size_t)vec_np(n) * C * sizeof(double) + VFIXED; }

// 8-byte asynchronous global -> shared copy; zero-fills when !valid (no read).
__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 8 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

struct VecJob {
  int diag, b, r0, nb, t0, tl, buf;
};

// Job sequence: for each block in solve order, its update tiles over the
// solved elements, then its diagonal block.  (s, t0): the block of the solve
// order and its next update start (a multiple of 32).
template <bool FWD>
__device__ __forceinline__ bool vec_next_job(int n, int nblk, int& s, int& t0, VecJob& J) {
  if (s >= nblk) return false;
  const int b = FWD ? s : nblk - 1 - s;
  const int r0 = b * TB, nb = min(TB, n - r0);
  const int tb = FWD ? r0 : n;
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
      const int b2 = FWD ? s : nblk - 1 - s;
      t0 = FWD ? 0 : b2 * TB + min(TB, n - b2 * TB);
    }
  }
  return true;
}

template <bool TRANS, bool FWD, bool UNIT>
__global__ void __launch_bounds__(256, 1) vec_solve_kernel(int n, long nvec, int C, const double* __restrict__ T,
                                                           long ldt, double* __restrict__ X, long vs, long es) {
  extern __shared__ double2 smv[];
  const int np = vec_np(n);
  double* x = reinterpret_cast<double*>(smv);   // x[c * np + t]
  double* As = x + (size_t)np * C;              // [2][TB][VS]
  double(*Ad)[TB + 1] = reinterpret_cast<double(*)[TB + 1]>(As + 2 * TB * VS);   // [2][TB]
  double* Ai = reinterpret_cast<double*>(Ad + 2 * TB);
  const long v0 = (long)blockIdx.x * C;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nt = blockDim.x;
  const int nblk = (n + TB - 1) / TB;
  int nu = 0;
  auto issue = [&](VecJob& J) {
    if (J.diag) {   // D[i][j] = A(r0 + i, r0 + j) in the solved direction and, unless UNIT, on the diagonal
      double(*D)[TB + 1] = Ad + (J.b & 1) * TB;
      for (int f = threadIdx.x; f < TB * TB; f += nt) {
        const int i = f % TB, j = f / TB;
        const bool ok = i < J.nb && j < J.nb && ((FWD ? j < i : j > i) || (!UNIT && i == j));
        const double* src = TRANS ? T + (J.r0 + j) + (long)(J.r0 + i) * ldt : T + (J.r0 + i) + (long)(J.r0 + j) * ldt;
        cp_async8(&D[i][j], ok ? src : T, ok);
      }
    } else {        // S[rr][tt] = A(r0 + rr, t0 + tt), zero past the tile
      J.buf = nu++ & 1;
      double* S = As + (size_t)J.buf * TB * VS;
      for (int f = threadIdx.x; f < VT * TB; f += nt) {
        const int tt = TRANS ? f % VT : f / TB, rr = TRANS ? f / VT : f % TB;
        const bool ok = tt < J.tl && rr < J.nb;
        const double* src = TRANS ? T + (J.t0 + tt) + (long)(J.r0 + rr) * ldt : T + (J.r0 + rr) + (long)(J.t0 + tt) * ldt;
        cp_async8(S + rr * VS + tt, ok ? src : T, ok);
      }
    }
    cp_async_commit();
  };
  int s = 0, tn = FWD ? 0 : n;
  VecJob cur, nxt;
  vec_next_job<FWD>(n, nblk, s, tn, cur);
  issue(cur);
  for (int f = threadIdx.x; f < np * C; f += nt) {   // vector index fastest
    const int c = f % C, t = f / C;
    x[(size_t)c * np + t] = (t < n && v0 + c < nvec) ? X[(v0 + c) * vs + (long)t * es] : 0.0;
  }
  double* xw = x + (size_t)w * np;   // this warp's vector
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  bool more = true;
  while (more) {
    more = vec_next_job<FWD>(n, nblk, s, tn, nxt);
    if (more) {
      issue(nxt);
      cp_async_wait_1();
    } else {
      cp_async_wait_0();
    }
    __syncthreads();
    if (!cur.diag) {
      const double* arow = As + (size_t)cur.buf * TB * VS + lane * VS;
      const double* xv = xw + cur.t0;   // 16-byte aligned: np and t0 are even
      for (int tt = 0; tt < cur.tl; tt += 4) {
        const double2 a01 = *reinterpret_cast<const double2*>(arow + tt);
        const double2 a23 = *reinterpret_cast<const double2*>(arow + tt + 2);
        const double2 x01 = *reinterpret_cast<const double2*>(xv + tt);
        const double2 x23 = *reinterpret_cast<const double2*>(xv + tt + 2);
        acc[0] = fma(a01.x, x01.x, acc[0]);
        acc[1] = fma(a01.y, x01.y, acc[1]);
        acc[2] = fma(a23.x, x23.x, acc[2]);
        acc[3] = fma(a23.y, x23.y, acc[3]);
      }
    } else {
      double(*D)[TB + 1] = Ad + (cur.b & 1) * TB;
      if (threadIdx.x < TB) {
        if (UNIT || threadIdx.x >= cur.nb) D[threadIdx.x][threadIdx.x] = 1.0;
        Ai[threadIdx.x] = 1.0 / D[threadIdx.x][threadIdx.x];
      }
      __syncthreads();
      const int nb = cur.nb;
      double xv = (lane < nb) ? xw[cur.r0 + lane] - ((acc[0] + acc[1]) + (acc[2] + acc[3])) : 0.0;
      if (FWD) {
        for (int r = 0; r < nb; ++r) {
          if (!UNIT && lane == r) xv *= Ai[r];
          const double xr = __shfl_sync(0xffffffffu, xv, r);
          if (lane > r) xv = fma(-D[lane][r], xr, xv);
        }
      } else {
        for (int r = nb - 1; r >= 0; --r) {
          if (!UNIT && lane == r) xv *= Ai[r];
          const double xr = __shfl_sync(0xffffffffu, xv, r);
          if (lane < r) xv = fma(-D[lane][r], xr, xv);
        }
      }
      if (lane < nb) xw[cur.r0 + lane] = xv;
#pragma unroll
      for (int u = 0; u < 4; ++u) acc[u] = 0.0;
    }
    __syncthreads();
    cur = nxt;
  }
  for (int f = threadIdx.x; f < n * C; f += nt) {
    const int c = f % C, t = f / C;
    if (v0 + c < nvec) X[(v0 + c) * vs + (long)t * es] = x[(size_t)c * np + t];
  }
}

template <bool TRANS, bool FWD, bool UNIT>
cudaError_t vec_solve(bbt_ctx* ctx, int n, long nvec, const double* T, long ldt, double* X, long vs, long es) {
  static bool attr = false;
  if (!attr) {
    const cudaError_t e = cudaFuncSetAttribute(vec_solve_kernel<TRANS, FWD, UNIT>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)VSMEM_MAX);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const int C = (int)std::min<long>(VC, std::max<long>(1, (nvec + ctx->num_sms - 1) / std::max(ctx->num_sms, 1)));
  vec_solve_kernel<TRANS, FWD, UNIT><<<(unsigned)((nvec + C - 1) / C), 32 * C, vec_smem(n, C), ctx->stream>>>(
      n, nvec, C, T, ldt, X, vs, es);
  return cudaGetLastError();
}

// Where the single-launch vector solve applies: short operands (the
// recursive form's GEMMs win on tall ones) whose vectors fit shared memory.
bool vec_solve_fits(long nvec, int n) { return nvec <= 2048 && vec_smem(n, VC) <= VSMEM_MAX; }

// G12 (n1 x n2, above the diagonal) <- X^T for X = G21 (n2 x n1, below), then X <- 0.
__global__ void mirror_kernel(int n1, int n2, double* __restrict__ G, long ld) {
  const long total = (long)n1 * n2;
  for (long f = blockIdx.x * (long)blockDim.x + threadIdx.x; f < total; f += (long)gridDim.x * blockDim.x) {
    const int i = (int)(f % n1), k = (int)(f / n1);
    double* lo = G + (n1 + k) + (long)i * ld;
    G[i + (long)(n1 + k) * ld] = *lo;
    *lo = 0.0;
  }
}

// G_ii += rel * max_j G_jj (one block).
__global__ void shift_diag_kernel(int n, double* __restrict__ G, long ld, double rel) {
  __shared__ double sh[256];
  double mx = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) mx = fmax(mx, G[i + (long)i * ld]);
  sh[threadIdx.x] = mx;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + o]);
    __syncthreads();
  }
  const double s = rel * sh[0];
  for (int i = threadIdx.x; i < n; i += blockDim.x) G[i + (long)i * ld] += s;
}

__global__ void symmetrize_kernel(int n, double* __restrict__ G, long ld) {
  const long total = (long)n * n;
  for (long f = blockIdx.x * (long)blockDim.x + threadIdx.x; f < total; f += (long)gridDim.x * blockDim.x) {
    const int i = (int)(f % n), j = (int)(f / n);
    if (i > j) G[i + (long)j * ld] = G[j + (long)i * ld];
  }
}

__global__ void identity_kernel(int n, double* __restrict__ W, long ld) {
  const long total = (long)n * n;
  for (long f = blockIdx.x * (long)blockDim.x + threadIdx.x; f < total; f += (long)gridDim.x * blockDim.x) {
    const int i = (int)(f % n), j = (int)(f / n);
    W[i + (long)j * ld] = (i == j) ? 1.0 : 0.0;
  }
}

// Signs of LAPACK's Householder QR from the top block of an orthonormal Q.
// Householder QR of Q (and of any A = Q R+ with R+ positive-diagonal)
// produces Q D with D = diag(d), d_j = sign(beta_j) = -sign(alpha_j); the
// compact-WY identity I - Q1 D = Y1 T Y1^T makes the unpivoted LU of
// I - Q1 D have pivots tau_j = 1 - d_j c_j >= 1, where c_j is the j-th
// diagonal entry of Q1 after the elimination of the previous columns.  So
// d_j = -sign(c_j) (c_j = 0 -> -1, dlarfg's choice for alpha = 0), and the
// elimination runs on Q1 itself with multipliers l_ij = -d_j q_ij / (1 + |c_j|).
// Leaf: one CTA, up to TB columns of a tall panel (rows >= cols).
__global__ void __launch_bounds__(1024) lu_sign_leaf(int rows, int cols, double* __restrict__ A, long lda,
                                                     double* __restrict__ d) {
  __shared__ double rowj[LB];
  __shared__ double sdj, su;
  for (int j = 0; j < cols; ++j) {
    if (threadIdx.x == 0) {
      const double c = A[j + (long)j * lda];
      sdj = c < 0.0 ? 1.0 : -1.0;
      su = 1.0 + fabs(c);
      d[j] = sdj;
    }
    if (threadIdx.x > j && threadIdx.x < cols) rowj[threadIdx.x] = A[j + (long)threadIdx.x * lda];
    __syncthreads();
    const double f = -sdj / su;
    for (int i = j + 1 + threadIdx.x; i < rows; i += blockDim.x) {
      const double l = f * A[i + (long)j * lda];
      A[i + (long)j * lda] = l;
      for (int k = j + 1; k < cols; ++k) A[i + (long)k * lda] -= l * rowj[k];
    }
    __syncthreads();
  }
}

// The same elimination with the panel in registers: thread t owns row t
// (rows <= 1024), row j is broadcast through shared memory at step j.
__global__ void __launch_bounds__(1024) lu_sign_leaf_reg(int rows, int cols, double* __restrict__ A, long lda,
                                                         double* __restrict__ d) {
  __shared__ double rowj[LB];
  __shared__ double sf;
  const int i = threadIdx.x;
  const bool live = i < rows;
  double x[LB];
#pragma unroll
  for (int k = 0; k < LB; ++k) x[k] = (live && k < cols) ? A[i + (long)k * lda] : 0.0;
#pragma unroll
  for (int j = 0; j < LB; ++j) {
    if (j < cols) {
      if (i == j) {
#pragma unroll
        for (int k = 0; k < LB; ++k) rowj[k] = x[k];
        const double c = x[j];
        const double dj = c < 0.0 ? 1.0 : -1.0;
        d[j] = dj;
        sf = -dj / (1.0 + fabs(c));
      }
      __syncthreads();
      if (i > j && live) {
        const double l = sf * x[j];
        x[j] = l;
#pragma unroll
        for (int k = j + 1; k < LB; ++k) x[k] -= l * rowj[k];
      }
      __syncthreads();
    }
  }
  if (live)
#pragma unroll
    for (int k = 0; k < LB; ++k)
      if (k < cols) A[i + (long)k * lda] = x[k];
}

// B (n x ncols) <- L^{-1} B, L unit lower n x n (n <= LB): one thread per
// column; rows past n are zero in shared memory.
__global__ void __launch_bounds__(128) trsm_llu_leaf(int n, long ncols, const double* __restrict__ L, long ldl,
                                                     double* __restrict__ B, long ldb) {
  __shared__ double l[LB][LB + 1];
  for (int f = threadIdx.x; f < LB * LB; f += blockDim.x) {
    const int i = f % LB, k = f / LB;
    l[i][k] = (i > k && i < n) ? L[i + (long)k * ldl] : 0.0;
  }
  __syncthreads();
  const long c = blockIdx.x * (long)blockDim.x + threadIdx.x;   // one column per thread
  if (c >= ncols) return;
  double x[LB];
#pragma unroll
  for (int i = 0; i < LB; ++i) x[i] = (i < n) ? B[i + c * ldb] : 0.0;
#pragma unroll
  for (int i = 1; i < LB; ++i) {
    double s = x[i];
#pragma unroll
    for (int k = 0; k < i; ++k) s -= l[i][k] * x[k];
    x[i] = s;
  }
#pragma unroll
  for (int i = 0; i < LB; ++i)
    if (i < n) B[i + c * ldb] = x[i];
}

// Row j of R (column-major, ld m) and column j of W (column-major, ld m) times d_j.
__global__ void apply_signs_kernel(int m, const double* __restrict__ d, double* __restrict__ R,
                                   double* __restrict__ W) {
  const long total = (long)m * m;
  for (long f = blockIdx.x * (long)blockDim.x + threadIdx.x; f < total; f += (long)gridDim.x * blockDim.x) {
    const int i = (int)(f % m), j = (int)(f / m);
    R[f] *= d[i];
    if (W) W[f] *= d[j];
  }
}

// ---- single-launch factorisations for square operands ---------------------
// Cooperative launches (every CTA resident), phases separated by bounded grid
// barriers (sync.cuh): a barrier that times out sets the tensor-core wait
// flag, reported by check_tc_flags, and every CTA leaves.

// Right-looking blocked Cholesky G = R^T R (upper, 32 x 32 tiles), in place.
// Per block row k: (1) every CTA that needs it factors the diagonal tile
// (chol_tile_cta), keeps R_kk and the reciprocals of its diagonal in shared
// memory, and solves its tile of the row panel, R_kj = R_kk^-T G_kj: the
// tile is staged through shared memory with coalesced loads, lane c
// substitutes column c in registers (trsm_col_warp); (2) the trailing tiles
// G_ij -= R_ki^T R_kj, i <= j: four tiles per CTA at a time, one per pair of
// warps, every load of the round (both panel tiles and the tile updated)
// issued before any arithmetic.  Only the upper triangle of G is read; the
// strictly lower triangle is zeroed at the end.
constexpr int CT = 256;      // threads of the cooperative Cholesky
constexpr int CGROUPS = 4;   // trailing tiles per CTA and round (two warps each)
constexpr int TSTR = 33;     // padded row stride of a shared tile
constexpr size_t POTRF_SMEM = (size_t)(1 + 2 * CGROUPS) * 32 * TSTR * sizeof(double) + 32 * sizeof(double);

struct PotrfArgs {
  int n;
  double* G;
  long ld;
  int* flag;       // not-positive pivot
  unsigned* bar;   // grid barrier
  int* err;        // barrier timeout
};

// D (upper kb x kb in a padded shared tile, zero elsewhere) <- its Cholesky
// factor, by the whole CTA; rinv[j] = 1 / R(j, j).  Step j: every thread
// forms R(j, j) and its reciprocal from D(j, j) (final since the previous
// step's update), the first warp scales row j, and after a CTA barrier
// thread j stores R(j, j) while every thread updates its share of the
// trailing triangle (a second barrier).  The
// loop stays rolled: the code is small enough to stay in the instruction
// cache between the kernel's phases, which a fully unrolled register
// version did not.
__device__ __forceinline__ void chol_tile_cta(double* D, double* rinv, int kb, int* flag) {
  const int tid = threadIdx.x;
  for (int j = 0; j < kb; ++j) {
    double d = D[j * TSTR + j];
    if (!(d > 0.0) || !isfinite(d)) {
      if (tid == 0) atomicExch(flag, 1);
      d = 1.0;
    }
    const double ri = rsqrt(d);   // 1 / R(j, j); R(j, j) = d / sqrt(d)
    const double r = d * ri;
    if (tid < 32 && tid > j && tid < kb) D[j * TSTR + tid] *= ri;
    __syncthreads();   // every thread has read D(j, j); row j is scaled
    if (tid == j) {    // R(j, j): not read again in this step or later ones
      D[j * TSTR + j] = r;
      rinv[j] = ri;
    }
    for (int e = tid; e < 1024; e += CT) {
      const int a = e >> 5, b = e & 31;
      if (a > j && a <= b && b < kb) D[a * TSTR + b] = fma(-D[j * TSTR + a], D[j * TSTR + b], D[a * TSTR + b]);
    }
    __syncthreads();
  }
}

// Column lane of the shared tile T <- R_kk^-T column lane, right-looking with
// the column in registers: step i finishes x_i = x_i / R(i, i) and removes it
// from the rows below.  The array is shifted down one place per step so its
// indices stay compile-time constants in a rolled loop (row i is always x[0]).
__device__ __forceinline__ void trsm_col_warp(double* T, const double* D, const double* rinv, int kb, int lane) {
  double x[32];
#pragma unroll
  for (int i = 0; i < 32; ++i) x[i] = T[i * TSTR + lane];
  for (int i = 0; i < kb; ++i) {
    const double xi = x[0] * rinv[i];
    T[i * TSTR + lane] = xi;
#pragma unroll
    for (int u = 1; u < 32; ++u) {
      const double rt = D[i * TSTR + min(i + u, 31)];   // R(i, i + u), clamped inside the tile
      x[u - 1] = (i + u < kb) ? fma(-rt, xi, x[u]) : x[u];
    }
    x[31] = 0.0;
  }
}

__global__ void __launch_bounds__(CT, 1) potrf_coop_kernel(PotrfArgs P) {
  extern __shared__ double psm[];
  double* D = psm;                          // R_kk
  double* T = psm + 32 * TSTR;              // group tiles: [group][2][32][TSTR]
  double* rinv = psm + (1 + 2 * CGROUPS) * 32 * TSTR;
  const int n = P.n, nb = (n + 31) / 32;
  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
  const long ld = P.ld;
  for (int k = 0; k < nb; ++k) {
    const int r0 = 32 * k, kb = min(32, n - r0);
    const int jt = k + 1 + blockIdx.x;   // this CTA's panel tile (at most one: nb <= 128 < 148)
    if (blockIdx.x == 0 || jt < nb) {
      for (int f = tid; f < 1024; f += CT) {
        const int i = f & 31, j = f >> 5;
        D[i * TSTR + j] = (i < kb && j < kb && i <= j) ? P.G[(r0 + i) + (long)(r0 + j) * ld] : 0.0;
      }
      // stage the panel tile G_kj (rows r0.., columns 32 jt..), coalesced along the rows
      const int c0 = 32 * jt, jb = jt < nb ? min(32, n - c0) : 0;
      for (int f = tid; f < 1024; f += CT) {
        const int i = f & 31, c = f >> 5;
        T[i * TSTR + c] = (i < kb && c < jb) ? P.G[(r0 + i) + (long)(c0 + c) * ld] : 0.0;
      }
      __syncthreads();
      chol_tile_cta(D, rinv, kb, P.flag);
      if (blockIdx.x == 0)
        for (int f = tid; f < 1024; f += CT) {
          const int i = f & 31, j = f >> 5;
          if (i < kb && j < kb && i <= j) P.G[(r0 + i) + (long)(r0 + j) * ld] = D[i * TSTR + j];
        }
      if (jb > 0) {
        if (w == 0) trsm_col_warp(T, D, rinv, kb, lane);
        __syncthreads();
        for (int f = tid; f < 1024; f += CT) {
          const int i = f & 31, c = f >> 5;
          if (i < kb && c < jb) P.G[(r0 + i) + (long)(c0 + c) * ld] = T[i * TSTR + c];
        }
      }
    }
    if (!grid_sync(P.bar, P.err)) return;
    // trailing tiles (bi, bj), k < bi <= bj, numbered row by row; group g of
    // this CTA takes tiles blockIdx.x + (g + CGROUPS r) gridDim.x
    const int Tn = nb - k - 1, count = Tn * (Tn + 1) / 2;
    const int g = w >> 1, gt = tid & 63;
    double* A1 = T + (size_t)g * 2 * 32 * TSTR;
    double* B1 = A1 + 32 * TSTR;
    for (int base = 0; base < count; base += CGROUPS * gridDim.x) {
      const int q = base + blockIdx.x + g * gridDim.x;
      const bool live = q < count;
      int bi = 0, bj = 0;
      if (live) {
        int a = 0, rem = q;
        while (rem >= Tn - a) {
          rem -= Tn - a;
          ++a;
        }
        bi = k + 1 + a;
        bj = k + 1 + a + rem;
      }
      const int i0 = 32 * bi, j0 = 32 * bj, ib = live ? min(32, n - i0) : 0, jb = live ? min(32, n - j0) : 0;
      const int ii = gt & 31, jh = gt >> 5;
      // the tile's 16 outputs of this thread, loaded with the panel tiles
      double c[16];
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        const int jj = jh + 2 * e;
        c[e] = (ii < ib && jj < jb) ? P.G[(i0 + ii) + (long)(j0 + jj) * ld] : 0.0;
      }
      double av[16], bv[16];
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        const int f = gt + 64 * e, t = f & 31, cc = f >> 5;
        av[e] = (t < kb && cc < ib) ? P.G[(r0 + t) + (long)(i0 + cc) * ld] : 0.0;
        bv[e] = (t < kb && cc < jb) ? P.G[(r0 + t) + (long)(j0 + cc) * ld] : 0.0;
      }
      __syncthreads();   // the previous round's readers are done with A1, B1
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        const int f = gt + 64 * e, t = f & 31, cc = f >> 5;
        A1[t * TSTR + cc] = av[e];
        B1[t * TSTR + cc] = bv[e];
      }
      __syncthreads();
      if (live) {
        double acc[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) acc[e] = 0.0;
#pragma unroll 4
        for (int t = 0; t < 32; ++t) {
          const double a = A1[t * TSTR + ii];
#pragma unroll
          for (int e = 0; e < 16; ++e) acc[e] = fma(a, B1[t * TSTR + jh + 2 * e], acc[e]);
        }
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          const int jj = jh + 2 * e;
          if (ii < ib && jj < jb && (bi < bj || ii <= jj)) P.G[(i0 + ii) + (long)(j0 + jj) * ld] = c[e] - acc[e];
        }
      }
    }
    if (!grid_sync(P.bar, P.err)) return;
  }
  const long total = (long)n * n;
  for (long f = blockIdx.x * (long)CT + tid; f < total; f += (long)gridDim.x * CT) {
    const int i = (int)(f % n), j = (int)(f / n);
    if (i > j) P.G[i + (long)j * ld] = 0.0;
  }
}

constexpr int LT = 1024;   // threads of the cooperative sign-recovery LU (one row each)

struct LuArgs {
  int rows, cols;
  double* A;
  long lda;
  double* d;
  unsigned* bar;
  int* err;
};

// The sign-recovery elimination (lu_sign_leaf_reg) on the 16-column panel at
// p0, rows p0.. in registers, one row per thread.  The pivot row and its
// multiplier scale go through two shared buffers used alternately, so each
// column needs one CTA barrier: the row written at step j + 1 goes to the
// buffer read at step j - 1, which every thread left before step j's barrier.
__device__ void lu_panel(const LuArgs& P, int p0, double (*rowj)[LB], double* sf) {
  const int pb = min(LB, P.cols - p0);
  const int i = p0 + threadIdx.x;
  const bool live = i < P.rows;
  double x[LB];
#pragma unroll
  for (int c = 0; c < LB; ++c) x[c] = (live && c < pb) ? P.A[i + (long)(p0 + c) * P.lda] : 0.0;
#pragma unroll
  for (int j = 0; j < LB; ++j) {
    if (j < pb) {
      const int b = j & 1;
      if ((int)threadIdx.x == j) {
#pragma unroll
        for (int c = 0; c < LB; ++c) rowj[b][c] = x[c];
        const double cj = x[j];
        const double dj = cj < 0.0 ? 1.0 : -1.0;
        P.d[p0 + j] = dj;
        sf[b] = -dj / (1.0 + fabs(cj));
      }
      __syncthreads();
      if ((int)threadIdx.x > j && live) {
        const double l = sf[b] * x[j];
        x[j] = l;
#pragma unroll
        for (int c = j + 1; c < LB; ++c) x[c] -= l * rowj[b][c];
      }
    }
  }
  if (live)
#pragma unroll
    for (int c = 0; c < LB; ++c)
      if (c < pb) P.A[i + (long)(p0 + c) * P.lda] = x[c];
}

// Right-looking blocked elimination with 16-column panels: per panel, every
// CTA takes 16-column chunks of the trailing columns, solves their panel rows
// U12 = L11^-1 A12 and updates A22 -= L21 U12 (one row per thread); CTA 0
// owns the chunk of the next panel and factors it right after updating it,
// so one grid barrier per panel suffices.
__global__ void __launch_bounds__(LT, 1) lu_sign_coop_kernel(LuArgs P) {
  __shared__ double rowj[2][LB];
  __shared__ double sf[2];
  __shared__ double L11[LB][LB + 1];
  __shared__ double U[LB][LB + 1];
  const int np = (P.cols + LB - 1) / LB;
  if (blockIdx.x == 0) lu_panel(P, 0, rowj, sf);
  if (!grid_sync(P.bar, P.err)) return;
  for (int k = 0; k < np; ++k) {
    const int p0 = k * LB, pb = min(LB, P.cols - p0);
    const int nch = np - k - 1;   // trailing chunks
    if (nch > 0 && (int)blockIdx.x < nch) {
      for (int f = threadIdx.x; f < LB * LB; f += LT) {   // unit lower L11 of the panel
        const int r = f % LB, c = f / LB;
        L11[r][c] = (r > c && r < pb && c < pb) ? P.A[(p0 + r) + (long)(p0 + c) * P.lda] : 0.0;
      }
      // this thread's row of L21 (rows below the panel)
      const int i = p0 + pb + threadIdx.x;
      const bool live = i < P.rows;
      double l[LB];
#pragma unroll
      for (int t = 0; t < LB; ++t) l[t] = (live && t < pb) ? P.A[i + (long)(p0 + t) * P.lda] : 0.0;
      for (int q = blockIdx.x; q < nch; q += gridDim.x) {
        const int c0 = p0 + LB * (q + 1), cw = min(LB, P.cols - c0);
        __syncthreads();
        for (int f = threadIdx.x; f < LB * LB; f += LT) {   // the panel rows of the chunk
          const int r = f % LB, c = f / LB;
          U[r][c] = (c < cw && r < pb) ? P.A[(p0 + r) + (long)(c0 + c) * P.lda] : 0.0;
        }
        __syncthreads();
        if (threadIdx.x < LB) {   // U12 column c = L11^-1 A12 column c (unit lower, forward)
          const int c = threadIdx.x;
          for (int r = 1; r < pb; ++r) {
            double acc = U[r][c];
            for (int t = 0; t < r; ++t) acc -= L11[r][t] * U[t][c];
            U[r][c] = acc;
          }
          if (c < cw)
            for (int r = 0; r < pb; ++r) P.A[(p0 + r) + (long)(c0 + c) * P.lda] = U[r][c];
        }
        __syncthreads();
        if (live)   // eight columns at a time: their loads issued before any store
#pragma unroll
          for (int h = 0; h < LB; h += 8) {
            double a[8];
#pragma unroll
            for (int c = 0; c < 8; ++c) a[c] = (h + c < cw) ? P.A[i + (long)(c0 + h + c) * P.lda] : 0.0;
#pragma unroll
            for (int c = 0; c < 8; ++c) {
              double s = 0.0;
#pragma unroll
              for (int t = 0; t < LB; ++t) s = fma(l[t], U[t][h + c], s);
              if (h + c < cw) P.A[i + (long)(c0 + h + c) * P.lda] = a[c] - s;
            }
          }
      }
      __syncthreads();
    }
    if (blockIdx.x == 0 && k + 1 < np) lu_panel(P, p0 + LB, rowj, sf);   // CTA 0 updated that chunk (q = 0)
    if (!grid_sync(P.bar, P.err)) return;
  }
}

// Co-resident CTAs of a cooperative kernel: at most one per SM, at most `want`.
template <class K>
int coop_grid(bbt_ctx* ctx, K kernel, int threads, int want, size_t smem = 0) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess || per_sm < 1)
    return 0;
  return std::max(1, std::min(want, ctx->num_sms));
}

int split_point(int n) { return (n / 2 + TB - 1) / TB * TB; }

bbt_status trsm_left_lower_unit(bbt_ctx* ctx, int n, long ncols, const double* L, long ldl, double* B, long ldb) {
  if (n <= 0 || ncols <= 0) return BBT_OK;
  if (n > LB && vec_solve_fits(ncols, n)) {   // columns of B: x_j -= L(j, t) x_t
    ProfScope prof(ctx, BBT_PROF_CHOL, (double)ncols * n * n);
    BBT_CUDA(ctx, (vec_solve<false, true, true>(ctx, n, ncols, L, ldl, B, ldb, 1)));
    return BBT_OK;
  }
  if (n <= LB) {
    const long blocks = (ncols + 127) / 128;
    trsm_llu_leaf<<<(unsigned)blocks, 128, 0, ctx->stream>>>(n, ncols, L, ldl, B, ldb);
    BBT_LAUNCHED(ctx);
    return BBT_OK;
  }
  const int h = (n / 2 + LB - 1) / LB * LB;
  BBT_TRY(trsm_left_lower_unit(ctx, h, ncols, L, ldl, B, ldb));
  BBT_TRY(dgemm(ctx, false, false, n - h, (int)ncols, h, -1.0, L + h, ldl, B, ldb, 1.0, B + h, ldb));
  return trsm_left_lower_unit(ctx, n - h, ncols, L + h + (long)h * ldl, ldl, B + h, ldb);
}

}  // namespace

bbt_status householder_signs(bbt_ctx* ctx, int rows, int cols, double* A, long lda, double* d) {
  if (cols <= 0) return BBT_OK;
  if (ctx->allow_coop && cols > LB && rows >= cols && rows <= LT) {   // one cooperative launch
    const int grid = coop_grid(ctx, lu_sign_coop_kernel, LT, (cols + LB - 1) / LB - 1);
    if (grid > 0) {
      ProfScope prof(ctx, BBT_PROF_CHOL, (double)rows * cols * cols);
      LuArgs P{rows, cols, A, lda, d, ctx->d_barrier, ctx->d_flag + FLAG_SKETCH};
      BBT_CUDA(ctx, cudaMemsetAsync(ctx->d_barrier, 0, 2 * sizeof(unsigned), ctx->stream));
      void* args[] = {&P};
      BBT_CUDA(ctx, cudaLaunchCooperativeKernel((void*)lu_sign_coop_kernel, dim3(grid), dim3(LT), args, 0,
                                                ctx->stream));
      BBT_LAUNCHED(ctx);
      return BBT_OK;
    }
  }
  if (cols <= LB) {
    ProfScope prof(ctx, BBT_PROF_CHOL, (double)rows * cols * cols);
    if (rows <= 1024)
      lu_sign_leaf_reg<<<1, 1024, 0, ctx->stream>>>(rows, cols, A, lda, d);
    else
      lu_sign_leaf<<<1, 1024, 0, ctx->stream>>>(rows, cols, A, lda, d);
    BBT_LAUNCHED(ctx);
    return BBT_OK;
  }
  const int h = (cols / 2 + LB - 1) / LB * LB;   // a multiple of the leaf width, < cols
  BBT_TRY(householder_signs(ctx, rows, h, A, lda, d));
  BBT_TRY(trsm_left_lower_unit(ctx, h, cols - h, A, lda, A + (long)h * lda, lda));
  BBT_TRY(dgemm(ctx, false, false, rows - h, cols - h, h, -1.0, A + h, lda, A + (long)h * lda, lda, 1.0,
                A + h + (long)h * lda, lda));
  return householder_signs(ctx, rows - h, cols - h, A + h + (long)h * lda, lda, d + h);
}

bbt_status apply_signs(bbt_ctx* ctx, int m, const double* d, double* R, double* W) {
  apply_signs_kernel<<<2 * ctx->num_sms, 256, 0, ctx->stream>>>(m, d, R, W);
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

bbt_status trsm_right_upper(bbt_ctx* ctx, long rows, int n, const double* R, long ldr, double* A, long lda,
                            bool oz) {
  if (rows <= 0 || n <= 0) return BBT_OK;
  if (n > TB && vec_solve_fits(rows, n)) {   // rows of A: x_j -= R(t, j) x_t, / R(j, j)
    ProfScope prof(ctx, BBT_PROF_CHOL, (double)rows * n * n);
    BBT_CUDA(ctx, (vec_solve<true, true, false>(ctx, n, rows, R, ldr, A, 1, lda)));
    return BBT_OK;
  }
  if (n <= TB) {
    const long blocks = (rows + 127) / 128;
    ProfScope prof(ctx, BBT_PROF_CHOL, (double)rows * n * n);
    if (n <= 16)
      trsm_leaf<16><<<(unsigned)blocks, 128, 0, ctx->stream>>>(rows, n, R, ldr, A, lda);
    else
      trsm_leaf<TB><<<(unsigned)blocks, 128, 0, ctx->stream>>>(rows, n, R, ldr, A, lda);
    BBT_LAUNCHED(ctx);
    return BBT_OK;
  }
  const int n1 = split_point(n), n2 = n - n1;
  BBT_TRY(trsm_right_upper(ctx, rows, n1, R, ldr, A, lda, oz));
  if (oz && oz_worthwhile((int)rows, n2, n1))   // A2 -= A1 R12 from exact int8 slices (ozaki.cu)
    BBT_TRY(gemm_oz(ctx, (int)rows, n2, n1, -1.0, A, 1, lda, R + (long)n1 * ldr, ldr, 1, 1.0, A + (long)n1 * lda, lda,
                    false, false));
  else
    BBT_TRY(dgemm(ctx, false, false, (int)rows, n2, n1, -1.0, A, lda, R + (long)n1 * ldr, ldr, 1.0,
                  A + (long)n1 * lda, lda));
  return trsm_right_upper(ctx, rows, n2, R + n1 + (long)n1 * ldr, ldr, A + (long)n1 * lda, lda, oz);
}

bbt_status potrf_upper(bbt_ctx* ctx, int n, double* G, long ld, int* flag) {
  if (n <= 0) return BBT_OK;
  if (ctx->allow_coop && n > PB && n <= 4096) {   // one cooperative launch
    const int nb = (n + 31) / 32;
    static bool attr = false;
    if (!attr) {
      BBT_CUDA(ctx, cudaFuncSetAttribute(potrf_coop_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)POTRF_SMEM));
      attr = true;
    }
    const int grid = coop_grid(ctx, potrf_coop_kernel, CT, nb * (nb - 1) / 2, POTRF_SMEM);
    if (grid >= nb - 1) {   // one CTA per tile of every row panel
      ProfScope prof(ctx, BBT_PROF_CHOL, (double)n * n * n / 3.0);
      PotrfArgs P{n, G, ld, flag, ctx->d_barrier, ctx->d_flag + FLAG_SKETCH};
      BBT_CUDA(ctx, cudaMemsetAsync(ctx->d_barrier, 0, 2 * sizeof(unsigned), ctx->stream));
      void* args[] = {&P};
      BBT_CUDA(ctx, cudaLaunchCooperativeKernel((void*)potrf_coop_kernel, dim3(grid), dim3(CT), args, POTRF_SMEM,
                                                ctx->stream));
      BBT_LAUNCHED(ctx);
      return BBT_OK;
    }
  }
  if (n <= PB) {
    ProfScope prof(ctx, BBT_PROF_CHOL, (double)n * n * n / 3.0);
    potrf_leaf<<<1, 32, 0, ctx->stream>>>(n, G, ld, flag);
    BBT_LAUNCHED(ctx);
    return BBT_OK;
  }
  const int n1 = split_point(n), n2 = n - n1;
  BBT_TRY(potrf_upper(ctx, n1, G, ld, flag));
  BBT_TRY(trsm_right_upper(ctx, n2, n1, G, ld, G + n1, ld));   // G21 <- G21 R11^{-1} = R12^T
  BBT_TRY(dgemm(ctx, false, true, n2, n2, n1, -1.0, G + n1, ld, G + n1, ld, 1.0, G + n1 + (long)n1 * ld, ld));
  BBT_TRY(potrf_upper(ctx, n2, G + n1 + (long)n1 * ld, ld, flag));
  mirror_kernel<<<2 * ctx->num_sms, 256, 0, ctx->stream>>>(n1, n2, G, ld);
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

bbt_status shift_diag(bbt_ctx* ctx, int n, double* G, long ld, double rel) {
  shift_diag_kernel<<<1, 256, 0, ctx->stream>>>(n, G, ld, rel);
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

bbt_status symmetrize_upper(bbt_ctx* ctx, int n, double* G, long ld) {
  symmetrize_kernel<<<2 * ctx->num_sms, 256, 0, ctx->stream>>>(n, G, ld);
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

bbt_status identity(bbt_ctx* ctx, int n, double* W, long ld) {
  identity_kernel<<<2 * ctx->num_sms, 256, 0, ctx->stream>>>(n, W, ld);
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

}  // namespace bbt
