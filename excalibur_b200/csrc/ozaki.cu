// FP64-accurate GEMM from exact int8 slices on the 5th-generation tensor
// cores (the Ozaki scheme), for the large FP64 products of the
// mixed-precision path: the Gram matrix and the triangular-solve updates of
// the Cholesky-QR refinement, and the V back-transform.
//
//   C (M x N, column-major) = alpha * A B^T + beta * C,
//   A(i, k) = A[i * rsA + k * csA]  (M x K),   B(j, k) = B[j * rsB + k * csB]  (N x K).
//
// Each row of A (of B) is scaled by a power of two s_i (t_j) so that
// |a / s_i| < 1/2, then split exactly into OS = 8 slices by rounding to
// nearest: a / s_i = sum_p q_p 2^-7(p+1) + (a remainder of at most 2^-57),
// q_p in [-64, 64] (unbiased, so the slicing errors of a long sum cancel
// instead of adding up).  Slice products are exact int8 x int8 -> int32 tensor-core
// MMAs (kind::i8); all pairs with p + q = t share the int32 accumulator t
// (scale 2^-7(t+2)); pairs with p + q >= OS are dropped (below 2^-56 of the
// row and column scales).  So
//   C(i, j) = s_i t_j sum_{t < OS} 2^-7(t+2) acc_t(i, j),
// accurate to about 2^-56 |a_i| |b_j| per term -- FP64 level.
//
// Kernel (one CTA = 320 threads per 128 x 64 output tile, 1 CTA per SM):
//   warp 8, one lane : TMA producer -- per K-block of 64, the S A-slice
//                      tiles (128 x 64 B) and the S B-slice tiles (64 x 64 B),
//                      SWIZZLE_64B, into a 2-stage ring (96 KB per stage at
//                      S = 8);
//   warp 9, one lane : tcgen05.mma issuer -- two 128 x 64 x 32 MMAs per slice
//                      pair (S (S+1) / 2 pairs) into S TMEM accumulators
//                      (8 x 64 = all 512 columns at S = 8);
//   warps 0-7        : every DRAIN K-blocks (before an int32 accumulator can
//                      overflow: 8 pairs x 8192 x 64^2 < 2^31) they read
//                      the 8 accumulators and add them, scaled, into 32 FP64
//                      registers per thread; at the end the FP64 tile is
//                      scaled by s_i t_j, alpha, beta and written.
// Every mbarrier wait is bounded; a wait that gives up sets an error flag.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "internal.h"
#include "tc.cuh"

namespace bbt {
namespace {

using namespace tc;

constexpr int OS = 8;
constexpr int TM = 128, TN = 64, TK = 64;
constexpr int STAGES = 2;
constexpr int A_SL = TM * TK, B_SL = TN * TK;
constexpr int STAGE_BYTES = OS * (A_SL + B_SL);
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;
constexpr int EPI_WARPS = 8;
constexpr int THREADS = (EPI_WARPS + 2) * 32;
constexpr uint32_t TMEM_COLS = OS * TN;   // 512
constexpr int DRAIN = 128;   // K-blocks of 64: 8192 terms
constexpr int MAX_SPLITS = 32;

struct OzArgs {
  double* out;          // C (ldo) or split partials [z][N][M] (ldo = M)
  long ldo;
  int M, N;
  int kblocks, kb_per_split;
  const double* sa;     // M row scales of A
  const double* sb;     // N row scales of B
  double alpha, beta;
  int partial;          // 1: write s_i t_j sum (no alpha, beta) to partial z
  int upper;            // 1: skip tiles strictly below the diagonal
  int S;                // slices used per operand (pairs p + q < S)
  int* err;
};

__global__ void __launch_bounds__(THREADS, 1)
oz_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, OzArgs P) {
  const int n0 = blockIdx.x * TN, m0 = blockIdx.y * TM;
  if (P.upper && m0 >= n0 + TN) return;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* bars = (uint64_t*)(smem + STAGES * STAGE_BYTES);
  uint32_t* tmem_slot = (uint32_t*)(bars + 2 * STAGES + 2);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int kb0 = blockIdx.z * P.kb_per_split;
  const int nk = min(P.kblocks - kb0, P.kb_per_split);
  const int ngroups = (nk + DRAIN - 1) / DRAIN;
  const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + STAGES);
  const uint32_t accf = smem_u32(bars + 2 * STAGES), acce = smem_u32(bars + 2 * STAGES + 1);
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    mbar_init(accf, 1);
    mbar_init(acce, EPI_WARPS);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == EPI_WARPS) {
    if (lane == 0) {   // ---- TMA producer
      int issued = 0;
      bool ok = true;
      for (int kb = 0; kb < nk; ++kb) {
        const int s = kb % STAGES;
        const uint32_t ph = (uint32_t)(kb / STAGES) & 1u;
        if (!mbar_wait(empty0 + 8 * s, ph ^ 1u)) { ok = false; break; }
        const uint32_t fb = full0 + 8 * s;
        mbar_expect_tx(fb, (uint32_t)(P.S * (A_SL + B_SL)));
        const uint32_t st = smem_u32(smem + (size_t)s * STAGE_BYTES);
        const int kx = (kb0 + kb) * TK;
        for (int p = 0; p < P.S; ++p) tma_load_3d(st + p * A_SL, &tmA, fb, kx, m0, p);
        for (int q = 0; q < P.S; ++q) tma_load_3d(st + OS * A_SL + q * B_SL, &tmB, fb, kx, n0, q);
        ++issued;
      }
      if (!ok) atomicExch(P.err, 1);
      for (int kb = max(0, issued - STAGES); kb < issued; ++kb)
        if (!mbar_wait(full0 + 8 * (kb % STAGES), (uint32_t)(kb / STAGES) & 1u)) atomicExch(P.err, 4);
    }
  } else if (warp == EPI_WARPS + 1) {
    if (lane == 0) {   // ---- MMA issuer: int8 x int8 -> int32 (c_format S32, a/b INT8, K-major)
      const uint32_t idesc =
          (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);
      bool ok = true;
      for (int g = 0; g < ngroups && ok; ++g) {
        if (!mbar_wait(acce, ((uint32_t)g & 1u) ^ 1u)) { ok = false; break; }
        tc_fence_after();
        const int kbeg = g * DRAIN, kend = min(nk, kbeg + DRAIN);
        for (int kb = kbeg; kb < kend; ++kb) {
          const int s = kb % STAGES;
          const uint32_t ph = (uint32_t)(kb / STAGES) & 1u;
          if (!mbar_wait(full0 + 8 * s, ph)) { ok = false; break; }
          tc_fence_after();
          const uint32_t st = smem_u32(smem + (size_t)s * STAGE_BYTES);
#pragma unroll 1
          for (int t = 0; t < P.S; ++t) {
            const uint32_t d = tmem + (uint32_t)(t * TN);
            for (int p = 0; p <= t; ++p) {
              const uint64_t ad = sw64_desc(st + p * A_SL);
              const uint64_t bd = sw64_desc(st + OS * A_SL + (t - p) * B_SL);
              mma_i8(d, ad, bd, idesc, (kb != kbeg || p != 0) ? 1u : 0u);
              mma_i8(d, ad + 2, bd + 2, idesc, 1u);   // second 32-byte K slice of the 64-byte rows
            }
          }
          mma_commit(empty0 + 8 * s);
        }
        mma_commit(accf);
      }
      if (!ok) atomicExch(P.err, 2);
    }
  } else {
    // ---- accumulators: TMEM lanes 32 (warp % 4).., columns 32 (warp / 4).. of each accumulator
    const int q4 = warp & 3, ch = warp >> 2;
    double acc[32];
#pragma unroll
    for (int c = 0; c < 32; ++c) acc[c] = 0.0;
    bool ok = true;
    for (int g = 0; g < ngroups; ++g) {
      if (!mbar_wait(accf, (uint32_t)g & 1u)) { ok = false; break; }
      tc_fence_after();
#pragma unroll 1
      for (int t = 0; t < P.S; ++t) {
        const uint32_t base = tmem + ((uint32_t)(q4 * 32) << 16) + (uint32_t)(t * TN + ch * 32);
        const double sc = ldexp(1.0, -7 * (t + 2));
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          uint32_t v[16];
          tmem_ld16(base + (uint32_t)(h * 16), v);
#pragma unroll
          for (int i = 0; i < 16; ++i) acc[h * 16 + i] += sc * (double)(int)v[i];
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acce);
    }
    if (!ok) {
      if (lane == 0) atomicExch(P.err, 3);
    } else {
      const int i = m0 + q4 * 32 + lane;
      if (i < P.M) {
        const double si = P.sa[i];
        double* o = P.out + (P.partial ? (size_t)blockIdx.z * P.M * (size_t)P.N : 0);
#pragma unroll
        for (int c = 0; c < 32; ++c) {
          const int j = n0 + ch * 32 + c;
          if (j < P.N) {
            const double v = acc[c] * si * P.sb[j];
            double* dst = o + i + (long)j * P.ldo;
            if (P.partial) *dst = v;
            else *dst = (P.beta == 0.0) ? P.alpha * v : P.alpha * v + P.beta * (*dst);
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
  }
}

// Row scales and slices of a strided operand X(i, k) = X[i * rs + k * cs]
// (rows x K): s_i = 2^(e+1) with max_k |X(i, k)| in [2^(e-1), 2^e); slices
// out[p][i][k] (row pitch Kp), exact.  Rows contiguous in k (cs == 1): one
// warp per row.
__device__ __forceinline__ void slice8(double r, int8_t* q) {   // |r| < 1/2
#pragma unroll
  for (int p = 0; p < OS; ++p) {
    r *= 128.0;
    const double t = rint(r);
    q[p] = (int8_t)(int)t;
    r -= t;
  }
}

// Row maxima of a row-contiguous operand: blocks of 256 threads over
// (row, chunk of 8192 columns); the maximum of non-negative doubles is the
// maximum of their bit patterns, so chunks combine by atomicMax.
__global__ void rowmax_kernel(int rows, long K, const double* __restrict__ X, long rs,
                              unsigned long long* __restrict__ mx) {
  const int i = blockIdx.y;
  const long k0 = (long)blockIdx.x * 8192;
  const double* x = X + (long)i * rs;
  double m = 0.0;
  for (long k = k0 + threadIdx.x; k < K && k < k0 + 8192; k += blockDim.x) m = fmax(m, fabs(x[k]));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ double sh[8];
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, sh[w]);
    m = fmax(m, sh[0]);
    atomicMax(mx + i, (unsigned long long)__double_as_longlong(m));
  }
}

__global__ void scale_kernel(int rows, const unsigned long long* __restrict__ mx, double* __restrict__ scale) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows) return;
  const double m = __longlong_as_double((long long)mx[i]);
  int e = 0;
  if (m > 0.0) frexp(m, &e);
  scale[i] = ldexp(1.0, e + 1);
}

// Slices of a row-contiguous operand, one thread per 4 consecutive elements.
__global__ void slice_rows_kernel(int rows, long K, const double* __restrict__ X, long rs, int8_t* __restrict__ out,
                                  long Kp, const double* __restrict__ scale) {
  const long kq = (K + 3) / 4;
  const long total = (long)rows * kq;
  const size_t plane = (size_t)rows * Kp;
  for (long f = blockIdx.x * (long)blockDim.x + threadIdx.x; f < total; f += (long)gridDim.x * blockDim.x) {
    const int i = (int)(f / kq);
    const long k = (f - (long)i * kq) * 4;
    const double inv = 1.0 / scale[i];   // a power of two: exact
    const double* x = X + (long)i * rs + k;
    uint32_t w[OS];
#pragma unroll
    for (int p = 0; p < OS; ++p) w[p] = 0;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if (k + e < K) {
        int8_t q[OS];
        slice8(x[e] * inv, q);
#pragma unroll
        for (int p = 0; p < OS; ++p) w[p] |= (uint32_t)(uint8_t)q[p] << (8 * e);
      }
    }
    if (k + 4 <= K) {
#pragma unroll
      for (int p = 0; p < OS; ++p) *reinterpret_cast<uint32_t*>(out + p * plane + (size_t)i * Kp + k) = w[p];
    } else {
      for (int e = 0; k + e < K; ++e)
#pragma unroll
        for (int p = 0; p < OS; ++p) out[p * plane + (size_t)i * Kp + k + e] = (int8_t)(w[p] >> (8 * e));
    }
  }
}

// Rows contiguous in i (rs == 1, column stride cs): 32 rows per block, staged
// through shared memory so both the reads and the slice writes are coalesced.
__global__ void __launch_bounds__(256) slice_cols_kernel(int rows, long K, const double* __restrict__ X, long cs,
                                                         int8_t* __restrict__ out, long Kp,
                                                         double* __restrict__ scale) {
  __shared__ double tile[32][33];
  __shared__ double red[8][32];
  __shared__ double inv[32];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int i0 = blockIdx.x * 32;
  const int i = i0 + tx;
  double mx = 0.0;
  if (i < rows)
    for (long k = ty; k < K; k += 8) mx = fmax(mx, fabs(X[i + k * cs]));
  red[ty][tx] = mx;
  __syncthreads();
  if (ty == 0) {
    double m = red[0][tx];
    for (int r = 1; r < 8; ++r) m = fmax(m, red[r][tx]);
    int e = 0;
    if (m > 0.0) frexp(m, &e);
    inv[tx] = ldexp(1.0, -(e + 1));
    if (i < rows) scale[i] = ldexp(1.0, e + 1);
  }
  __syncthreads();
  const size_t plane = (size_t)rows * Kp;
  for (long k0 = 0; k0 < K; k0 += 32) {
    for (int r = ty; r < 32; r += 8) {   // tile[k][row]
      const long k = k0 + r;
      tile[r][tx] = (i < rows && k < K) ? X[i + k * cs] : 0.0;
    }
    __syncthreads();
    const long k = k0 + tx;
    for (int r = ty; r < 32; r += 8) {
      const int ii = i0 + r;
      if (ii < rows && k < K) {
        int8_t q[OS];
        slice8(tile[tx][r] * inv[r], q);
#pragma unroll
        for (int p = 0; p < OS; ++p) out[p * plane + (size_t)ii * Kp + k] = q[p];
      }
    }
    __syncthreads();
  }
}

__global__ void oz_reduce(int M, int N, int S, const double* __restrict__ P, double alpha, double beta,
                          double* __restrict__ C, long ldc, int upper) {
  const long total = (long)M * N;
  for (long f = blockIdx.x * (long)blockDim.x + threadIdx.x; f < total; f += (long)gridDim.x * blockDim.x) {
    const int i = (int)(f % M);
    const long j = f / M;
    if (upper && (i / TM) * TM >= (j / TN) * TN + TN) continue;   // tile never computed
    double s = 0.0;
    for (int z = 0; z < S; ++z) s += P[(long)z * total + f];
    double* c = C + i + j * ldc;
    *c = (beta == 0.0) ? alpha * s : alpha * s + beta * (*c);
  }
}

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn() {
  static EncodeTiled fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(p);
  }
  return fn;
}

long pitch16(long K) { return (K + 15) / 16 * 16; }

struct Plan {
  int splits, kb_per_split, kblocks;
};

Plan plan(int M, int N, long K, int num_sms, bool upper) {
  Plan r;
  r.kblocks = (int)((K + TK - 1) / TK);
  const long tm = (M + TM - 1) / TM, tn = (N + TN - 1) / TN;
  long tiles = tm * tn;
  if (upper) {   // tiles that touch the upper triangle
    tiles = 0;
    for (long a = 0; a < tm; ++a)
      for (long b = 0; b < tn; ++b) tiles += (a * TM < b * TN + TN);
  }
  double best = 1e300;
  int bs = 1;
  const int smax = std::min(MAX_SPLITS, r.kblocks);
  std::vector<double> cost(smax + 1);
  for (int s = 1; s <= smax; ++s) {
    const long waves = (tiles * s + num_sms - 1) / num_sms;
    cost[s] = (double)waves * ((r.kblocks + s - 1) / s) + 4.0 * s;   // + the partial write/reduce per split
    best = std::min(best, cost[s]);
  }
  for (int s = 1; s <= smax; ++s)
    if (cost[s] <= 1.02 * best) { bs = s; break; }
  r.kb_per_split = (r.kblocks + bs - 1) / bs;
  r.splits = (r.kblocks + r.kb_per_split - 1) / r.kb_per_split;
  return r;
}

bbt_status slices(bbt_ctx* ctx, int rows, long K, const double* X, long rs, long cs, int8_t* out, long Kp,
                  double* scale) {
  if (cs == 1) {
    unsigned long long* mx = reinterpret_cast<unsigned long long*>(out);   // the slices' first bytes as scratch
    BBT_CUDA(ctx, cudaMemsetAsync(mx, 0, (size_t)rows * 8, ctx->stream));
    rowmax_kernel<<<dim3((unsigned)((K + 8191) / 8192), rows), 256, 0, ctx->stream>>>(rows, K, X, rs, mx);
    BBT_LAUNCHED(ctx);
    scale_kernel<<<(rows + 255) / 256, 256, 0, ctx->stream>>>(rows, mx, scale);
    BBT_LAUNCHED(ctx);
    slice_rows_kernel<<<16 * ctx->num_sms, 256, 0, ctx->stream>>>(rows, K, X, rs, out, Kp, scale);
  } else if (rs == 1) {
    slice_cols_kernel<<<(rows + 31) / 32, 256, 0, ctx->stream>>>(rows, K, X, cs, out, Kp, scale);
  } else {
    return fail(ctx, BBT_ERR_ARG, "ozaki: operand needs a unit stride");
  }
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

}  // namespace

// Row chunk of a product whose A slices exceed this many bytes (rows of C are
// independent; B's slices are formed again per chunk).
constexpr size_t OZ_CHUNK_DEFAULT = (size_t)6 << 30;
int oz_row_chunk(int M, long K) {
  const size_t cap = long_chunk_bytes(OZ_CHUNK_DEFAULT);
  const size_t per_row = (size_t)OS * pitch16(K);
  if ((size_t)M * per_row <= cap) return M;
  const long c = std::max(128L, (long)(cap / per_row) / 128 * 128);
  const long chunks = (M + c - 1) / c;
  return (int)(((M + chunks - 1) / chunks + 127) / 128 * 128);
}

size_t oz_workspace_bytes(const bbt_ctx* ctx, int M, int N, long K, bool same) {
  if (!same) M = oz_row_chunk(M, K);
  const long Kp = pitch16(K);
  const int sms = ctx->num_sms > 0 ? ctx->num_sms : 148;
  const int splits = std::max(plan(M, N, K, sms, false).splits, plan(M, N, K, sms, true).splits);
  size_t b = (size_t)OS * M * Kp + (same ? 0 : (size_t)OS * N * Kp) + (size_t)(M + N) * 8;
  if (splits > 1) b += (size_t)splits * M * N * 8;
  return b + 8192;
}

// Large products with K of at least 768 (measured: below that the per-tile
// overhead cancels the gain over the FP64 DMMA GEMM).
bool oz_worthwhile(int M, int N, long K) {
  return M >= 128 && N >= 64 && K >= 768 && (double)M * N * K >= 4e9;
}

namespace {
bbt_status gemm_oz_one(bbt_ctx* ctx, int M, int N, long K, double alpha, const double* A, long rsA, long csA,
                       const double* B, long rsB, long csB, double beta, double* C, long ldc, bool same, bool upper,
                       int S);
}  // namespace

bbt_status gemm_oz(bbt_ctx* ctx, int M, int N, long K, double alpha, const double* A, long rsA, long csA,
                   const double* B, long rsB, long csB, double beta, double* C, long ldc, bool same, bool upper,
                   int S) {
  if (S < 4 || S > OS) return fail(ctx, BBT_ERR_ARG, "ozaki: %d slices (4..8)", S);
  if (M < 1 || N < 1 || K < 1 || K > (1L << 31) - TK) return fail(ctx, BBT_ERR_ARG, "ozaki: M=%d N=%d K=%ld", M, N, K);
  if (!same && !upper) {   // a long A: row chunks of bounded slice scratch (rows of C are independent)
    const int rc = oz_row_chunk(M, K);
    for (long r0 = 0; r0 < M; r0 += rc)
      BBT_TRY(gemm_oz_one(ctx, (int)std::min<long>(rc, M - r0), N, K, alpha, A + r0 * rsA, rsA, csA, B, rsB, csB,
                          beta, C + r0, ldc, false, false, S));
    return BBT_OK;
  }
  return gemm_oz_one(ctx, M, N, K, alpha, A, rsA, csA, B, rsB, csB, beta, C, ldc, same, upper, S);
}

namespace {
bbt_status gemm_oz_one(bbt_ctx* ctx, int M, int N, long K, double alpha, const double* A, long rsA, long csA,
                       const double* B, long rsB, long csB, double beta, double* C, long ldc, bool same, bool upper,
                       int S) {
  EncodeTiled enc = encode_fn();
  if (!enc) return fail(ctx, BBT_ERR_CUDA, "ozaki: cuTensorMapEncodeTiled is not available");
  const long Kp = pitch16(K);
  const Plan pl = plan(M, N, K, ctx->num_sms, upper);
  const size_t mark = ctx->ws.top;
  int8_t* sA = ctx->ws.take<int8_t>((size_t)OS * M * Kp);
  int8_t* sB = same ? sA : ctx->ws.take<int8_t>((size_t)OS * N * Kp);
  double* scA = ctx->ws.take<double>(M);
  double* scB = same ? scA : ctx->ws.take<double>(N);
  double* part = pl.splits > 1 ? ctx->ws.take<double>((size_t)pl.splits * M * N) : nullptr;
  if (!scB || (pl.splits > 1 && !part)) return fail(ctx, BBT_ERR_NOMEM, "ozaki: workspace");
  BBT_TRY(slices(ctx, M, K, A, rsA, csA, sA, Kp, scA));
  if (!same) BBT_TRY(slices(ctx, N, K, B, rsB, csB, sB, Kp, scB));

  CUtensorMap ta, tb;
  {
    const cuuint64_t dims[3] = {(cuuint64_t)K, (cuuint64_t)M, (cuuint64_t)OS};
    const cuuint64_t strides[2] = {(cuuint64_t)Kp, (cuuint64_t)Kp * M};
    const cuuint32_t box[3] = {TK, TM, 1}, es[3] = {1, 1, 1};
    if (enc(&ta, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, sA, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return fail(ctx, BBT_ERR_CUDA, "ozaki: tensor map of A");
  }
  {
    const cuuint64_t dims[3] = {(cuuint64_t)K, (cuuint64_t)N, (cuuint64_t)OS};
    const cuuint64_t strides[2] = {(cuuint64_t)Kp, (cuuint64_t)Kp * N};
    const cuuint32_t box[3] = {TK, TN, 1}, es[3] = {1, 1, 1};
    if (enc(&tb, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, sB, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return fail(ctx, BBT_ERR_CUDA, "ozaki: tensor map of B");
  }
  static bool attr = false;
  if (!attr) {
    BBT_CUDA(ctx, cudaFuncSetAttribute(oz_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
    attr = true;
  }
  OzArgs a;
  a.out = part ? part : C;
  a.ldo = part ? M : ldc;
  a.M = M;
  a.N = N;
  a.kblocks = pl.kblocks;
  a.kb_per_split = pl.kb_per_split;
  a.sa = scA;
  a.sb = scB;
  a.alpha = alpha;
  a.beta = beta;
  a.partial = part ? 1 : 0;
  a.upper = upper ? 1 : 0;
  a.S = S;
  a.err = ctx->d_flag + FLAG_SKETCH;
  const unsigned gy = (unsigned)((M + TM - 1) / TM);
  if (gy > 65535) return fail(ctx, BBT_ERR_ARG, "ozaki: M=%d too large", M);
  {
    ProfScope prof(ctx, BBT_PROF_OZAKI, (upper ? 1.0 : 2.0) * (double)M * N * K);
    oz_kernel<<<dim3((N + TN - 1) / TN, gy, pl.splits), THREADS, SMEM_BYTES, ctx->stream>>>(ta, tb, a);
    BBT_LAUNCHED(ctx);
  }
  if (part) {
    oz_reduce<<<4 * ctx->num_sms, 256, 0, ctx->stream>>>(M, N, pl.splits, part, alpha, beta, C, ldc, upper ? 1 : 0);
    BBT_LAUNCHED(ctx);
  }
  ctx->ws.top = mark;
  return BBT_OK;
}
}  // namespace

}  // namespace bbt
