// FP64 GEMM on the FP64 tensor path (DMMA, mma.sync m8n8k4 .f64).
//
// Column-major BLAS convention: C = alpha * op(A) op(B) + beta * C with
// op(A) M x K and op(B) K x N.  A CTA computes a 128 x 64 tile of C with
// 8 warps (4 x 2), each warp a 32 x 32 block as 4 x 4 m8n8k4 fragments;
// K advances 16 at a time through double-buffered shared-memory tiles
// (register-staged global loads overlap the tensor work of the previous
// tile).  For the tall-skinny shapes of Householder QR (K up to 10^6,
// M*N small) K is split across CTAs; the partial tiles are summed in a
// fixed order by a second kernel so results are deterministic.
#include <cuda_runtime.h>

#include "internal.h"

namespace bbt {
namespace {

constexpr int BK = 16;
constexpr int PADA = 4, PADB = 4;   // row strides = 4 (mod 16) doubles: conflict-free fragment loads

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// WM x WN warps, each a 32 x 32 block of C: CTA tile (32 WM) x (32 WN).
template <bool TA, bool TB, int WM, int WN>
__global__ void __launch_bounds__(32 * WM * WN)
dgemm_kernel(int M, int N, long K, long kchunk, double alpha, const double* __restrict__ A, long lda,
             const double* __restrict__ B, long ldb, double beta, double* __restrict__ C, long ldc,
             double* __restrict__ P, int nfast) {
  constexpr int BM = 32 * WM, BN = 32 * WN, THREADS = 32 * WM * WN;
  // nfast bit 0: blockIdx.x walks the N tiles, so the CTAs that share a
  // block of rows of A run together and read it from HBM once (tall A,
  // narrow C).  Bit 1: only tiles touching the upper triangle of C are
  // computed (symmetric products A^T A; the caller mirrors the rest).
  const int nf = nfast & 1;
  const int bm = nf ? blockIdx.y : blockIdx.x, bn = nf ? blockIdx.x : blockIdx.y;
  extern __shared__ double smem_[];
  auto As = reinterpret_cast<double(*)[BK][BM + PADA]>(smem_);
  auto Bs = reinterpret_cast<double(*)[BK][BN + PADB]>(smem_ + 2 * BK * (BM + PADA));
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp % WM, wn = warp / WM;
  const int i0 = bm * BM, j0 = bn * BN;
  if ((nfast & 2) && i0 >= j0 + BN) return;   // entirely below the diagonal
  const long kbeg = (long)blockIdx.z * kchunk;
  const long kend = min(K, kbeg + kchunk);

  double acc[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;

  double ra[BM * BK / THREADS];   // 8
  double rb[BN * BK / THREADS];   // 4

  auto load = [&](long k0) {
#pragma unroll
    for (int r = 0; r < BM * BK / THREADS; ++r) {
      const int e = tid + r * THREADS;
      int il, kl;
      if (TA) { kl = e % BK; il = e / BK; } else { il = e % BM; kl = e / BM; }
      const int i = i0 + il;
      const long k = k0 + kl;
      double v = 0.0;
      if (i < M && k < kend) v = TA ? A[k + (long)i * lda] : A[(long)i + k * lda];
      ra[r] = v;
    }
#pragma unroll
    for (int r = 0; r < BN * BK / THREADS; ++r) {
      const int e = tid + r * THREADS;
      int jl, kl;
      if (TB) { jl = e % BN; kl = e / BN; } else { kl = e % BK; jl = e / BK; }
      const int j = j0 + jl;
      const long k = k0 + kl;
      double v = 0.0;
      if (j < N && k < kend) v = TB ? B[(long)j + k * ldb] : B[k + (long)j * ldb];
      rb[r] = v;
    }
  };
  auto store = [&](int buf) {
#pragma unroll
    for (int r = 0; r < BM * BK / THREADS; ++r) {
      const int e = tid + r * THREADS;
      int il, kl;
      if (TA) { kl = e % BK; il = e / BK; } else { il = e % BM; kl = e / BM; }
      As[buf][kl][il] = ra[r];
    }
#pragma unroll
    for (int r = 0; r < BN * BK / THREADS; ++r) {
      const int e = tid + r * THREADS;
      int jl, kl;
      if (TB) { jl = e % BN; kl = e / BN; } else { kl = e % BK; jl = e / BK; }
      Bs[buf][kl][jl] = rb[r];
    }
  };

  if (kbeg < kend) {
    load(kbeg);
    store(0);
    __syncthreads();
    int buf = 0;
    for (long k0 = kbeg; k0 < kend; k0 += BK) {
      const bool more = k0 + BK < kend;
      if (more) load(k0 + BK);
#pragma unroll
      for (int ks = 0; ks < BK; ks += 4) {
        double af[4], bf[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          af[t] = As[buf][ks + (lane & 3)][wm * 32 + t * 8 + (lane >> 2)];
          bf[t] = Bs[buf][ks + (lane & 3)][wn * 32 + t * 8 + (lane >> 2)];
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) dmma(acc[a][b][0], acc[a][b][1], af[a], bf[b]);
      }
      if (more) {
        store(buf ^ 1);
        __syncthreads();
        buf ^= 1;
      }
    }
  }

  // epilogue: fragment (a,b) element e at row wm*32+a*8+lane/4, col wn*32+b*8+2*(lane%4)+e
  double* out = P ? P + (long)blockIdx.z * M * (long)N : C;
  const long ldo = P ? M : ldc;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int i = i0 + wm * 32 + a * 8 + (lane >> 2);
    if (i >= M) continue;
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int j = j0 + wn * 32 + b * 8 + 2 * (lane & 3) + e;
        if (j >= N) continue;
        double* c = out + i + (long)j * ldo;
        const double v = alpha * acc[a][b][e];
        if (P || beta == 0.0) *c = v;
        else *c = v + beta * (*c);
      }
  }
}

// C = beta*C + sum_z P[z] in order z = 0..S-1.
__global__ void splitk_reduce(int M, int N, int S, const double* __restrict__ P, double beta,
                              double* __restrict__ C, long ldc) {
  const long total = (long)M * N;
  for (long f = blockIdx.x * (long)blockDim.x + threadIdx.x; f < total; f += (long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int z = 0; z < S; ++z) s += P[(long)z * total + f];
    const int i = (int)(f % M);
    const long j = f / M;
    double* c = C + i + j * ldc;
    *c = (beta == 0.0) ? s : s + beta * (*c);
  }
}

template <int WM, int WN>
constexpr int smem_bytes() { return 2 * BK * (32 * WM + PADA + 32 * WN + PADB) * (int)sizeof(double); }

template <bool TA, bool TB, int WM, int WN>
cudaError_t launch(dim3 g, cudaStream_t st, int M, int N, long K, long kc, double alpha, const double* A,
                   long lda, const double* B, long ldb, double beta, double* C, long ldc, double* P, int nfast) {
  static bool attr = false;   // set once per process (per kernel instantiation)
  constexpr int SM = smem_bytes<WM, WN>();
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(dgemm_kernel<TA, TB, WM, WN>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, SM);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  dgemm_kernel<TA, TB, WM, WN><<<g, 32 * WM * WN, SM, st>>>(M, N, K, kc, alpha, A, lda, B, ldb, beta, C, ldc, P,
                                                             nfast);
  return cudaSuccess;
}

template <int WM, int WN>
cudaError_t launch_t(bool ta, bool tb, dim3 g, cudaStream_t st, int M, int N, long K, long kc, double alpha,
                     const double* A, long lda, const double* B, long ldb, double beta, double* C, long ldc,
                     double* P, int nf) {
  if (!ta && !tb) return launch<false, false, WM, WN>(g, st, M, N, K, kc, alpha, A, lda, B, ldb, beta, C, ldc, P, nf);
  if (ta && !tb) return launch<true, false, WM, WN>(g, st, M, N, K, kc, alpha, A, lda, B, ldb, beta, C, ldc, P, nf);
  if (!ta && tb) return launch<false, true, WM, WN>(g, st, M, N, K, kc, alpha, A, lda, B, ldb, beta, C, ldc, P, nf);
  return launch<true, true, WM, WN>(g, st, M, N, K, kc, alpha, A, lda, B, ldb, beta, C, ldc, P, nf);
}

// Tile shape from the output shape: avoid computing padding rows/columns of
// small outputs (the V^T C products of Householder QR have 16..128 rows).
void pick_tile(int M, int N, int* wm, int* wn) {
  if (M <= 32) { *wm = 1; *wn = 4; }
  else if (M <= 64) { *wm = 2; *wn = N <= 64 ? 2 : 4; }
  else { *wm = 4; *wn = 2; }
}

}  // namespace

size_t dgemm_workspace_bytes(const bbt_ctx* ctx, int M, int N, long K) {
  if (M <= 0 || N <= 0) return 0;
  int wm, wn;
  pick_tile(M, N, &wm, &wn);
  const long tiles = (long)((M + 32 * wm - 1) / (32 * wm)) * ((N + 32 * wn - 1) / (32 * wn));
  const long target = 2L * ctx->num_sms;
  if (!(tiles < target && K >= 2048)) return 0;
  long s = (target + tiles - 1) / tiles;
  if (s > K / 1024) s = K / 1024;
  if (s > 256) s = 256;
  return s > 1 ? (size_t)s * M * N * sizeof(double) + 256 : 0;
}

bbt_status dgemm(bbt_ctx* ctx, bool ta, bool tb, int M, int N, long K, double alpha, const double* A,
                 long lda, const double* B, long ldb, double beta, double* C, long ldc, int splits, bool upper) {
  if (M < 0 || N < 0 || K < 0) return fail(ctx, BBT_ERR_ARG, "dgemm: M=%d N=%d K=%ld", M, N, K);
  if (M == 0 || N == 0) return BBT_OK;
  int wm, wn;
  pick_tile(M, N, &wm, &wn);
  const int BM = 32 * wm, BN = 32 * wn;
  const int tm = (M + BM - 1) / BM, tn = (N + BN - 1) / BN;
  if (splits <= 0) {
    const long tiles = (long)tm * tn;
    const long target = 2L * ctx->num_sms;
    splits = 1;
    if (tiles < target && K >= 2048) {
      long s = (target + tiles - 1) / tiles;
      const long maxs = K / 1024;
      if (s > maxs) s = maxs;
      if (s > 256) s = 256;
      splits = (int)(s < 1 ? 1 : s);
    }
  }
  long kc = (K + splits - 1) / splits;
  kc = ((kc + BK - 1) / BK) * BK;
  if (kc == 0) kc = BK;
  splits = (int)((K + kc - 1) / kc);
  if (splits < 1) splits = 1;
  double* P = nullptr;
  size_t mark = ctx->ws.top;
  if (splits > 1) {
    P = ctx->ws.take<double>((size_t)splits * M * N);
    if (!P) return fail(ctx, BBT_ERR_NOMEM, "dgemm: split-K workspace (%d x %d x %d)", splits, M, N);
  }
  const int nfast = ((tm >= tn && tm <= 65535) ? 1 : 0) | (upper ? 2 : 0);
  dim3 g((nfast & 1) ? tn : tm, (nfast & 1) ? tm : tn, splits);
  if (K == 0) {   // C = beta * C
    g.z = 1;
    P = nullptr;
  }
  cudaError_t e;
  ProfScope prof(ctx, BBT_PROF_DGEMM, 2.0 * M * (double)N * (double)K);
  if (wm == 1) e = launch_t<1, 4>(ta, tb, g, ctx->stream, M, N, K, kc, alpha, A, lda, B, ldb, beta, C, ldc, P, nfast);
  else if (wm == 2 && wn == 2) e = launch_t<2, 2>(ta, tb, g, ctx->stream, M, N, K, kc, alpha, A, lda, B, ldb, beta, C, ldc, P, nfast);
  else if (wm == 2) e = launch_t<2, 4>(ta, tb, g, ctx->stream, M, N, K, kc, alpha, A, lda, B, ldb, beta, C, ldc, P, nfast);
  else e = launch_t<4, 2>(ta, tb, g, ctx->stream, M, N, K, kc, alpha, A, lda, B, ldb, beta, C, ldc, P, nfast);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "dgemm: shared-memory attribute");
  BBT_LAUNCHED(ctx);
  if (P) {
    splitk_reduce<<<4 * ctx->num_sms, 256, 0, ctx->stream>>>(M, N, splits, P, beta, C, ldc);
    BBT_LAUNCHED(ctx);
  }
  ctx->ws.top = mark;
  return BBT_OK;
}

}  // namespace bbt
