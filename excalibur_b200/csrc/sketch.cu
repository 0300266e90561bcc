// Split-precision (BF16x3) sketch product on the 5th-generation tensor cores.
//
//   Y^T (m x N, row-major FP64) = X (m x n, row-major FP64) * S^T,
//   S (N x n) a Rademacher (+-1) sketch held exactly in bf16.
//
// X is split into three bf16 pieces x0 + x1 + x2 (x0 = bf16(x), x1 =
// bf16(x - x0), x2 = bf16(x - x0 - x1): 24 significant bits), so that
// X S^T = x0 S^T + x1 S^T + x2 S^T with every product exact.  The tensor
// cores accumulate in FP32 (with truncation: the error grows with the number
// of accumulation steps), so the FP32 tile in tensor memory only ever holds
// GROUP = 4 K-blocks (256 terms); the epilogue warps then drain it into FP64
// registers while the MMAs fill the other half of a double-buffered
// accumulator.  K is split across CTAs only for parallelism; the FP64
// partial tiles are summed in a fixed order by a second kernel.
//
// Kernel structure (one CTA = 320 threads per 128 x 128 output tile):
//   warp 8, one lane : TMA producer -- per K-block of 64, the three 128 x 64
//                      bf16 tiles of x0/x1/x2 (one 3-D tensor map) and the
//                      128 x 64 tile of S, SWIZZLE_128B, into a 3-stage ring;
//   warp 9, one lane : tcgen05.mma issuer -- 3 pieces x 4 MMAs of
//                      128 x 128 x 16 (kind::f16, bf16 in, f32 accumulate)
//                      per K-block into TMEM buffer (group & 1);
//                      tcgen05.commit frees each stage and hands each full
//                      buffer to the epilogue;
//   warps 0-7        : accumulators -- warp w reads TMEM lanes 32 (w % 4)..
//                      and columns 64 (w / 4).., adds them to 64 FP64
//                      registers per thread, releases the buffer; at the end
//                      writes its 32 x 64 FP64 block of the partial tile.
// Every mbarrier wait is bounded; a wait that gives up sets an error flag
// and the CTA drains its copies, frees its tensor memory and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "internal.h"
#include "tc.cuh"

namespace bbt {
namespace {

using namespace tc;

constexpr int TM = 128, TN = 128, TK = 64;
constexpr int PIECES = 3;
constexpr int STAGES = 3;
constexpr int GROUP = 4;                                  // K-blocks per FP32 accumulation
constexpr int EPI_WARPS = 8;
constexpr int THREADS = (EPI_WARPS + 2) * 32;
constexpr int A_TILE = TM * TK * 2;                       // 16 KB
constexpr int B_TILE = TN * TK * 2;                       // 16 KB
constexpr int STAGE_BYTES = PIECES * A_TILE + B_TILE;     // 64 KB
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;
constexpr uint32_t TMEM_COLS = 2 * TN;
constexpr int MAX_SPLITS = 32;

struct SketchArgs {
  double* part;       // [splits][M][N]
  int M, N;
  int kblocks, kb_per_split;
  int* err;
};

__global__ void __launch_bounds__(THREADS, 1)
sketch_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, SketchArgs P) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* bars = (uint64_t*)(smem + STAGES * STAGE_BYTES);
  uint32_t* tmem_slot = (uint32_t*)(bars + 2 * STAGES + 4);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n0 = blockIdx.x * TN, m0 = blockIdx.y * TM;
  const int kb0 = blockIdx.z * P.kb_per_split;
  const int nk = min(P.kblocks - kb0, P.kb_per_split);
  const int ngroups = (nk + GROUP - 1) / GROUP;
  const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + STAGES);
  const uint32_t accf0 = smem_u32(bars + 2 * STAGES), acce0 = smem_u32(bars + 2 * STAGES + 2);
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(accf0 + 8 * b, 1);
      mbar_init(acce0 + 8 * b, EPI_WARPS);
    }
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
        mbar_expect_tx(fb, STAGE_BYTES);
        const uint32_t st = smem_u32(smem + (size_t)s * STAGE_BYTES);
        const int kx = (kb0 + kb) * TK;
        for (int p = 0; p < PIECES; ++p) tma_load_3d(st + p * A_TILE, &tmA, fb, kx, m0, p);
        tma_load_2d(st + PIECES * A_TILE, &tmB, fb, kx, n0);
        ++issued;
      }
      if (!ok) atomicExch(P.err, 1);
      // drain: every issued copy has landed before the CTA may exit
      for (int kb = max(0, issued - STAGES); kb < issued; ++kb)
        if (!mbar_wait(full0 + 8 * (kb % STAGES), (uint32_t)(kb / STAGES) & 1u)) atomicExch(P.err, 4);
    }
  } else if (warp == EPI_WARPS + 1) {
    if (lane == 0) {   // ---- MMA issuer
      const uint32_t idesc =
          (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);
      bool ok = true;
      for (int g = 0; g < ngroups && ok; ++g) {
        const int buf = g & 1;
        if (!mbar_wait(acce0 + 8 * buf, ((uint32_t)(g >> 1) & 1u) ^ 1u)) { ok = false; break; }
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(buf * TN);
        const int kend = min(nk, (g + 1) * GROUP);
        for (int kb = g * GROUP; kb < kend; ++kb) {
          const int s = kb % STAGES;
          const uint32_t ph = (uint32_t)(kb / STAGES) & 1u;
          if (!mbar_wait(full0 + 8 * s, ph)) { ok = false; break; }
          tc_fence_after();
          const uint32_t st = smem_u32(smem + (size_t)s * STAGE_BYTES);
          const uint64_t bd = sw128_desc(st + PIECES * A_TILE);
          for (int p = 0; p < PIECES; ++p) {
            const uint64_t ad = sw128_desc(st + p * A_TILE);
#pragma unroll
            for (int kk = 0; kk < TK / 16; ++kk)   // +32 bytes along K = +2 in the descriptor's address field
              mma_bf16(d, ad + 2 * kk, bd + 2 * kk, idesc, (kb != g * GROUP || p != 0 || kk != 0) ? 1u : 0u);
          }
          mma_commit(empty0 + 8 * s);
        }
        mma_commit(accf0 + 8 * buf);   // arrives once this group's MMAs have completed
      }
      if (!ok) atomicExch(P.err, 2);
    }
  } else {
    // ---- accumulators: lanes 32 (warp % 4).., columns 64 (warp / 4)..
    const int q = warp & 3, ch = warp >> 2;
    double acc[64];
#pragma unroll
    for (int i = 0; i < 64; ++i) acc[i] = 0.0;
    bool ok = true;
    for (int g = 0; g < ngroups; ++g) {
      const int buf = g & 1;
      if (!mbar_wait(accf0 + 8 * buf, (uint32_t)(g >> 1) & 1u)) { ok = false; break; }
      tc_fence_after();
      const uint32_t base = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * TN + ch * 64);
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        uint32_t v[16];
        tmem_ld16(base + (uint32_t)(c * 16), v);
#pragma unroll
        for (int i = 0; i < 16; ++i) acc[c * 16 + i] += (double)__uint_as_float(v[i]);
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acce0 + 8 * buf);
    }
    if (!ok) {
      if (lane == 0) atomicExch(P.err, 3);
    } else {
      const int row = m0 + q * 32 + lane;
      if (row < P.M) {
        double2* o = reinterpret_cast<double2*>(P.part + ((size_t)blockIdx.z * P.M + row) * P.N + n0 + ch * 64);
#pragma unroll
        for (int i = 0; i < 32; ++i) o[i] = make_double2(acc[2 * i], acc[2 * i + 1]);
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

// X (m x n row-major, ld ldx) -> three bf16 pieces A[p][i][j] (row pitch `pitch`);
// rows over blockIdx.y, columns over the x grid (no index division).  With
// mx, also each row's max |x| (as its bit pattern: the maximum of
// non-negative doubles is the maximum of their patterns) by atomicMax, the
// row maxima the CRT scales of the same X need, from this pass over X.
__global__ void split3_kernel(int m, long n, const double* __restrict__ X, long ldx, __nv_bfloat16* __restrict__ A,
                              long pitch, unsigned long long* __restrict__ mx) {
  const size_t plane = (size_t)m * pitch;
  for (int i = blockIdx.y; i < m; i += gridDim.y) {
    const double* xr = X + (long)i * ldx;
    __nv_bfloat16* ar = A + (size_t)i * pitch;
    double amax = 0.0;
    for (long j = blockIdx.x * (long)blockDim.x + threadIdx.x; j < n; j += (long)gridDim.x * blockDim.x) {
      const double x = xr[j];
      amax = fmax(amax, fabs(x));
      const __nv_bfloat16 b0 = __double2bfloat16(x);
      const double r1 = x - (double)__bfloat162float(b0);
      const __nv_bfloat16 b1 = __double2bfloat16(r1);
      const double r2 = r1 - (double)__bfloat162float(b1);
      const __nv_bfloat16 b2 = __double2bfloat16(r2);
      ar[j] = b0;
      ar[plane + j] = b1;
      ar[2 * plane + j] = b2;
    }
    if (mx) {   // uniform across the block
      for (int o = 16; o > 0; o >>= 1) amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
      if ((threadIdx.x & 31) == 0) atomicMax(mx + i, (unsigned long long)__double_as_longlong(amax));
    }
  }
}

__device__ __forceinline__ uint64_t mix64(uint64_t z) {   // splitmix64 finaliser
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// S (N x n, row pitch `pitch`, a multiple of 8) with independent +-1 entries:
// the eight entries (i, 8g .. 8g + 7) take their signs from bits 0..7 of one
// splitmix64 hash of i ceil(n / 8) + g (a set bit gives -1: bf16 0x3F80 with
// its sign bit set); eight entries per 16-byte store.
__global__ void rademacher_kernel(int N, long n, long pitch, __nv_bfloat16* __restrict__ S, uint64_t seed) {
  const uint64_t groups = (uint64_t)((n + 7) / 8);
  for (int i = blockIdx.y; i < N; i += gridDim.y) {
    uint16_t* row = reinterpret_cast<uint16_t*>(S) + (size_t)i * pitch;
    for (long j0 = (blockIdx.x * (long)blockDim.x + threadIdx.x) * 8; j0 < n; j0 += (long)gridDim.x * blockDim.x * 8) {
      const uint64_t g = (uint64_t)i * groups + (uint64_t)(j0 / 8);
      const uint32_t bits = (uint32_t)mix64(seed ^ g * 0xD1B54A32D192ED03ull);
      uint32_t w[4];
#pragma unroll
      for (int e = 0; e < 4; ++e)
        w[e] = 0x3F803F80u | ((bits >> (2 * e)) & 1u) << 15 | ((bits >> (2 * e + 1)) & 1u) << 31;
      if (j0 + 8 <= n && (reinterpret_cast<uintptr_t>(row + j0) & 15) == 0) {
        *reinterpret_cast<uint4*>(row + j0) = make_uint4(w[0], w[1], w[2], w[3]);
      } else {
        for (int e = 0; e < 8 && j0 + e < n; ++e) row[j0 + e] = (uint16_t)(w[e / 2] >> (16 * (e % 2)));
      }
    }
  }
}

// Y = sum of the K-splits' partial products (accumulate: Y += the sum, for
// every K-chunk after the first).
__global__ void sketch_reduce(long MN, int splits, const double* __restrict__ part, double* __restrict__ Y,
                              int accumulate) {
  for (long f = blockIdx.x * (long)blockDim.x + threadIdx.x; f < MN; f += (long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int z = 0; z < splits; ++z) s += part[(size_t)z * MN + f];
    Y[f] = accumulate ? Y[f] + s : s;
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

struct Split {
  int splits, kb_per_split, kblocks;
};

// K split: the number of splits s (<= MAX_SPLITS) minimising
// (waves of CTAs) x (K-blocks per CTA), the smallest s within 2% of it.
Split plan_split(int m, long n, int N, int num_sms) {
  Split r;
  r.kblocks = (int)((n + TK - 1) / TK);
  const long tiles = (long)(N / TN) * ((m + TM - 1) / TM);
  double best = 1e300;
  int bs = 1;
  const int smax = std::min(MAX_SPLITS, r.kblocks);
  std::vector<double> cost(smax + 1);
  for (int s = 1; s <= smax; ++s) {
    const long waves = (tiles * s + num_sms - 1) / num_sms;
    cost[s] = (double)waves * ((r.kblocks + s - 1) / s);
    best = std::min(best, cost[s]);
  }
  for (int s = 1; s <= smax; ++s)
    if (cost[s] <= 1.02 * best) { bs = s; break; }
  r.kb_per_split = (r.kblocks + bs - 1) / bs;
  r.splits = (r.kblocks + r.kb_per_split - 1) / r.kb_per_split;
  return r;
}

}  // namespace

long sketch_pitch(long n) { return (n + 7) / 8 * 8; }

int sketch_rows(int m) { return (2 * m + TN - 1) / TN * TN; }

namespace {
// The bf16 pieces of X are staged in HBM; over a long dimension they are
// formed in K-chunks of at most this many bytes (multiples of 2^15 columns),
// each chunk's products added into Y, so a block of any length needs bounded
// workspace.
constexpr size_t PIECES_CHUNK_DEFAULT = (size_t)4 << 30;
long sketch_chunk(int m, long n) {
  const size_t cap = long_chunk_bytes(PIECES_CHUNK_DEFAULT);
  const size_t full = (size_t)PIECES * m * sketch_pitch(n) * 2;
  if (full <= cap) return n;
  long c = (long)(cap / ((size_t)PIECES * m * 2)) / 32768 * 32768;
  c = std::max(c, 32768L);
  const long chunks = (n + c - 1) / c;
  return ((n + chunks - 1) / chunks + 32767) / 32768 * 32768;
}
}  // namespace

size_t sketch_workspace_bytes(const bbt_ctx* ctx, int m, long n, int N) {
  const long kc = sketch_chunk(m, n);
  const Split s = plan_split(m, kc, N, ctx->num_sms > 0 ? ctx->num_sms : 148);
  return (size_t)PIECES * m * sketch_pitch(kc) * 2 + (size_t)s.splits * m * N * 8 + 4096;
}

bbt_status rademacher(bbt_ctx* ctx, int N, long n, void* S, uint64_t seed) {
  const long pitch = sketch_pitch(n);
  if (pitch % 8 != 0) return fail(ctx, BBT_ERR_ARG, "rademacher: pitch %ld", pitch);
  const dim3 g((unsigned)std::max(1L, std::min((n + 2047) / 2048, 64L)), (unsigned)std::min(N, 65535));
  rademacher_kernel<<<g, 256, 0, ctx->stream>>>(N, n, pitch, (__nv_bfloat16*)S, seed);
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

bbt_status sketch_chunk_run(bbt_ctx* ctx, int m, long n, const double* X, long ldx, int N, const __nv_bfloat16* S,
                            long spitch, double* Y, __nv_bfloat16* A, double* part, bool accumulate,
                            unsigned long long* rowmax);

// Stream-ordered; a pipeline wait that gave up leaves a nonzero code in
// ctx->d_flag[FLAG_SKETCH] (cleared and read by the caller).
bbt_status sketch_bf16x3(bbt_ctx* ctx, int m, long n, const double* X, long ldx, int N, const void* S, long spitch,
                         double* Y, unsigned long long* rowmax) {
  if (m < 1 || n < 1 || N < TN || N % TN != 0 || n > (1L << 31) - TK || spitch < n || spitch % 8 != 0)
    return fail(ctx, BBT_ERR_ARG, "sketch: m=%d n=%ld N=%d", m, n, N);
  EncodeTiled enc = encode_fn();
  if (!enc) return fail(ctx, BBT_ERR_CUDA, "sketch: cuTensorMapEncodeTiled is not available");
  const long kc = sketch_chunk(m, n);
  const size_t mark = ctx->ws.top;
  const long cpitch = sketch_pitch(kc);
  __nv_bfloat16* A = ctx->ws.take<__nv_bfloat16>((size_t)PIECES * m * cpitch);
  double* part = ctx->ws.take<double>((size_t)plan_split(m, kc, N, ctx->num_sms).splits * m * N);
  if (!part) return fail(ctx, BBT_ERR_NOMEM, "sketch: workspace");
  for (long k0 = 0; k0 < n; k0 += kc)   // chunk offsets are multiples of 2^15: 16-byte TMA bases in S
    BBT_TRY(sketch_chunk_run(ctx, m, std::min(kc, n - k0), X + k0, ldx, N,
                             static_cast<const __nv_bfloat16*>(S) + k0, spitch, Y, A, part, k0 > 0, rowmax));
  ctx->ws.top = mark;
  return BBT_OK;
}

// One K-chunk of sketch_bf16x3: its bf16 pieces in A (pitch sketch_pitch(n)),
// the products of its K-splits in part, summed into Y (added with accumulate);
// the chunk's row maxima of |X| merged into rowmax (when given).
bbt_status sketch_chunk_run(bbt_ctx* ctx, int m, long n, const double* X, long ldx, int N, const __nv_bfloat16* S,
                            long spitch, double* Y, __nv_bfloat16* A, double* part, bool accumulate,
                            unsigned long long* rowmax) {
  EncodeTiled enc = encode_fn();
  const long pitch = sketch_pitch(n);
  const Split sp = plan_split(m, n, N, ctx->num_sms);
  split3_kernel<<<dim3((unsigned)std::max(1L, std::min((n + 255) / 256, 16L)), (unsigned)std::min(m, 65535)), 256, 0,
                  ctx->stream>>>(m, n, X, ldx, A, pitch, rowmax);
  BBT_LAUNCHED(ctx);

  CUtensorMap ta, tb;
  {
    const cuuint64_t dims[3] = {(cuuint64_t)n, (cuuint64_t)m, (cuuint64_t)PIECES};
    const cuuint64_t strides[2] = {(cuuint64_t)pitch * 2, (cuuint64_t)pitch * 2 * m};
    const cuuint32_t box[3] = {TK, TM, 1}, es[3] = {1, 1, 1};
    if (enc(&ta, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, A, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return fail(ctx, BBT_ERR_CUDA, "sketch: tensor map of X");
  }
  {
    const cuuint64_t dims[2] = {(cuuint64_t)n, (cuuint64_t)N};
    const cuuint64_t strides[1] = {(cuuint64_t)spitch * 2};
    const cuuint32_t box[2] = {TK, TN}, es[2] = {1, 1};
    if (enc(&tb, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(S), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return fail(ctx, BBT_ERR_CUDA, "sketch: tensor map of S");
  }
  static bool attr = false;
  if (!attr) {
    BBT_CUDA(ctx, cudaFuncSetAttribute(sketch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
    attr = true;
  }
  SketchArgs a;
  a.part = part;
  a.M = m;
  a.N = N;
  a.kblocks = sp.kblocks;
  a.kb_per_split = sp.kb_per_split;
  a.err = ctx->d_flag + FLAG_SKETCH;
  {
    ProfScope prof(ctx, BBT_PROF_SKETCH, 2.0 * PIECES * (double)m * N * n);
    sketch_kernel<<<dim3(N / TN, (m + TM - 1) / TM, sp.splits), THREADS, SMEM_BYTES, ctx->stream>>>(ta, tb, a);
    BBT_LAUNCHED(ctx);
  }
  const long MN = (long)m * N;
  sketch_reduce<<<4 * ctx->num_sms, 256, 0, ctx->stream>>>(MN, sp.splits, part, Y, accumulate ? 1 : 0);
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

}  // namespace bbt
