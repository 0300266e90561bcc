// Exact integer matrix products on the int8 tensor cores by the Chinese
// remainder theorem: the FP64-accurate (and, for the Gram matrix, exact)
// products of the mixed-precision path.
//
//   C (M x N, column-major) = A B^T,  A(i, k), B(j, k) given as residue planes.
//
// Every row of an operand is scaled by a power of two s_i (|x / s_i| < 1/2)
// and rounded to a b-bit integer t = rint(x 2^(b-1) / s_i), |t| <= 2^(b-2).
// The integer product T = A_int B_int^T is then computed exactly modulo n
// pairwise coprime moduli p <= 256: with residues in [0, p) every modulus is
// one u8 x u8 -> int32 GEMM (tcgen05 kind::i8, 128 x 256 tiles, one TMEM
// accumulator), exact for up to 2^15 terms per K-split.  The
// residues of T are written as bytes and the integer is rebuilt from them
// (crt_combine): T/M = sum_p (T mod p) ((M/p)^-1 mod p) / p mod 1 (M = prod p),
// evaluated as a 128-bit fixed-point sum of (T mod p) G_p, G_p =
// floor(2^128 ((M/p)^-1 mod p) / p), whose wrap-around discards the integer
// part exactly (no reduction of the CRT digit mod p is needed).  n is
// chosen so that |T| < M / 2, so the centred fraction times M is T itself, to
// about 2^-110 of the largest possible |T|.
//
// Against the slice-pair (Ozaki) products of ozaki.cu this needs n int8
// products instead of S(S+1)/2, each with a 256-column accumulator instead of
// S accumulators sharing 512 TMEM columns (so half the shared-memory operand
// traffic per multiply-add), at the price of a per-output epilogue: it pays
// where K is long (the Gram matrix).
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <utility>
#include <vector>

#include "internal.h"
#include "tc.cuh"

namespace bbt {
namespace {

using namespace tc;

constexpr int MAXMOD = 24;
// Pairwise coprime, largest first after 2^8: 255 = 3 5 17, 253 = 11 23,
// 247 = 13 19, 217 = 7 31; the others are primes.
constexpr int MODULI[MAXMOD] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217,
                                211, 199, 197, 193, 191, 181, 179, 173, 167, 163, 157, 151};

// Compile-time constants of modulus Q of an NM-modulus set, for the kernels
// templated on NM (every per-modulus constant becomes an immediate once the
// loop over the moduli is unrolled).
constexpr int inv_mod_c(int a, int p) {   // a^-1 mod p, gcd(a, p) = 1
  int t = 0, nt = 1, r = p, nr = a % p;
  while (nr) {
    const int q = r / nr;
    const int x = t - q * nt;
    t = nt;
    nt = x;
    const int y = r - q * nr;
    r = nr;
    nr = y;
  }
  return t < 0 ? t + p : t;
}
constexpr int crt_inv_c(int q, int n) {   // ((M / p_q) mod p_q)^-1 mod p_q, M the product of n moduli
  long long prod = 1;
  for (int r = 0; r < n; ++r)
    if (r != q) prod = prod * (MODULI[r] % MODULI[q]) % MODULI[q];
  return inv_mod_c((int)prod, MODULI[q]);
}
constexpr uint32_t flimb_c(int p, int l) {   // 32-bit limb l of floor(2^128 / p), least significant first
  const uint32_t digits[5] = {1, 0, 0, 0, 0};   // 2^128 in base 2^32, most significant first
  uint32_t q[5] = {0, 0, 0, 0, 0};
  uint64_t rem = 0;
  for (int d = 0; d < 5; ++d) {
    const uint64_t cur = (rem << 32) | digits[d];
    q[d] = (uint32_t)(cur / (uint64_t)p);
    rem = cur % (uint64_t)p;
  }
  return q[4 - l];
}
// 32-bit limb l of G = floor(2^128 inv / p) (inv < p, so G < 2^128):
// inv floor(2^128 / p) + floor(inv (2^128 mod p) / p), least significant limb first.
constexpr uint32_t glimb_c(int p, int inv, int l) {
  uint64_t limb[4] = {flimb_c(p, 0), flimb_c(p, 1), flimb_c(p, 2), flimb_c(p, 3)};
  uint64_t rem = 1;   // 2^128 mod p, by doubling
  for (int i = 0; i < 128; ++i) rem = (2 * rem) % (uint64_t)p;
  uint64_t carry = ((uint64_t)inv * rem) / (uint64_t)p;
  uint32_t out[4] = {0, 0, 0, 0};
  for (int i = 0; i < 4; ++i) {
    const uint64_t t = limb[i] * (uint64_t)inv + carry;
    out[i] = (uint32_t)t;
    carry = t >> 32;
  }
  return out[l];
}
constexpr uint32_t byte_weight(int p, int j) { return (uint32_t)(((uint64_t)1 << (8 * j)) % (uint64_t)p); }
template <int Q>
struct ModR {   // residues of an integer t from the bytes of u = t + 2^51
  static constexpr int p = MODULI[Q];
  // 256^j mod p for the bytes j = 0..3 of u's low word and 4..6 of its high word
  static constexpr uint32_t W0 = byte_weight(p, 0) | byte_weight(p, 1) << 8 | byte_weight(p, 2) << 16 |
                                 byte_weight(p, 3) << 24;
  static constexpr uint32_t W1 = byte_weight(p, 4) | byte_weight(p, 5) << 8 | byte_weight(p, 6) << 16;
  static constexpr uint32_t off = (uint32_t)p - (uint32_t)(((uint64_t)1 << 51) % (uint64_t)p);   // -2^51 mod p, in [1, p]
  static constexpr uint32_t magic32 = (uint32_t)((((uint64_t)1 << 32) + p - 1) / p);
};
template <int Q, int NM>
struct ModK {   // reconstruction from the residues of an NM-modulus set
  static constexpr int p = MODULI[Q];
  static constexpr uint32_t magic32 = (uint32_t)((((uint64_t)1 << 32) + p - 1) / p);
  static constexpr uint32_t inv = (uint32_t)crt_inv_c(Q, NM);
  // r G / 2^128 = r inv / p (mod 1) up to r units of 2^-128: the CRT digit's
  // fraction straight from the residue r, with no reduction of r inv mod p
  static constexpr uint32_t G0 = glimb_c(p, (int)inv, 0), G1 = glimb_c(p, (int)inv, 1),
                            G2 = glimb_c(p, (int)inv, 2), G3 = glimb_c(p, (int)inv, 3);
};

constexpr int TM = 128, TN = 256, TK = 128;   // TK: bytes of K per stage row (SWIZZLE_128B)
constexpr int STAGES = 4;
constexpr int A_TILE = TM * TK, B_TILE = TN * TK;
constexpr int STAGE_BYTES = A_TILE + B_TILE;   // 48 KB
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;
constexpr int EPI_WARPS = 16;   // four per TMEM lane quarter, each draining TN / 4 columns
constexpr int EPI_COLS = TN / (EPI_WARPS / 4);
constexpr int THREADS = (EPI_WARPS + 2) * 32;
constexpr uint32_t TMEM_COLS = 2 * TN;          // two accumulators: modulus p+1 runs while p drains
constexpr int MAX_KB_PER_SPLIT = 32768 / TK;    // T < 2^15 * 2^16 per split: no int32 overflow
constexpr int MAX_SPLITS = 64;

struct Mods {
  int n;
  int p[MAXMOD];
  int c16[MAXMOD];     // 2^16 mod p
  float invf[MAXMOD];  // 1 / p
  int inv[MAXMOD];     // ((M / p) mod p)^-1 mod p
  uint32_t F[MAXMOD][4];   // floor(2^128 / p), 32-bit limbs, least significant first
  double mod_hi, mod_lo;   // M as a double-double
  double mod_bits;         // log2 M
};

// ---- residues of integer-valued operands --------------------------------

__device__ __forceinline__ int centre(int r, int p) {
  const int hi = (p - 1) >> 1, lo = hi - p + 1;
  if (r > hi) r -= p;
  if (r > hi) r -= p;
  if (r < lo) r += p;
  if (r < lo) r += p;
  return r;
}

// t an integer-valued double, |t| <= 2^53 (so |t / p| < 2^51).  Rounding and
// the conversion to an integer by adding 1.5 2^52 (the integer lands in the
// low mantissa bits) instead of conversion instructions.
__device__ __forceinline__ int residue(double t, int p, double invp) {
  const double RND = 6755399441055744.0;   // 1.5 * 2^52
  const double q = (t * invp + RND) - RND;
  const double r = fma(-q, (double)p, t);   // exact, |r| < 2p
  return centre(__double2loint(r + RND), p);
}

// Residue of an integer-valued double of any size below 2^100: t = m 2^e with
// an integer m < 2^53, residue(m) times 2^e mod p.
__device__ __forceinline__ int residue_big(double t, int p, double invp) {
  if (fabs(t) < 9007199254740992.0) return residue(t, p, invp);   // 2^53
  int e = 0;
  frexp(t, &e);
  e -= 53;
  int r = residue(ldexp(t, -e), p, invp);
  for (int s = 0; s < e; ++s) r = centre(2 * r, p);
  return r;
}

// Row maxima: blocks of 256 threads over (rows, chunks of 8192 columns); the
// maximum of non-negative doubles is the maximum of their bit patterns, so
// chunks combine by atomicMax.  Short rows: one warp per row.
__global__ void rowmax_kernel(int rows, long K, const double* __restrict__ X, long rs,
                              unsigned long long* __restrict__ mx) {
  __shared__ double sh[8];
  for (int i = blockIdx.y; i < rows; i += gridDim.y) {
    const long k0 = (long)blockIdx.x * 8192;
    const double* x = X + (long)i * rs;
    double m = 0.0;
    for (long k = k0 + threadIdx.x; k < K && k < k0 + 8192; k += blockDim.x) m = fmax(m, fabs(x[k]));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, sh[w]);
      atomicMax(mx + i, (unsigned long long)__double_as_longlong(m));
    }
    __syncthreads();
  }
}

__global__ void rowmax_short_kernel(int rows, long K, const double* __restrict__ X, long rs,
                                    unsigned long long* __restrict__ mx) {
  const int lane = threadIdx.x & 31;
  for (long i = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5; i < rows; i += ((long)gridDim.x * blockDim.x) >> 5) {
    const double* x = X + i * rs;
    double m = 0.0;
    for (long k = lane; k < K; k += 32) m = fmax(m, fabs(x[k]));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) mx[i] = (unsigned long long)__double_as_longlong(m);
  }
}

// s_i = 2^(e+1) with max |x| in [2^(e-1), 2^e) (1 for an all-zero row)
__global__ void scale_kernel(int rows, const unsigned long long* __restrict__ mx, double* __restrict__ scale) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows) return;
  const double m = __longlong_as_double((long long)mx[i]);
  int e = 0;
  if (m > 0.0) frexp(m, &e);
  scale[i] = ldexp(1.0, e + 1);
}

// 2^(b-1) / s for s a normal power of two, by exponent arithmetic.
__device__ __forceinline__ double pow2_ratio(int b, double s) {
  const int e = (int)((__double_as_longlong(s) >> 52) & 0x7FF) - 1023;
  return __longlong_as_double((long long)(1023 + (b - 1) - e) << 52);
}

struct ModTab {
  int n;
  int p[MAXMOD];
  double invp[MAXMOD];
};

// An integer-valued t with |t| <= 2^51 as u = t + 2^51 in [0, 2^52]:
// y = t + 1.5 2^52 is exact (unit spacing below 2^53, and u = 2^52 gives
// y = 2^53 exactly), y's low word is u's low 32 bits, and y's high word less
// that of 2^52 is u >> 32 (at y = 2^53 the exponent step leaves 2^20 there,
// which is 2^52 >> 32).
struct U52 {
  uint32_t lo, hi;
};
__device__ __forceinline__ U52 offset_u52(double t) {
  const double y = __dadd_rn(t, 0x1.8p52);
  return {(uint32_t)__double2loint(y), (uint32_t)__double2hiint(y) - 0x43300000u};
}

// The residue in [0, p) of modulus Q: u's seven bytes (the high word is at
// most 2^20) weighted by 256^j mod p in two byte dot products, plus -2^51 mod
// p: 0 < x < 2^19, so the multiply-high quotient by ceil(2^32 / p) is exact.
template <int Q>
__device__ __forceinline__ uint32_t res_q(const U52& u) {
  using C = ModR<Q>;
  const uint32_t x = __dp4a(u.lo, C::W0, __dp4a(u.hi, C::W1, C::off));
  return x - __umulhi(x, C::magic32) * (uint32_t)C::p;
}

template <int Q>
__device__ __forceinline__ void store4_q(const U52 (&t)[4], int8_t* o, int valid) {
  const uint32_t w = __byte_perm(__byte_perm(res_q<Q>(t[0]), res_q<Q>(t[1]), 0x0040),
                                 __byte_perm(res_q<Q>(t[2]), res_q<Q>(t[3]), 0x0040), 0x5410);
  if (valid == 4) {
    *reinterpret_cast<uint32_t*>(o) = w;
  } else {
    for (int e = 0; e < valid; ++e) o[e] = (int8_t)(w >> (8 * e));
  }
}
template <int... Q>
__device__ __forceinline__ void store4_all(const U52 (&t)[4], int8_t* o, size_t plane, int valid,
                                           std::integer_sequence<int, Q...>) {
  (store4_q<Q>(t, o + (size_t)Q * plane, valid), ...);
}

// Rows contiguous in k: planes out[p][i][k] (row pitch Kp), four elements per
// thread; rows over blockIdx.y, K over the x grid.
template <int NM>
__global__ void residues_rows_kernel(int rows, long K, const double* __restrict__ X, long rs,
                                     const double* __restrict__ scale, int b, int8_t* __restrict__ out, long Kp) {
  const long kq = (K + 3) / 4;
  const size_t plane = (size_t)rows * Kp;
  for (int i = blockIdx.y; i < rows; i += gridDim.y)
  for (long kk = blockIdx.x * (long)blockDim.x + threadIdx.x; kk < kq; kk += (long)gridDim.x * blockDim.x) {
    const long k = kk * 4;
    const double mul = pow2_ratio(b, scale[i]);   // a power of two: exact
    const double* x = X + (long)i * rs + k;
    U52 t[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) t[e] = offset_u52((k + e < K) ? rint(x[e] * mul) : 0.0);
    store4_all(t, out + (size_t)i * Kp + k, plane, (int)min(4L, K - k), std::make_integer_sequence<int, NM>{});
  }
}

// Rows contiguous in i, K stride cs; the scale belongs to the K index
// (kscale) -- the integers are those residues_rows_kernel forms for the
// transposed operand.  Tiles of 128 K x 32 rows staged through shared memory
// (coalesced along i on the way in); four consecutive K per thread on the way
// out, packed into 32-bit stores (a warp writes 128 contiguous bytes of a plane).
template <int NM>
__global__ void __launch_bounds__(256) residues_cols_kernel(int rows, long K, const double* __restrict__ X, long cs,
                                                            const double* __restrict__ kscale, int b,
                                                            int8_t* __restrict__ out, long Kp) {
  __shared__ double tile[128][33];   // tile[k][i]
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int i0 = blockIdx.x * 32;
  const long k0 = (long)blockIdx.y * 128;
  for (int r = ty; r < 128; r += 8) {
    const long k = k0 + r;
    const int i = i0 + tx;
    tile[r][tx] = (i < rows && k < K) ? rint(X[i + k * cs] * pow2_ratio(b, kscale[k])) : 0.0;
  }
  __syncthreads();
  const size_t plane = (size_t)rows * Kp;
  const long k = k0 + 4 * tx;
  for (int r = ty; r < 32; r += 8) {
    const int i = i0 + r;
    if (i < rows && k < K) {
      U52 t[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) t[e] = offset_u52(tile[4 * tx + e][r]);
      store4_all(t, out + (size_t)i * Kp + k, plane, (int)min(4L, K - k), std::make_integer_sequence<int, NM>{});
    }
  }
}

// Double-double rows (hi + lo), rows contiguous in k, b up to 100 bits:
// t = T_hi + T_lo with T_hi = rint(hi 2^(b-1) / s_i) (any size, m 2^e with an
// integer m < 2^53) and T_lo = rint(lo 2^(b-1) / s_i + the fraction of hi's).
__global__ void residues_dd_kernel(int rows, long K, const double* __restrict__ Xh, const double* __restrict__ Xl,
                                   long rs, const double* __restrict__ scale, int b, ModTab T,
                                   int8_t* __restrict__ out, long Kp) {
  const long total = (long)rows * K;
  const size_t plane = (size_t)rows * Kp;
  for (long f = blockIdx.x * (long)blockDim.x + threadIdx.x; f < total; f += (long)gridDim.x * blockDim.x) {
    const int i = (int)(f / K);
    const long k = f - (long)i * K;
    const double mul = pow2_ratio(b, scale[i]);
    const double h = Xh[(long)i * rs + k] * mul, l = Xl[(long)i * rs + k] * mul;
    const double th = rint(h);
    const double tl = rint(l + (h - th));
    for (int q = 0; q < T.n; ++q) {
      const int p = T.p[q];
      int r = centre(residue_big(th, p, T.invp[q]) + residue_big(tl, p, T.invp[q]), p);
      if (r < 0) r += p;   // stored in [0, p)
      out[q * plane + (size_t)i * Kp + k] = (int8_t)r;
    }
  }
}

// ---- one int8 GEMM per modulus ------------------------------------------

struct CrtArgs {
  uint8_t* out;   // residues of T: out[((z * n + q) * N + j) * Mp + i], Mp = M rounded up to 4
  int M, N, Mp;
  int kblocks, kb_per_split;
  int n;
  int upper;      // 1: skip tiles strictly below the diagonal
  int p[MAXMOD], c16[MAXMOD];
  uint32_t magic[MAXMOD];   // ceil(2^32 / p): exact quotients below 2^24
  int* err;
};

// AMN: A's residue planes are MN-major (the row index i of A contiguous, K
// along the planes' rows), as the Gram's planes of X serve the products
// X_int^T Z: the TMA box and the K advance change, and the instruction
// descriptor marks A as MN-major (valid for 8-bit integer operands).
template <bool AMN>
__global__ void __launch_bounds__(THREADS, 1)
crt_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, CrtArgs P) {
  const int n0 = blockIdx.x * TN, m0 = blockIdx.y * TM;
  if (P.upper && m0 >= n0 + TN) return;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* bars = (uint64_t*)(smem + STAGES * STAGE_BYTES);
  uint32_t* tmem_slot = (uint32_t*)(bars + 2 * STAGES + 4);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int kb0 = blockIdx.z * P.kb_per_split;
  const int nk = min(P.kblocks - kb0, P.kb_per_split);
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
  const int total = P.n * nk;

  if (warp == EPI_WARPS) {
    if (lane == 0) {   // ---- TMA producer: modulus after modulus, K-block after K-block
      int issued = 0;
      bool ok = true;
      for (int it = 0; it < total; ++it) {
        const int q = it / nk, kb = it - q * nk;
        const int s = it % STAGES;
        const uint32_t ph = (uint32_t)(it / STAGES) & 1u;
        if (!mbar_wait(empty0 + 8 * s, ph ^ 1u)) { ok = false; break; }
        const uint32_t fb = full0 + 8 * s;
        mbar_expect_tx(fb, (uint32_t)STAGE_BYTES);
        const uint32_t st = smem_u32(smem + (size_t)s * STAGE_BYTES);
        const int kx = (kb0 + kb) * TK;
        if (AMN)
          tma_load_3d(st, &tmA, fb, m0, kx, q);
        else
          tma_load_3d(st, &tmA, fb, kx, m0, q);
        tma_load_3d(st + A_TILE, &tmB, fb, kx, n0, q);
        ++issued;
      }
      if (!ok) atomicExch(P.err, 1);
      for (int it = max(0, issued - STAGES); it < issued; ++it)
        if (!mbar_wait(full0 + 8 * (it % STAGES), (uint32_t)(it / STAGES) & 1u)) atomicExch(P.err, 4);
    }
  } else if (warp == EPI_WARPS + 1) {
    if (lane == 0) {   // ---- MMA issuer: u8 x u8 -> int32, K-major, 128 x 256 x 32 per instruction
      const uint32_t idesc =   // c_format S32, a/b unsigned 8-bit, A K-major or MN-major (bit 15)
          (2u << 4) | (0u << 7) | (0u << 10) | ((AMN ? 1u : 0u) << 15) | ((uint32_t)(TN >> 3) << 17) |
          ((uint32_t)(TM >> 4) << 24);
      bool ok = true;
      for (int q = 0; q < P.n && ok; ++q) {
        const int buf = q & 1, use = q >> 1;
        if (use > 0 && !mbar_wait(acce0 + 8 * buf, (uint32_t)(use - 1) & 1u)) { ok = false; break; }
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(buf * TN);
        for (int kb = 0; kb < nk; ++kb) {
          const int it = q * nk + kb;
          const int s = it % STAGES;
          if (!mbar_wait(full0 + 8 * s, (uint32_t)(it / STAGES) & 1u)) { ok = false; break; }
          tc_fence_after();
          const uint32_t st = smem_u32(smem + (size_t)s * STAGE_BYTES);
          const uint64_t ad = sw128_desc(st), bd = sw128_desc(st + A_TILE);
          // +32 along K: +32 bytes (K-major, +2 in the descriptor's address field) or
          // +32 rows of 128 bytes (MN-major, +256)
#pragma unroll
          for (int kk = 0; kk < TK / 32; ++kk)
            mma_i8(d, ad + (AMN ? 256 : 2) * kk, bd + 2 * kk, idesc, (kb != 0 || kk != 0) ? 1u : 0u);
          mma_commit(empty0 + 8 * s);
        }
        mma_commit(accf0 + 8 * buf);
      }
      if (!ok) atomicExch(P.err, 2);
    }
  } else {
    // ---- epilogue: TMEM lanes 32 (warp % 4).., columns EPI_COLS (warp / 4).. of the
    //      accumulator; T mod p as a byte per element, i (the TMEM lane) contiguous in memory.
    //      The accumulator sums at most 2^15 products of bytes, so 0 <= v < 2^31:
    //      (v >> 16) c16 + (v & 0xFFFF) < 2^24 is congruent to it and its
    //      multiply-high quotient by p is exact
    const int q4 = warp & 3, ch = warp >> 2;
    const int i = m0 + q4 * 32 + lane;
    const bool row_ok = i < P.M;
    bool ok = true;
    for (int q = 0; q < P.n; ++q) {
      const int buf = q & 1, use = q >> 1;
      if (!mbar_wait(accf0 + 8 * buf, (uint32_t)use & 1u)) { ok = false; break; }
      tc_fence_after();
      const uint32_t p = (uint32_t)P.p[q], c16 = (uint32_t)P.c16[q], magic = P.magic[q];
      uint8_t* o = P.out + ((size_t)blockIdx.z * P.n + q) * (size_t)P.N * P.Mp + i;
#pragma unroll 1
      for (int c = 0; c < EPI_COLS / 16; ++c) {
        uint32_t v[16];
        tmem_ld16(tmem + ((uint32_t)(q4 * 32) << 16) + (uint32_t)(buf * TN + ch * EPI_COLS + c * 16), v);
        const int j0 = n0 + ch * EPI_COLS + c * 16;
        const int jn = row_ok ? min(16, P.N - j0) : 0;   // columns of this chunk to store
        uint8_t* oc = o + (size_t)j0 * P.Mp;
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          const uint32_t x = (v[e] >> 16) * c16 + (v[e] & 0xFFFFu);
          const uint32_t r = x - __umulhi(x, magic) * p;
          if (e < jn) oc[(size_t)e * P.Mp] = (uint8_t)r;
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acce0 + 8 * buf);
    }
    if (!ok && lane == 0) atomicExch(P.err, 3);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
  }
}

// ---- rebuilding T from its residues ---------------------------------------

struct CombArgs {
  const uint8_t* R;        // [split][modulus][N][Mp]
  int M, N, Mp, splits, upper;
  double mod_hi, mod_lo;   // M as a double-double
};

// x mod p for 0 <= x < 2^24 by the multiply-high quotient.
template <class C>
__device__ __forceinline__ uint32_t mod_c(uint32_t x) {
  return x - __umulhi(x, C::magic32) * (uint32_t)C::p;
}

// Four consecutive outputs: one 32-bit word of residues per modulus (and split).
// The fraction T / M (mod 1) is sum_q r_q G_q / 2^128 (mod 1), r_q = T mod p_q
// and G_q = floor(2^128 ((M / p_q)^-1 mod p_q) / p_q): each term is short by
// less than r_q < 256 units of its last limb.  LIMBS = 4: the fraction to 128
// bits (double-double outputs); 3: to 96 bits (FP64 outputs: the missing 32
// bits are below 2^-75 of the largest |T|), the top three limbs of G_q.
// SPLIT: the product came in several K-splits, whose residues are summed
// first; with one split every byte is already a residue in [0, p).
template <int Q, int NM, int LIMBS, bool SPLIT>
__device__ __forceinline__ void frac4_q(const CombArgs& A, long f, long total, uint64_t (&L)[4][4]) {
  using C = ModK<Q, NM>;
  uint32_t s[4];
  const uint32_t w = *reinterpret_cast<const uint32_t*>(A.R + (size_t)Q * total + f);
#pragma unroll
  for (int e = 0; e < 4; ++e) s[e] = (w >> (8 * e)) & 0xFFu;
  if (SPLIT)
    for (int z = 1; z < A.splits; ++z) {
      const uint32_t v = *reinterpret_cast<const uint32_t*>(A.R + ((size_t)z * NM + Q) * total + f);
#pragma unroll
      for (int e = 0; e < 4; ++e) s[e] += (v >> (8 * e)) & 0xFFu;
    }
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const uint32_t r = SPLIT ? mod_c<C>(s[e]) : s[e];
    if (LIMBS == 4) L[e][0] += (uint64_t)r * C::G0;   // 32 x 32 -> 64-bit products, < 2^40 each
    L[e][1] += (uint64_t)r * C::G1;
    L[e][2] += (uint64_t)r * C::G2;
    L[e][3] += (uint64_t)r * C::G3;
  }
}
template <int NM, int LIMBS, bool SPLIT, int... Q>
__device__ __forceinline__ void frac4_all(const CombArgs& A, long f, long total, uint64_t (&L)[4][4],
                                          std::integer_sequence<int, Q...>) {
  (frac4_q<Q, NM, LIMBS, SPLIT>(A, f, total, L), ...);
}

// The centred fractions T / M (mod 1) of four consecutive outputs as signed
// 128-bit fixed-point numbers (two 64-bit halves each).
template <int NM, int LIMBS, bool SPLIT = true>
__device__ __forceinline__ void crt_fraction4(const CombArgs& A, long f, long total, uint64_t (&hi)[4],
                                              uint64_t (&lo)[4]) {
  uint64_t L[4][4] = {};
  frac4_all<NM, LIMBS, SPLIT>(A, f, total, L, std::make_integer_sequence<int, NM>{});
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    L[e][1] += L[e][0] >> 32;
    L[e][2] += L[e][1] >> 32;
    L[e][3] += L[e][2] >> 32;
    lo[e] = (L[e][0] & 0xFFFFFFFFull) | (L[e][1] << 32);
    hi[e] = (L[e][2] & 0xFFFFFFFFull) | (L[e][3] << 32);
  }
}

__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = __dadd_rn(a, b);
  const double bb = __dsub_rn(s, a);
  e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
}

// A signed 128-bit integer (two's complement, hi:lo) as a double-double: its
// magnitude split exactly into three 53-bit chunks, summed with error terms.
__device__ __forceinline__ void fixed_to_dd(uint64_t hi, uint64_t lo, double& dh, double& dl) {
  const bool neg = (int64_t)hi < 0;
  if (neg) {
    lo = ~lo + 1;
    hi = ~hi + (lo == 0 ? 1 : 0);
  }
  const uint64_t m53 = (1ull << 53) - 1;
  const double c0 = (double)(lo & m53);
  const double c1 = ldexp((double)(((lo >> 53) | (hi << 11)) & m53), 53);
  const double c2 = ldexp((double)(hi >> 42), 106);
  double s, e1, t, e2;
  two_sum(c2, c1, s, e1);
  two_sum(s, c0, t, e2);
  const double e = e1 + e2;
  dh = t + e;
  dl = e - (dh - t);
  if (neg) {
    dh = -dh;
    dl = -dl;
  }
}

__device__ __forceinline__ void two_prod(double a, double b, double& p, double& e) {
  p = __dmul_rn(a, b);   // rounded on its own: never fused with a later sum
  e = fma(a, b, -p);
}

// A signed 128-bit fraction (two's complement, hi:lo) as the nearest-ish
// double times 2^128: magnitude first (no cancellation between the halves),
// then hi 2^64 + lo converted in two roundings (within 2 ulps).
__device__ __forceinline__ double fixed_to_double(uint64_t hi, uint64_t lo) {
  const bool neg = (int64_t)hi < 0;
  if (neg) {
    lo = ~lo + 1;
    hi = ~hi + (lo == 0 ? 1 : 0);
  }
  const double v = fma((double)hi, 18446744073709551616.0, (double)lo);   // 2^64
  return neg ? -v : v;
}

// C (column-major, ldc) = alpha * sa_i sb_j 2^-shift T + beta * C; four
// consecutive i per thread.  scale = M 2^(-128 - shift) (M the moduli's
// product): the fraction T / M (mod 1) times M, back at the operands' scale.
template <int NM, bool SPLIT>
__global__ void __launch_bounds__(256, 4)
combine_kernel(CombArgs A, const double* __restrict__ sa, const double* __restrict__ sb, double scale, double alpha,
               double beta, double* __restrict__ C, long ldc) {
  const long total = (long)A.Mp * A.N;
  for (int j = blockIdx.y; j < A.N; j += gridDim.y)
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) * 4; i < A.M; i += gridDim.x * blockDim.x * 4) {
    if (A.upper && (i / TM) * TM >= (j / TN) * TN + TN) continue;   // tile never computed
    uint64_t hi[4], lo[4];
    crt_fraction4<NM, 3, SPLIT>(A, i + (long)j * A.Mp, total, hi, lo);
    const double sbj = sb[j] * scale;
    double v[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) v[e] = fixed_to_double(hi[e], lo[e]) * (sa ? sa[min(i + e, A.M - 1)] : 1.0) * sbj;
    double* c = C + i + (long)j * ldc;
    if (i + 4 <= A.M && ((reinterpret_cast<uintptr_t>(c) & 15) == 0)) {   // two 16-byte stores
      double2* c2 = reinterpret_cast<double2*>(c);
      if (beta == 0.0) {
        c2[0] = make_double2(alpha * v[0], alpha * v[1]);
        c2[1] = make_double2(alpha * v[2], alpha * v[3]);
      } else {
        const double2 o0 = c2[0], o1 = c2[1];
        c2[0] = make_double2(alpha * v[0] + beta * o0.x, alpha * v[1] + beta * o0.y);
        c2[1] = make_double2(alpha * v[2] + beta * o1.x, alpha * v[3] + beta * o1.y);
      }
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        if (i + e >= A.M) break;
        c[e] = (beta == 0.0) ? alpha * v[e] : alpha * v[e] + beta * c[e];
      }
    }
  }
}

// The same value as a double-double (Ch + Cl), alpha = 1, beta = 0.
template <int NM>
__global__ void __launch_bounds__(256, 2)
combine_dd_kernel(CombArgs A, const double* __restrict__ sa, const double* __restrict__ sb, int shift,
                  double* __restrict__ Ch, double* __restrict__ Cl, long ldc) {
  const long total = (long)A.Mp * A.N;
  for (int j = blockIdx.y; j < A.N; j += gridDim.y)
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) * 4; i < A.M; i += gridDim.x * blockDim.x * 4) {
    if (A.upper && (i / TM) * TM >= (j / TN) * TN + TN) continue;
    uint64_t hi[4], lo[4];
    crt_fraction4<NM, 4>(A, i + (long)j * A.Mp, total, hi, lo);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if (i + e >= A.M) break;
      double fh, fl;
      fixed_to_dd(hi[e], lo[e], fh, fl);
      // (fh + fl) (mod_hi + mod_lo), then exact power-of-two scalings
      double p, er;
      two_prod(fh, A.mod_hi, p, er);
      er += fh * A.mod_lo + fl * A.mod_hi;
      const double s = __dadd_rn(p, er);
      const double t = __dsub_rn(er, __dsub_rn(s, p));
      const double sc = ldexp((sa ? sa[i + e] : 1.0) * sb[j], -128 - shift);
      Ch[(i + e) + (long)j * ldc] = s * sc;
      Cl[(i + e) + (long)j * ldc] = t * sc;
    }
  }
}

// ---- products with a short K and an MN-major A: A kept in shared memory ----
// The products with Q (C = X_int^T Z2, K = m <= 1024) read B (Z2's residues,
// N x K per modulus, L2-resident) for every 128-row block of A.  Here one CTA
// owns a 128-row block and every 256-column tile of it: per modulus, A's K
// blocks (up to 8 x 16 KB) are loaded once into resident slots and each column
// tile streams only its B blocks through a 3-stage ring, so the operand
// traffic from L2 per tile falls from A + B to A / tiles + B (a quarter less at
// N = 1000: the products are bound by that traffic).  A slot is refilled with
// the next modulus as soon as the last tile's MMAs on it have completed
// (tcgen05.commit on the slot's barrier), so the ring keeps running across
// moduli.  The epilogue and the residue layout are crt_kernel's.
constexpr int AR_SLOTS = 8;     // resident K blocks of A: K <= 1024
constexpr int AR_BSTAGES = 3;
constexpr int AR_SMEM = AR_SLOTS * A_TILE + AR_BSTAGES * B_TILE + 1024 + 256;

__global__ void __launch_bounds__(THREADS, 1)
crt_apply_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, CrtArgs P) {
  const int m0 = blockIdx.x * TM;
  const int nt = (P.N + TN - 1) / TN, nk = P.kblocks;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* aslots = smem;
  uint8_t* bring = smem + AR_SLOTS * A_TILE;
  uint64_t* bars = (uint64_t*)(bring + AR_BSTAGES * B_TILE);
  // [0, 8) A full, [8, 16) A empty, [16, 19) B full, [19, 22) B empty, [22, 24) acc full, [24, 26) acc empty
  uint32_t* tmem_slot = (uint32_t*)(bars + 26);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t afull0 = smem_u32(bars), aempty0 = smem_u32(bars + 8);
  const uint32_t bfull0 = smem_u32(bars + 16), bempty0 = smem_u32(bars + 19);
  const uint32_t accf0 = smem_u32(bars + 22), acce0 = smem_u32(bars + 24);
  if (threadIdx.x == 0) {
    for (int k = 0; k < AR_SLOTS; ++k) {
      mbar_init(afull0 + 8 * k, 1);
      mbar_init(aempty0 + 8 * k, 1);
    }
    for (int s = 0; s < AR_BSTAGES; ++s) {
      mbar_init(bfull0 + 8 * s, 1);
      mbar_init(bempty0 + 8 * s, 1);
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
      bool ok = true;
      int it = 0;      // B ring position
      for (int q = 0; q < P.n && ok; ++q)
        for (int t = 0; t < nt && ok; ++t)
          for (int kb = 0; kb < nk; ++kb) {
            const int kx = kb * TK;
            if (t == 0) {   // A's block kb of modulus q, once its slot is free
              const uint32_t fa = afull0 + 8 * kb;
              if (q > 0 && !mbar_wait(aempty0 + 8 * kb, (uint32_t)(q - 1) & 1u)) { ok = false; break; }
              mbar_expect_tx(fa, (uint32_t)A_TILE);
              tma_load_3d(smem_u32(aslots + (size_t)kb * A_TILE), &tmA, fa, m0, kx, q);
            }
            const int s = it % AR_BSTAGES;
            const uint32_t fb = bfull0 + 8 * s;
            if (!mbar_wait(bempty0 + 8 * s, ((uint32_t)(it / AR_BSTAGES) & 1u) ^ 1u)) { ok = false; break; }
            mbar_expect_tx(fb, (uint32_t)B_TILE);
            tma_load_3d(smem_u32(bring + (size_t)s * B_TILE), &tmB, fb, kx, t * TN, q);
            ++it;
          }
      if (!ok) atomicExch(P.err, 1);
      // copies still in flight land before the CTA leaves (all consumed on success)
      for (int k = max(0, it - AR_BSTAGES); k < it; ++k)
        if (!mbar_wait(bfull0 + 8 * (k % AR_BSTAGES), (uint32_t)(k / AR_BSTAGES) & 1u)) atomicExch(P.err, 4);
      if (it > 0) {
        const int qlast = (it - 1) / (nt * nk);   // the last modulus whose A blocks were issued
        for (int kb = 0; kb < nk; ++kb)
          if (!mbar_wait(afull0 + 8 * kb, (uint32_t)qlast & 1u)) atomicExch(P.err, 4);
      }
    }
  } else if (warp == EPI_WARPS + 1) {
    if (lane == 0) {   // ---- MMA issuer: A MN-major (bit 15), u8 x u8 -> int32
      const uint32_t idesc = (2u << 4) | (1u << 15) | ((uint32_t)(TN >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);
      bool ok = true;
      int it = 0, tile = 0;
      for (int q = 0; q < P.n && ok; ++q)
        for (int t = 0; t < nt && ok; ++t, ++tile) {
          const int buf = tile & 1, use = tile >> 1;
          if (use > 0 && !mbar_wait(acce0 + 8 * buf, (uint32_t)(use - 1) & 1u)) { ok = false; break; }
          tc_fence_after();
          const uint32_t d = tmem + (uint32_t)(buf * TN);
          for (int kb = 0; kb < nk; ++kb) {
            if (t == 0 && !mbar_wait(afull0 + 8 * kb, (uint32_t)q & 1u)) { ok = false; break; }
            const int s = it % AR_BSTAGES;
            if (!mbar_wait(bfull0 + 8 * s, (uint32_t)(it / AR_BSTAGES) & 1u)) { ok = false; break; }
            tc_fence_after();
            const uint64_t ad = sw128_desc(smem_u32(aslots + (size_t)kb * A_TILE));
            const uint64_t bd = sw128_desc(smem_u32(bring + (size_t)s * B_TILE));
#pragma unroll
            for (int kk = 0; kk < TK / 32; ++kk)
              mma_i8(d, ad + 256 * kk, bd + 2 * kk, idesc, (kb != 0 || kk != 0) ? 1u : 0u);
            mma_commit(bempty0 + 8 * s);
            if (t == nt - 1) mma_commit(aempty0 + 8 * kb);   // slot kb free once these MMAs complete
            ++it;
          }
          mma_commit(accf0 + 8 * buf);
        }
      if (!ok) atomicExch(P.err, 2);
    }
  } else {
    // ---- epilogue: as crt_kernel's, tile after tile
    const int q4 = warp & 3, ch = warp >> 2;
    const int i = m0 + q4 * 32 + lane;
    const bool row_ok = i < P.M;
    bool ok = true;
    int tile = 0;
    for (int q = 0; q < P.n && ok; ++q) {
      const uint32_t p = (uint32_t)P.p[q], c16 = (uint32_t)P.c16[q], magic = P.magic[q];
      uint8_t* o = P.out + (size_t)q * (size_t)P.N * P.Mp + i;
      for (int t = 0; t < nt; ++t, ++tile) {
        const int buf = tile & 1, use = tile >> 1;
        if (!mbar_wait(accf0 + 8 * buf, (uint32_t)use & 1u)) { ok = false; break; }
        tc_fence_after();
#pragma unroll 1
        for (int c = 0; c < EPI_COLS / 16; ++c) {
          uint32_t v[16];
          tmem_ld16(tmem + ((uint32_t)(q4 * 32) << 16) + (uint32_t)(buf * TN + ch * EPI_COLS + c * 16), v);
          const int j0 = t * TN + ch * EPI_COLS + c * 16;
          const int jn = row_ok ? min(16, P.N - j0) : 0;
          uint8_t* oc = o + (size_t)j0 * P.Mp;
#pragma unroll
          for (int e = 0; e < 16; ++e) {
            const uint32_t x = (v[e] >> 16) * c16 + (v[e] & 0xFFFFu);
            const uint32_t r = x - __umulhi(x, magic) * p;
            if (e < jn) oc[(size_t)e * P.Mp] = (uint8_t)r;
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(acce0 + 8 * buf);
      }
    }
    if (!ok && lane == 0) atomicExch(P.err, 3);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
  }
}

// ---- the product fused with its reconstruction --------------------------
// For products with one K-split (K <= 2^15), one CTA owns a 128 x TNF output
// tile over every modulus: the MMAs of modulus q run into one of two TMEM
// accumulators while the epilogue warps reduce the other one mod p_q and add
// (T mod p_q) G_q into a 96-bit fixed-point sum per output (three
// 32-bit limbs, the carries propagated every modulus: the same value mod 2^96
// as crt_combine's 64-bit limb sums).  The two low limbs live in TMEM beside
// the accumulators (2 x 128 + 2 x 128 = 512 columns), the high limb in
// registers.  After the last modulus the centred fraction is scaled as
// crt_combine scales it and written as FP64: the product's residues never
// leave the SM, and the result equals crt_product + crt_combine bit for bit.
constexpr int TNF = 128;
constexpr int FSTAGES = 6;
constexpr int FB_TILE = TNF * TK;
constexpr int FSTAGE_BYTES = A_TILE + FB_TILE;   // 32 KB
constexpr int FSMEM_BYTES = FSTAGES * FSTAGE_BYTES + 1024 + 256;
constexpr int FEPI_COLS = TNF / (EPI_WARPS / 4);   // 32 columns per epilogue warp
constexpr uint32_t FTMEM_COLS = 512;               // accumulators [0, 2 TNF), limbs 0 and 1 [2 TNF, 4 TNF)
constexpr uint32_t LIMB0 = 2 * TNF, LIMB1 = 3 * TNF;

struct FusedArgs {
  double* C;
  long ldc;
  int M, N, kblocks;
  const double* sb;   // per-column scales of the product
  double scale;       // M 2^(-128 - shift)
  double alpha;
  int* err;
};

// One 8-column batch of modulus Q: r = T mod p_Q from the int32 accumulator
// (as the unfused epilogue reduces it), S += r G_Q (mod 2^96, the top three
// limbs of G_Q = floor(2^128 ((M / p)^-1 mod p) / p)).
// The accumulator of u8 x u8 products over at most 2^15 terms is a
// non-negative int32 below 2^31: (a >> 16) c16 + (a & 0xFFFF) < 2^24 is
// congruent to it, and its multiply-high quotient by p is exact, so r is
// T mod p in [0, p) -- the residue the two-pass epilogue stores.
template <int Q, int NM>
__device__ __forceinline__ void fused_add8(const uint32_t (&v)[8], uint32_t (&s0)[8], uint32_t (&s1)[8],
                                           uint32_t* s2) {
  using K = ModK<Q, NM>;
  constexpr int p = MODULI[Q];
  constexpr uint32_t c16 = 65536u % p;
  constexpr uint32_t magic = (uint32_t)((((uint64_t)1 << 32) + p - 1) / p);
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    const uint32_t a = v[e];
    const uint32_t x = (a >> 16) * c16 + (a & 0xFFFFu);
    const uint32_t r = x - __umulhi(x, magic) * (uint32_t)p;
    uint64_t t = (uint64_t)r * K::G1 + s0[e];
    s0[e] = (uint32_t)t;
    t = (uint64_t)r * K::G2 + s1[e] + (t >> 32);
    s1[e] = (uint32_t)t;
    s2[e] += r * K::G3 + (uint32_t)(t >> 32);
  }
}

// Modulus Q's accumulator (buffer Q % 2) folded into the state of this warp's
// 32 lanes x FEPI_COLS columns; the buffer is handed back to the MMA warp.
template <int NM, int Q>
__device__ __forceinline__ void fused_drain(uint32_t tmem, uint32_t accf0, uint32_t acce0, int lane, uint32_t col,
                                            uint32_t (&s2)[FEPI_COLS], bool& ok) {
  constexpr int buf = Q & 1, use = Q >> 1;
  if (!ok) return;
  if (!mbar_wait(accf0 + 8 * buf, (uint32_t)use & 1u)) { ok = false; return; }
  tc_fence_after();
#pragma unroll
  for (int b = 0; b < FEPI_COLS / 8; ++b) {
    uint32_t v[8], s0[8], s1[8];
    tmem_ld8_nowait(tmem + col + (uint32_t)(buf * TNF + 8 * b), v);
    if (Q > 0) {
      tmem_ld8_nowait(tmem + col + LIMB0 + (uint32_t)(8 * b), s0);
      tmem_ld8_nowait(tmem + col + LIMB1 + (uint32_t)(8 * b), s1);
    } else {
#pragma unroll
      for (int e = 0; e < 8; ++e) s0[e] = s1[e] = 0u;
    }
    tmem_wait_ld();
    fused_add8<Q, NM>(v, s0, s1, s2 + 8 * b);
    tmem_st8(tmem + col + LIMB0 + (uint32_t)(8 * b), s0);
    tmem_st8(tmem + col + LIMB1 + (uint32_t)(8 * b), s1);
  }
  tmem_wait_st();
  tc_fence_before();
  __syncwarp();
  if (lane == 0) mbar_arrive(acce0 + 8 * buf);
}

template <int NM, int... Q>
__device__ __forceinline__ void fused_drain_all(uint32_t tmem, uint32_t accf0, uint32_t acce0, int lane, uint32_t col,
                                                uint32_t (&s2)[FEPI_COLS], bool& ok,
                                                std::integer_sequence<int, Q...>) {
  (fused_drain<NM, Q>(tmem, accf0, acce0, lane, col, s2, ok), ...);
}

template <bool AMN, int NM>
__global__ void __launch_bounds__(THREADS, 1)
crt_fused_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, FusedArgs P) {
  const int n0 = blockIdx.x * TNF, m0 = blockIdx.y * TM;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* bars = (uint64_t*)(smem + FSTAGES * FSTAGE_BYTES);
  uint32_t* tmem_slot = (uint32_t*)(bars + 2 * FSTAGES + 4);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nk = P.kblocks;
  const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + FSTAGES);
  const uint32_t accf0 = smem_u32(bars + 2 * FSTAGES), acce0 = smem_u32(bars + 2 * FSTAGES + 2);
  if (threadIdx.x == 0) {
    for (int s = 0; s < FSTAGES; ++s) {
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
                 "r"(FTMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int total = NM * nk;

  if (warp == EPI_WARPS) {
    if (lane == 0) {   // ---- TMA producer: modulus after modulus, K-block after K-block
      int issued = 0;
      bool ok = true;
      for (int it = 0; it < total; ++it) {
        const int q = it / nk, kb = it - q * nk;
        const int s = it % FSTAGES;
        const uint32_t ph = (uint32_t)(it / FSTAGES) & 1u;
        if (!mbar_wait(empty0 + 8 * s, ph ^ 1u)) { ok = false; break; }
        const uint32_t fb = full0 + 8 * s;
        mbar_expect_tx(fb, (uint32_t)FSTAGE_BYTES);
        const uint32_t st = smem_u32(smem + (size_t)s * FSTAGE_BYTES);
        const int kx = kb * TK;
        if (AMN)
          tma_load_3d(st, &tmA, fb, m0, kx, q);
        else
          tma_load_3d(st, &tmA, fb, kx, m0, q);
        tma_load_3d(st + A_TILE, &tmB, fb, kx, n0, q);
        ++issued;
      }
      if (!ok) atomicExch(P.err, 1);
      for (int it = max(0, issued - FSTAGES); it < issued; ++it)
        if (!mbar_wait(full0 + 8 * (it % FSTAGES), (uint32_t)(it / FSTAGES) & 1u)) atomicExch(P.err, 4);
    }
  } else if (warp == EPI_WARPS + 1) {
    if (lane == 0) {   // ---- MMA issuer: u8 x u8 -> int32, 128 x 128 x 32 per instruction
      const uint32_t idesc = (2u << 4) | ((AMN ? 1u : 0u) << 15) | ((uint32_t)(TNF >> 3) << 17) |
                             ((uint32_t)(TM >> 4) << 24);
      bool ok = true;
      for (int q = 0; q < NM && ok; ++q) {
        const int buf = q & 1, use = q >> 1;
        if (use > 0 && !mbar_wait(acce0 + 8 * buf, (uint32_t)(use - 1) & 1u)) { ok = false; break; }
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(buf * TNF);
        for (int kb = 0; kb < nk; ++kb) {
          const int it = q * nk + kb;
          const int s = it % FSTAGES;
          if (!mbar_wait(full0 + 8 * s, (uint32_t)(it / FSTAGES) & 1u)) { ok = false; break; }
          tc_fence_after();
          const uint32_t st = smem_u32(smem + (size_t)s * FSTAGE_BYTES);
          const uint64_t ad = sw128_desc(st), bd = sw128_desc(st + A_TILE);
#pragma unroll
          for (int kk = 0; kk < TK / 32; ++kk)
            mma_i8(d, ad + (AMN ? 256 : 2) * kk, bd + 2 * kk, idesc, (kb != 0 || kk != 0) ? 1u : 0u);
          mma_commit(empty0 + 8 * s);
        }
        mma_commit(accf0 + 8 * buf);
      }
      if (!ok) atomicExch(P.err, 2);
    }
  } else {
    // ---- epilogue: TMEM lanes 32 (warp % 4).. (rows), columns FEPI_COLS (warp / 4).. of
    //      the tile; the fraction of every output accumulates over the moduli
    const int q4 = warp & 3, ch = warp >> 2;
    uint32_t s2[FEPI_COLS];
#pragma unroll
    for (int e = 0; e < FEPI_COLS; ++e) s2[e] = 0u;
    bool ok = true;
    const uint32_t col = ((uint32_t)(q4 * 32) << 16) + (uint32_t)(ch * FEPI_COLS);
    fused_drain_all<NM>(tmem, accf0, acce0, lane, col, s2, ok, std::make_integer_sequence<int, NM>{});
    if (!ok) {
      if (lane == 0) atomicExch(P.err, 3);
    } else {
      const int i = m0 + q4 * 32 + lane;
#pragma unroll
      for (int b = 0; b < FEPI_COLS / 8; ++b) {
        uint32_t s0[8], s1[8];
        tmem_ld8_nowait(tmem + col + LIMB0 + (uint32_t)(8 * b), s0);
        tmem_ld8_nowait(tmem + col + LIMB1 + (uint32_t)(8 * b), s1);
        tmem_wait_ld();
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const int j = n0 + ch * FEPI_COLS + 8 * b + e;
          if (i < P.M && j < P.N) {
            const uint64_t hi = (uint64_t)s1[e] | ((uint64_t)s2[8 * b + e] << 32), lo = (uint64_t)s0[e] << 32;
            const double v = fixed_to_double(hi, lo) * (P.sb[j] * P.scale);
            P.C[i + (long)j * P.ldc] = P.alpha * v;
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(FTMEM_COLS));
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

// ---- host tables -------------------------------------------------------------

int inverse_mod(int a, int p) {   // a^-1 mod p, gcd(a, p) = 1
  int t = 0, nt = 1, r = p, nr = a % p;
  while (nr) {
    const int q = r / nr;
    int x = t - q * nt;
    t = nt;
    nt = x;
    x = r - q * nr;
    r = nr;
    nr = x;
  }
  return t < 0 ? t + p : t;
}

Mods make_mods(int n) {
  Mods m{};
  m.n = n;
  double bits = 0.0, hi = 1.0, lo = 0.0;
  for (int q = 0; q < n; ++q) {
    const int p = MODULI[q];
    m.p[q] = p;
    m.c16[q] = 65536 % p;
    m.invf[q] = 1.0f / (float)p;
    int prod = 1;   // (M / p) mod p
    for (int r = 0; r < n; ++r)
      if (r != q) prod = (int)((long)prod * (MODULI[r] % p) % p);
    m.inv[q] = inverse_mod(prod, p);
    unsigned __int128 F = ~(unsigned __int128)0 / (unsigned)p;
    if (~(unsigned __int128)0 % (unsigned)p == (unsigned)p - 1) F += 1;   // p divides 2^128
    for (int l = 0; l < 4; ++l) m.F[q][l] = (uint32_t)(F >> (32 * l));
    // M as a double-double: (hi + lo) * p with an exact error term
    const double ph = hi * p;
    const double pe = std::fma(hi, (double)p, -ph) + lo * p;
    hi = ph + pe;
    lo = pe - (hi - ph);
    bits += std::log2((double)p);
  }
  m.mod_hi = hi;
  m.mod_lo = lo;
  m.mod_bits = bits;
  return m;
}

ModTab mod_tab(int n) {
  ModTab t{};
  t.n = n;
  for (int q = 0; q < n; ++q) {
    const int p = MODULI[q];
    t.p[q] = p;
    t.invp[q] = 1.0 / p;
  }
  return t;
}

struct Plan {
  int splits, kb_per_split, kblocks;
};

Plan plan(int M, int N, long K, int num_sms, bool upper) {
  Plan r;
  r.kblocks = (int)((K + TK - 1) / TK);
  const long tm = (M + TM - 1) / TM, tn = (N + TN - 1) / TN;
  long tiles = 0;
  for (long a = 0; a < tm; ++a)
    for (long b = 0; b < tn; ++b) tiles += (!upper || a * TM < b * TN + TN);
  const int smin = (r.kblocks + MAX_KB_PER_SPLIT - 1) / MAX_KB_PER_SPLIT;
  const int smax = std::max(smin, std::min(MAX_SPLITS, r.kblocks));
  double best = 1e300;
  int bs = smin;
  for (int s = smin; s <= smax; ++s) {
    const long waves = (tiles * s + num_sms - 1) / num_sms;
    const double cost = (double)waves * ((r.kblocks + s - 1) / s + 8) + 2.0 * s;
    if (cost < best * 0.98) { best = cost; bs = s; }
  }
  r.kb_per_split = (r.kblocks + bs - 1) / bs;
  r.splits = (r.kblocks + r.kb_per_split - 1) / r.kb_per_split;
  return r;
}

}  // namespace

#define CRT_NM_CASES(X) \
  X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17) X(18) X(19) X(20) X(21) X(22) X(23) X(24)

long crt_pitch(long K) { return (K + 15) / 16 * 16; }

int crt_moduli(int bits_a, int bits_b, long K) {
  const double need = (bits_a - 2) + (bits_b - 2) + std::log2((double)std::max(K, 1L)) + 2.0;
  double bits = 0.0;
  for (int n = 0; n < MAXMOD; ++n) {
    bits += std::log2((double)MODULI[n]);
    if (bits >= need) return std::max(n + 1, 4);   // the kernels are built for 4..24 moduli
  }
  return -1;
}

bbt_status crt_row_scales(bbt_ctx* ctx, int rows, long K, const double* X, long rs, double* scale) {
  unsigned long long* mx = ctx->ws.take<unsigned long long>(rows);
  if (!mx) return fail(ctx, BBT_ERR_NOMEM, "crt: workspace (row maxima)");
  BBT_CUDA(ctx, cudaMemsetAsync(mx, 0, (size_t)rows * 8, ctx->stream));
  ProfScope prof(ctx, BBT_PROF_CRT_PREP, 8.0 * (double)rows * K);
  if (K <= 4096) {
    rowmax_short_kernel<<<8 * ctx->num_sms, 256, 0, ctx->stream>>>(rows, K, X, rs, mx);
  } else {
    const unsigned gy = (unsigned)std::min(rows, 65535);
    rowmax_kernel<<<dim3((unsigned)((K + 8191) / 8192), gy), 256, 0, ctx->stream>>>(rows, K, X, rs, mx);
  }
  BBT_LAUNCHED(ctx);
  scale_kernel<<<(rows + 255) / 256, 256, 0, ctx->stream>>>(rows, mx, scale);
  BBT_LAUNCHED(ctx);
  return BBT_OK;   // mx stays taken until the caller releases its workspace mark
}

bbt_status crt_scales_from_max(bbt_ctx* ctx, int rows, const unsigned long long* mx, double* scale) {
  scale_kernel<<<(rows + 255) / 256, 256, 0, ctx->stream>>>(rows, mx, scale);
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

bbt_status crt_residues_rows(bbt_ctx* ctx, int rows, long K, const double* X, long rs, const double* scale, int b,
                             int n, int8_t* planes, long Kp) {
  if (b < 2 || b > 53) return fail(ctx, BBT_ERR_ARG, "crt: %d-bit integers from doubles", b);
  const long kq = (K + 3) / 4;
  const unsigned gx = (unsigned)std::min<long>((kq + 255) / 256, 4096), gy = (unsigned)std::min(rows, 65535);
  ProfScope prof(ctx, BBT_PROF_CRT_PREP, (8.0 + n) * (double)rows * K);
  switch (n) {
#define CASE(NM)                                                                                          \
  case NM:                                                                                                \
    residues_rows_kernel<NM><<<dim3(gx, gy), 256, 0, ctx->stream>>>(rows, K, X, rs, scale, b, planes, Kp); \
    break;
    CRT_NM_CASES(CASE)
#undef CASE
    default:
      return fail(ctx, BBT_ERR_ARG, "crt: %d moduli", n);
  }
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

bbt_status crt_residues_cols(bbt_ctx* ctx, int rows, long K, const double* X, long cs, const double* kscale, int b,
                             int n, int8_t* planes, long Kp) {
  if (b < 2 || b > 53) return fail(ctx, BBT_ERR_ARG, "crt: %d-bit integers from doubles", b);
  const long gy = (K + 127) / 128;
  if (gy > 65535) return fail(ctx, BBT_ERR_ARG, "crt: K=%ld too long for the column layout", K);
  const dim3 g((unsigned)((rows + 31) / 32), (unsigned)gy);
  ProfScope prof(ctx, BBT_PROF_CRT_PREP, (8.0 + n) * (double)rows * K);
  switch (n) {
#define CASE(NM)                                                                                             \
  case NM:                                                                                                   \
    residues_cols_kernel<NM><<<g, 256, 0, ctx->stream>>>(rows, K, X, cs, kscale, b, planes, Kp);             \
    break;
    CRT_NM_CASES(CASE)
#undef CASE
    default:
      return fail(ctx, BBT_ERR_ARG, "crt: %d moduli", n);
  }
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

bbt_status crt_residues_dd(bbt_ctx* ctx, int rows, long K, const double* Xh, const double* Xl, long rs,
                           const double* scale, int b, int n, int8_t* planes, long Kp) {
  if (b < 2 || b > 100) return fail(ctx, BBT_ERR_ARG, "crt: %d-bit integers from double-doubles", b);
  residues_dd_kernel<<<8 * ctx->num_sms, 256, 0, ctx->stream>>>(rows, K, Xh, Xl, rs, scale, b, mod_tab(n), planes, Kp);
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

size_t crt_product_bytes(const bbt_ctx* ctx, int M, int N, long K, int n, bool upper) {
  const int sms = ctx->num_sms > 0 ? ctx->num_sms : 148;
  const Plan pl = plan(M, N, K, sms, upper);
  return (size_t)pl.splits * n * (size_t)((M + 3) & ~3) * N + 4096;
}

namespace {
// A: K-major planes [n][M][Kp] (lda = 0) or MN-major planes [n][K][lda] (A(i, k) at k lda + i).
bbt_status crt_launch(bbt_ctx* ctx, int M, int N, long K, int n, const int8_t* RA, long lda, const int8_t* RB,
                      long Kp, bool upper, uint8_t* R, int* splits_out) {
  if (n < 1 || n > MAXMOD) return fail(ctx, BBT_ERR_ARG, "crt: %d moduli", n);
  if (M < 1 || N < 1 || K < 1) return fail(ctx, BBT_ERR_ARG, "crt: M=%d N=%d K=%ld", M, N, K);
  const bool amn = lda > 0;
  if (amn && (lda < M || lda % 16 != 0 || upper)) return fail(ctx, BBT_ERR_ARG, "crt: MN-major A, pitch %ld", lda);
  const unsigned gy = (unsigned)((M + TM - 1) / TM);
  if (gy > 65535) return fail(ctx, BBT_ERR_ARG, "crt: M=%d too large", M);
  EncodeTiled enc = encode_fn();
  if (!enc) return fail(ctx, BBT_ERR_CUDA, "crt: cuTensorMapEncodeTiled is not available");
  const Plan pl = plan(M, N, K, ctx->num_sms, upper);
  CUtensorMap ta, tb;
  {
    cuuint64_t dims[3] = {(cuuint64_t)K, (cuuint64_t)M, (cuuint64_t)n};
    cuuint64_t strides[2] = {(cuuint64_t)Kp, (cuuint64_t)Kp * M};
    cuuint32_t box[3] = {TK, TM, 1};
    if (amn) {   // i contiguous (TM bytes of it per box row), TK rows of K
      dims[0] = (cuuint64_t)M;
      dims[1] = (cuuint64_t)K;
      strides[0] = (cuuint64_t)lda;
      strides[1] = (cuuint64_t)lda * K;
      box[0] = TM;
      box[1] = TK;
    }
    const cuuint32_t es[3] = {1, 1, 1};
    if (enc(&ta, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<int8_t*>(RA), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return fail(ctx, BBT_ERR_CUDA, "crt: tensor map of A");
  }
  {
    const cuuint64_t dims[3] = {(cuuint64_t)K, (cuuint64_t)N, (cuuint64_t)n};
    const cuuint64_t strides[2] = {(cuuint64_t)Kp, (cuuint64_t)Kp * N};
    const cuuint32_t box[3] = {TK, TN, 1}, es[3] = {1, 1, 1};
    if (enc(&tb, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<int8_t*>(RB), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return fail(ctx, BBT_ERR_CUDA, "crt: tensor map of B");
  }
  // A kept in shared memory (crt_apply_kernel): MN-major A, one K-split of at
  // most AR_SLOTS blocks, and enough 128-row blocks to occupy every SM
  const bool resident = amn && pl.splits == 1 && pl.kblocks <= AR_SLOTS && (long)gy >= (long)ctx->num_sms;
  static bool attr[3] = {false, false, false};
  const int kind = resident ? 2 : (amn ? 1 : 0);
  if (!attr[kind]) {
    if (kind == 2)
      BBT_CUDA(ctx, cudaFuncSetAttribute(crt_apply_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, AR_SMEM));
    else
      BBT_CUDA(ctx, cudaFuncSetAttribute(kind == 1 ? crt_kernel<true> : crt_kernel<false>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
    attr[kind] = true;
  }
  const Mods md = make_mods(n);
  CrtArgs a;
  a.out = R;
  a.M = M;
  a.N = N;
  a.Mp = (M + 3) & ~3;
  a.kblocks = pl.kblocks;
  a.kb_per_split = pl.kb_per_split;
  a.n = n;
  a.upper = upper ? 1 : 0;
  for (int q = 0; q < n; ++q) {
    a.p[q] = md.p[q];
    a.c16[q] = md.c16[q];
    a.magic[q] = (uint32_t)((((uint64_t)1 << 32) + md.p[q] - 1) / md.p[q]);
  }
  a.err = ctx->d_flag + FLAG_SKETCH;
  ProfScope prof(ctx, BBT_PROF_CRT, (upper ? 1.0 : 2.0) * n * (double)M * N * K);   // int8 operations
  const dim3 grid((N + TN - 1) / TN, gy, pl.splits);
  if (kind == 2)
    crt_apply_kernel<<<dim3(gy), THREADS, AR_SMEM, ctx->stream>>>(ta, tb, a);
  else if (kind == 1)
    crt_kernel<true><<<grid, THREADS, SMEM_BYTES, ctx->stream>>>(ta, tb, a);
  else
    crt_kernel<false><<<grid, THREADS, SMEM_BYTES, ctx->stream>>>(ta, tb, a);
  BBT_LAUNCHED(ctx);
  *splits_out = pl.splits;
  return BBT_OK;
}
}  // namespace

namespace {
// Tensor maps of the fused kernel: A as in crt_launch, B with TNF-row boxes.
bbt_status fused_maps(bbt_ctx* ctx, int M, int N, long K, int n, const int8_t* RA, long lda, const int8_t* RB, long Kp,
                      CUtensorMap* ta, CUtensorMap* tb) {
  EncodeTiled enc = encode_fn();
  if (!enc) return fail(ctx, BBT_ERR_CUDA, "crt: cuTensorMapEncodeTiled is not available");
  const bool amn = lda > 0;
  cuuint64_t dims[3] = {(cuuint64_t)K, (cuuint64_t)M, (cuuint64_t)n};
  cuuint64_t strides[2] = {(cuuint64_t)Kp, (cuuint64_t)Kp * M};
  cuuint32_t box[3] = {TK, TM, 1};
  if (amn) {
    dims[0] = (cuuint64_t)M;
    dims[1] = (cuuint64_t)K;
    strides[0] = (cuuint64_t)lda;
    strides[1] = (cuuint64_t)lda * K;
    box[0] = TM;
    box[1] = TK;
  }
  const cuuint32_t es[3] = {1, 1, 1};
  if (enc(ta, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<int8_t*>(RA), dims, strides, box, es,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return fail(ctx, BBT_ERR_CUDA, "crt: tensor map of A (fused)");
  const cuuint64_t bd[3] = {(cuuint64_t)K, (cuuint64_t)N, (cuuint64_t)n};
  const cuuint64_t bs[2] = {(cuuint64_t)Kp, (cuuint64_t)Kp * N};
  const cuuint32_t bb[3] = {TK, TNF, 1};
  if (enc(tb, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<int8_t*>(RB), bd, bs, bb, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
          CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return fail(ctx, BBT_ERR_CUDA, "crt: tensor map of B (fused)");
  return BBT_OK;
}

template <bool AMN, int NM>
bbt_status fused_launch(bbt_ctx* ctx, const CUtensorMap& ta, const CUtensorMap& tb, const FusedArgs& a, dim3 grid) {
  static bool attr = false;
  if (!attr) {
    BBT_CUDA(ctx, cudaFuncSetAttribute(crt_fused_kernel<AMN, NM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       FSMEM_BYTES));
    attr = true;
  }
  crt_fused_kernel<AMN, NM><<<grid, THREADS, FSMEM_BYTES, ctx->stream>>>(ta, tb, a);
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}
}  // namespace

bool crt_fused_supported(long K, int n) { return K >= 1 && K <= (long)MAX_KB_PER_SPLIT * TK && n >= 16 && n <= 20; }

bbt_status crt_product_fused(bbt_ctx* ctx, int M, int N, long K, int n, const int8_t* RA, long lda, const int8_t* RB,
                             long Kp, const double* sb, int shift, double alpha, double* C, long ldc) {
  if (!crt_fused_supported(K, n)) return fail(ctx, BBT_ERR_ARG, "crt: fused product with K=%ld, %d moduli", K, n);
  if (M < 1 || N < 1) return fail(ctx, BBT_ERR_ARG, "crt: M=%d N=%d", M, N);
  const bool amn = lda > 0;
  if (amn && (lda < M || lda % 16 != 0)) return fail(ctx, BBT_ERR_ARG, "crt: MN-major A, pitch %ld", lda);
  const unsigned gy = (unsigned)((M + TM - 1) / TM);
  if (gy > 65535) return fail(ctx, BBT_ERR_ARG, "crt: M=%d too large", M);
  CUtensorMap ta, tb;
  BBT_TRY(fused_maps(ctx, M, N, K, n, RA, lda, RB, Kp, &ta, &tb));
  const Mods md = make_mods(n);
  FusedArgs a;
  a.C = C;
  a.ldc = ldc;
  a.M = M;
  a.N = N;
  a.kblocks = (int)((K + TK - 1) / TK);
  a.sb = sb;
  a.scale = std::ldexp(md.mod_hi, -128 - shift);
  a.alpha = alpha;
  a.err = ctx->d_flag + FLAG_SKETCH;
  const dim3 grid((N + TNF - 1) / TNF, gy);   // N-tiles fastest: CTAs sharing A's row block run together
  ProfScope prof(ctx, BBT_PROF_CRT, 2.0 * n * (double)M * N * K);   // int8 operations
  switch (n) {
#define CASE(NM) \
  case NM:       \
    return amn ? fused_launch<true, NM>(ctx, ta, tb, a, grid) : fused_launch<false, NM>(ctx, ta, tb, a, grid);
    CASE(16) CASE(17) CASE(18) CASE(19) CASE(20)
#undef CASE
    default:
      return fail(ctx, BBT_ERR_ARG, "crt: fused product with %d moduli", n);
  }
}

bbt_status crt_product(bbt_ctx* ctx, int M, int N, long K, int n, const int8_t* RA, const int8_t* RB, long Kp,
                       bool upper, uint8_t* R, int* splits_out) {
  return crt_launch(ctx, M, N, K, n, RA, 0, RB, Kp, upper, R, splits_out);
}

bbt_status crt_product_amn(bbt_ctx* ctx, int M, int N, long K, int n, const int8_t* RA, long lda, const int8_t* RB,
                           long Kp, uint8_t* R, int* splits_out) {
  return crt_launch(ctx, M, N, K, n, RA, lda, RB, Kp, false, R, splits_out);
}

namespace {
CombArgs comb_args(const uint8_t* R, int M, int N, int n, int splits, bool upper) {
  const Mods md = make_mods(n);
  CombArgs c;
  c.R = R;
  c.M = M;
  c.N = N;
  c.Mp = (M + 3) & ~3;
  c.splits = splits;
  c.upper = upper ? 1 : 0;
  c.mod_hi = md.mod_hi;
  c.mod_lo = md.mod_lo;
  return c;
}
}  // namespace

bbt_status crt_combine(bbt_ctx* ctx, int M, int N, int n, int splits, const uint8_t* R, bool upper, const double* sa,
                       const double* sb, int shift, double alpha, double beta, double* C, long ldc) {
  const dim3 g((unsigned)std::min((M + 1023) / 1024, 1024), (unsigned)std::min(N, 65535));   // 4 outputs a thread
  const CombArgs A = comb_args(R, M, N, n, splits, upper);
  // M 2^(-128 - shift): a power of two times the moduli's product, normal for every shift used
  const double scale = std::ldexp(A.mod_hi, -128 - shift);
  ProfScope prof(ctx, BBT_PROF_CRT_COMBINE, ((double)n * splits + 8.0) * (double)M * N);
  switch (n) {
#define CASE(NM)                                                                                   \
  case NM:                                                                                         \
    if (splits > 1)                                                                                \
      combine_kernel<NM, true><<<g, 256, 0, ctx->stream>>>(A, sa, sb, scale, alpha, beta, C, ldc);  \
    else                                                                                           \
      combine_kernel<NM, false><<<g, 256, 0, ctx->stream>>>(A, sa, sb, scale, alpha, beta, C, ldc); \
    break;
    CRT_NM_CASES(CASE)
#undef CASE
    default:
      return fail(ctx, BBT_ERR_ARG, "crt: %d moduli", n);
  }
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

bbt_status crt_combine_dd(bbt_ctx* ctx, int M, int N, int n, int splits, const uint8_t* R, bool upper,
                          const double* sa, const double* sb, int shift, double* Ch, double* Cl, long ldc) {
  const dim3 g((unsigned)std::min((M + 1023) / 1024, 1024), (unsigned)std::min(N, 65535));   // 4 outputs a thread
  const CombArgs A = comb_args(R, M, N, n, splits, upper);
  ProfScope prof(ctx, BBT_PROF_CRT_COMBINE, ((double)n * splits + 8.0) * (double)M * N);
  switch (n) {
#define CASE(NM)                                                                                   \
  case NM:                                                                                         \
    combine_dd_kernel<NM><<<g, 256, 0, ctx->stream>>>(A, sa, sb, shift, Ch, Cl, ldc);              \
    break;
    CRT_NM_CASES(CASE)
#undef CASE
    default:
      return fail(ctx, BBT_ERR_ARG, "crt: %d moduli", n);
  }
  BBT_LAUNCHED(ctx);
  return BBT_OK;
}

namespace {
// K-chunk of gemm_crt's residue planes: all of K when they fit the cap, else
// equal chunks, multiples of 2^15 columns (one K-split each at most).
constexpr size_t CRT_CHUNK_DEFAULT = (size_t)6 << 30;
long crt_k_chunk(int rows, long K, int n) {
  const size_t cap = long_chunk_bytes(CRT_CHUNK_DEFAULT);
  const size_t full = (size_t)n * rows * crt_pitch(K);
  if (full <= cap) return K;
  long c = (long)(cap / ((size_t)n * rows)) / 32768 * 32768;
  c = std::max(c, 32768L);
  const long chunks = (K + c - 1) / c;
  return ((K + chunks - 1) / chunks + 32767) / 32768 * 32768;
}
size_t chunked_product_bytes(const bbt_ctx* ctx, int M, int N, long K, int n, bool upper, long kc) {
  size_t b = 0;
  for (long k0 = 0; k0 < K; k0 += kc) b += crt_product_bytes(ctx, M, N, std::min(kc, K - k0), n, upper) - 4096;
  return b + 4096;
}
}  // namespace

size_t crt_gemm_workspace_bytes(const bbt_ctx* ctx, int M, int N, long K, int bits, bool same, bool upper) {
  const int n = crt_moduli(bits, bits, K);
  if (n < 1) return 0;
  const long kc = crt_k_chunk(same ? M : M + N, K, n);
  const long Kp = crt_pitch(kc);
  return (size_t)n * (same ? M : M + N) * Kp + chunked_product_bytes(ctx, M, N, K, n, upper, kc) +
         (size_t)(M + N) * 16 + (size_t)std::max(M, N) * 8 + 8192;
}

// The Gram matrix of a long operand: K long enough for the CRT product (one
// exact int8 GEMM per modulus, 128 x 256 tiles) to beat the slice pairs.
bool crt_worthwhile(int M, int N, long K) { return M >= 128 && N >= 128 && K >= 16384 && (double)M * N * K >= 4e9; }

// C = alpha A B^T + beta C for strided FP64 operands (each with a unit stride
// in its row or its K index), every operand rounded to b bits per row.
bbt_status gemm_crt(bbt_ctx* ctx, int M, int N, long K, double alpha, const double* A, long rsA, long csA,
                    const double* B, long rsB, long csB, double beta, double* C, long ldc, bool same, bool upper,
                    int bits) {
  const int n = crt_moduli(bits, bits, K);
  if (n < 1) return fail(ctx, BBT_ERR_ARG, "crt: %d bits over K=%ld needs too many moduli", bits, K);
  if (csA != 1 || (!same && csB != 1))   // row scales need each row contiguous along K
    return fail(ctx, BBT_ERR_ARG, "crt: operands must be contiguous along K");
  // long K: residue planes in K-chunks (scales over all of K first), the
  // chunks' K-splits side by side, summed by one reconstruction
  const long kc = crt_k_chunk(same ? M : M + N, K, n);
  const long Kp = crt_pitch(kc);
  const size_t mark = ctx->ws.top;
  int8_t* RA = ctx->ws.take<int8_t>((size_t)n * M * Kp);
  int8_t* RB = same ? RA : ctx->ws.take<int8_t>((size_t)n * N * Kp);
  double* sa = ctx->ws.take<double>(M);
  double* sb = same ? sa : ctx->ws.take<double>(N);
  uint8_t* R = ctx->ws.take<uint8_t>(chunked_product_bytes(ctx, M, N, K, n, upper, kc));
  if (!R) return fail(ctx, BBT_ERR_NOMEM, "crt: workspace");
  {
    const size_t m2 = ctx->ws.top;
    BBT_TRY(crt_row_scales(ctx, M, K, A, rsA, sa));
    ctx->ws.top = m2;
    if (!same) BBT_TRY(crt_row_scales(ctx, N, K, B, rsB, sb));
    ctx->ws.top = m2;
  }
  const size_t split_bytes = (size_t)n * ((M + 3) & ~3) * N;
  int splits = 0;
  for (long k0 = 0; k0 < K; k0 += kc) {
    const long Kc = std::min(kc, K - k0);
    BBT_TRY(crt_residues_rows(ctx, M, Kc, A + k0, rsA, sa, bits, n, RA, Kp));
    if (!same) BBT_TRY(crt_residues_rows(ctx, N, Kc, B + k0, rsB, sb, bits, n, RB, Kp));
    int sp = 1;
    BBT_TRY(crt_product(ctx, M, N, Kc, n, RA, RB, Kp, upper, R + (size_t)splits * split_bytes, &sp));
    splits += sp;
  }
  BBT_TRY(crt_combine(ctx, M, N, n, splits, R, upper, sa, sb, 2 * (bits - 1), alpha, beta, C, ldc));
  ctx->ws.top = mark;
  return BBT_OK;
}

}  // namespace bbt
