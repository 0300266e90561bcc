// The reference's own C++ API (Excalibur include/bbtsvd.hpp:22-47), exported
// with identical signatures (and therefore identical mangled names) so that
// the reference's DecentralizedClient links libexcalibur_b200.so in place of
// src/bbtsvd.cpp.  Host pointers in and out, as in the reference; each call
// copies to a process-wide device context, runs the kernels, copies back.
// The masks draw their random tables on the host with the same calls as the
// reference, so glibc's rand() state after a call is the reference's.
//
// Functions the reference declares but never calls from client.cpp (the dead
// mask variants and the opt_control 0/2 dense mask) abort with a message
// instead of silently computing on the CPU.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "internal.h"

namespace {

bbt_ctx* g_ctx = nullptr;
std::mutex g_mu;

bbt_ctx* ctx() {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_ctx) {
    int dev = 0;
    if (const char* e = getenv("BBT_DEVICE")) dev = atoi(e);
    if (bbt_create(&g_ctx, dev) != BBT_OK) {
      fprintf(stderr, "libexcalibur_b200: no usable CUDA device %d (there is no CPU fallback)\n", dev);
      abort();
    }
  }
  return g_ctx;
}

[[noreturn]] void die(const char* what, bbt_status s) {
  fprintf(stderr, "libexcalibur_b200: %s failed: %s (%s)\n", what, bbt_status_string(s),
          g_ctx ? bbt_last_error(g_ctx) : "");
  abort();
}

[[noreturn]] void not_provided(const char* fn) {
  fprintf(stderr,
          "libexcalibur_b200: %s is not provided (declared by bbtsvd.hpp but not on the path "
          "DecentralizedClient::run() takes with opt_control 1/3)\n",
          fn);
  abort();
}

// RAII device copy of a host array.
struct Dev {
  double* p = nullptr;
  size_t n = 0;
  Dev(const double* h, size_t count) : n(count) {
    if (cudaMalloc(&p, (count ? count : 1) * sizeof(double)) != cudaSuccess) die("cudaMalloc", BBT_ERR_NOMEM);
    if (h && count && cudaMemcpy(p, h, count * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
      die("cudaMemcpy", BBT_ERR_CUDA);
  }
  void back(double* h, size_t count) const {
    if (count && cudaMemcpy(h, p, count * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
      die("cudaMemcpy", BBT_ERR_CUDA);
  }
  ~Dev() { cudaFree(p); }
};

}  // namespace

// ---- the reference's structs (bbtsvd.hpp:11-20), same layout ----
struct BISECTION_SV {
  double low;
  int nc_low;
  double high;
  int nc_high;
};
struct SquareMaskConvert {
  size_t k, m, n, remain;
};

int negative_count(int n, double* x_diagonal, double* x_upper_diagonal, double mu) {
  bbt_ctx* c = ctx();
  Dev a(x_diagonal, n), b(x_upper_diagonal, n > 1 ? n - 1 : 0), m(&mu, 1);
  int* dc = nullptr;
  if (cudaMalloc(&dc, sizeof(int)) != cudaSuccess) die("cudaMalloc", BBT_ERR_NOMEM);
  bbt_status s = bbt_negative_count(c, n, a.p, b.p, m.p, 1, dc);
  if (s != BBT_OK) die("negative_count", s);
  int h = 0;
  cudaMemcpy(&h, dc, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(dc);
  return h;
}

void bisection_singular_values(int n, double* x_diagonal, double* x_upper_diagonal, double a, double b, double tol,
                               int top_k, double* sigma, int* sigma_count) {
  bbt_ctx* c = ctx();
  Dev da(x_diagonal, n), db(x_upper_diagonal, n > 1 ? n - 1 : 0), ds(nullptr, n);
  int cnt = 0;
  bbt_status s = bbt_bisection(c, n, da.p, db.p, a, b, tol, top_k, ds.p, &cnt);
  if (s != BBT_OK) die("bisection_singular_values", s);
  ds.back(sigma, cnt);
  *sigma_count = cnt;
}

void two_side_singular_vectors_twisted_factorization(int n, int omege_count, double* omege, double* x_diagonal,
                                                     double* x_upper_diagonal, double* u, double* v) {
  bbt_ctx* c = ctx();
  Dev ds(omege, omege_count), da(x_diagonal, n), db(x_upper_diagonal, n > 1 ? n - 1 : 0);
  Dev dU(nullptr, (size_t)n * omege_count), dV(nullptr, (size_t)n * omege_count);
  bbt_status s = bbt_twisted_vectors(c, n, omege_count, ds.p, da.p, db.p, dU.p, dV.p);
  if (s != BBT_OK) die("two_side_singular_vectors_twisted_factorization", s);
  dU.back(u, (size_t)n * omege_count);
  dV.back(v, (size_t)n * omege_count);
}

void bidiagonal_bisection_twisted_svd(int k, double* alpha, double* beta, double* bidiagonal_u,
                                      double* bidiagonal_v, double* sigma, int top_k) {
  bbt_ctx* c = ctx();
  Dev da(alpha, k), db(beta, k > 1 ? k - 1 : 0);
  Dev dU(nullptr, (size_t)k * top_k), dV(nullptr, (size_t)k * top_k), ds(nullptr, top_k);
  bbt_status s = bbt_bidiagonal_svd(c, k, da.p, db.p, dU.p, dV.p, ds.p, top_k);
  if (s != BBT_OK) die("bidiagonal_bisection_twisted_svd", s);   // the reference asserts (bbtsvd.cpp:938)
  dU.back(bidiagonal_u, (size_t)k * top_k);
  dV.back(bidiagonal_v, (size_t)k * top_k);
  ds.back(sigma, top_k);
}

// Callee-allocating overloads (bbtsvd.cpp:878-930): every singular value
// the bisection finds, vectors allocated with new[].
void bidiagonal_bisection_twisted_svd(int k, double* alpha, double* beta, double** bidiagonal_u,
                                      double** bidiagonal_v, double** sigma, int* sigma_count) {
  bbt_ctx* c = ctx();
  Dev da(alpha, k), db(beta, k > 1 ? k - 1 : 0), ds(nullptr, k);
  *sigma = new double[k]();
  std::vector<double> hb(1);
  // bound = ||alpha||^2 + ||beta||^2 with the library's norm
  {
    Dev bound(nullptr, 1);
    bbt_status s = bbt::bidiag_bound(c, k, da.p, db.p, bound.p);
    if (s != BBT_OK) die("bidiagonal_bisection_twisted_svd", s);
    cudaStreamSynchronize(c->stream);
    bound.back(hb.data(), 1);
  }
  int cnt = 0;
  bbt_status s = bbt_bisection(c, k, da.p, db.p, 0.0, hb[0], 1e-20, k, ds.p, &cnt);
  if (s != BBT_OK) die("bidiagonal_bisection_twisted_svd", s);
  ds.back(*sigma, cnt);
  *sigma_count = cnt;
  *bidiagonal_u = new double[(size_t)k * (cnt > 0 ? cnt : 1)]();
  *bidiagonal_v = new double[(size_t)k * (cnt > 0 ? cnt : 1)]();
  if (cnt == 0) return;
  Dev dU(nullptr, (size_t)k * cnt), dV(nullptr, (size_t)k * cnt);
  s = bbt::twisted(c, k, cnt, ds.p, da.p, db.p, dU.p, cnt, dV.p, true);
  if (s == BBT_OK) s = bbt_synchronize(c);
  if (s != BBT_OK) die("bidiagonal_bisection_twisted_svd", s);
  dU.back(*bidiagonal_u, (size_t)k * cnt);
  dV.back(*bidiagonal_v, (size_t)k * cnt);
}

void bidiagonal_bisection_twisted_svd(int k, double* alpha, double* beta, double** bidiagonal_u,
                                      double** bidiagonal_v, double** sigma, int* sigma_count, bool) {
  bidiagonal_bisection_twisted_svd(k, alpha, beta, bidiagonal_u, bidiagonal_v, sigma, sigma_count);
}

void givens_mask_cache_optimized_parallel_with_simd(size_t m, size_t n, size_t mask_times, double* x, bool mask,
                                                    bool is_left, unsigned int seed) {
  bbt_ctx* c = ctx();
  Dev dx(x, m * n);
  bbt_status s = bbt_givens_mask(c, m, n, mask_times, dx.p, mask, is_left, seed);
  if (s == BBT_OK) s = bbt_synchronize(c);
  if (s != BBT_OK) die("givens_mask_cache_optimized_parallel_with_simd", s);
  dx.back(x, m * n);
}

void block_shift_mask(size_t m, size_t n, size_t mask_times, double* x, bool mask, bool is_left,
                      unsigned int seed) {
  bbt_ctx* c = ctx();
  Dev dx(x, m * n);
  bbt_status s = bbt_block_shift_mask(c, m, n, mask_times, dx.p, mask, is_left, seed);
  if (s == BBT_OK) s = bbt_synchronize(c);
  if (s != BBT_OK) die("block_shift_mask", s);
  dx.back(x, m * n);
}

// Shape planner of the large-k mask path (bbtsvd.cpp:166-188): integer
// host logic, same rule as the device path uses.
void find_best_convert(struct SquareMaskConvert* smc) {
  const size_t lim = 10000;
  if (smc->k > lim * lim) { fprintf(stderr, "find_best_convert: k too large\n"); abort(); }
  for (;;) {
    const size_t kk = smc->k - smc->remain;
    size_t bm = kk, bn = 1;
    for (size_t i = lim; i > 1; --i) {
      if (kk % i) continue;
      const size_t q = kk / i;
      if (i > q && q < lim && q > 1 && (i - q) < (bm - bn) && ((double)i / (double)q) < 2) { bm = i; bn = q; }
    }
    if (bm < lim) { smc->m = bm; smc->n = bn; return; }
    smc->remain += 1;
  }
}

// ---- declared by bbtsvd.hpp, not on the run() path (see file comment) ----
void ldl_decomposition(int, double*, double*, double*, double*) { not_provided("ldl_decomposition"); }
void inverse_iteration(int, int, double*, double*, double*, int) { not_provided("inverse_iteration"); }
void dstqds(int, double*, double*, double, double*, double*, double*) { not_provided("dstqds"); }
void dpqds(int, double*, double*, double, double*, double*, double*) { not_provided("dpqds"); }
void one_pair_singular_vector_twisted_factorization(int, int, double, double*, double*, double*, double*, double*,
                                                    double*) {
  not_provided("one_pair_singular_vector_twisted_factorization");
}
void generate_house(int, double*, int, double*) { not_provided("generate_house"); }
void house_mask(size_t, size_t, size_t, double*, bool, bool, unsigned int) { not_provided("house_mask"); }
void mmap_drot(size_t, double*, size_t, double*, size_t, double, double) { not_provided("mmap_drot"); }
void householder_reflector_mask(size_t, size_t, size_t, double*, bool, bool, unsigned int) {
  not_provided("householder_reflector_mask");
}
void naive_givens_mask_parallel(size_t, size_t, size_t, double*, bool, bool, unsigned int) {
  not_provided("naive_givens_mask_parallel");
}
void givens_mask_cache_optimized_parallel(size_t, size_t, size_t, double*, bool, bool, unsigned int) {
  not_provided("givens_mask_cache_optimized_parallel");
}
void generate_random_orthogonal_matrix(int, size_t, double*, double*, unsigned int) {
  not_provided("generate_random_orthogonal_matrix");
}
void generate_random_orthogonal_matrix(size_t, size_t, double*, unsigned int) {
  not_provided("generate_random_orthogonal_matrix");
}
void shuffle_matrix(size_t, size_t, double*, unsigned int, bool, bool) { not_provided("shuffle_matrix"); }
void block_mask(size_t, size_t, size_t, double*, bool, bool, unsigned int) { not_provided("block_mask"); }
void shuffle_block_mask(size_t, size_t, size_t, int, double*, bool, bool, unsigned int) {
  not_provided("shuffle_block_mask");
}
