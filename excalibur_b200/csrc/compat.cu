// The reference's own C++ API (Excalibur include/bbtsvd.hpp:22-47), exported
// with identical signatures (and therefore identical mangled names) so that
// the reference's DecentralizedClient links libexcalibur_b200.so in place of
// src/bbtsvd.cpp.  Host pointers in and out, as in the reference; each call
// copies to a process-wide device context, runs the kernels, copies back.
// The masks draw their random tables on the host with the same calls as the
// reference, so glibc's rand() state after a call is the reference's.
//
// The masks off the opt_control 1/3 path (the dense masks of opt_control
// 0/2 and the variants the reference declares but never calls) run on the
// GPU as well; where a size is outside what they provide they abort with a
// message instead of computing on the CPU.  The random orthogonal matrix
// generators run the reference's LAPACK calls through the LAPACK the process
// links (they are random-number generation, not arithmetic this library
// accelerates).
#include <cuda_runtime.h>

#include <dlfcn.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <random>
#include <string>
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

// RAII device copy of a host array.  The copies run on the context's stream
// (non-blocking), in order with the kernels: in, kernels, out, then a wait.
struct Dev {
  double* p = nullptr;
  size_t n = 0;
  Dev(const double* h, size_t count) : n(count) {
    if (cudaMalloc(&p, (count ? count : 1) * sizeof(double)) != cudaSuccess) die("cudaMalloc", BBT_ERR_NOMEM);
    if (h && count &&
        cudaMemcpyAsync(p, h, count * sizeof(double), cudaMemcpyHostToDevice, g_ctx->stream) != cudaSuccess)
      die("cudaMemcpyAsync", BBT_ERR_CUDA);
  }
  void back(double* h, size_t count) const {
    if (count && (cudaMemcpyAsync(h, p, count * sizeof(double), cudaMemcpyDeviceToHost, g_ctx->stream) != cudaSuccess ||
                  cudaStreamSynchronize(g_ctx->stream) != cudaSuccess))
      die("cudaMemcpyAsync", BBT_ERR_CUDA);
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
  if (cudaMemcpyAsync(&h, dc, sizeof(int), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess)
    die("negative_count", BBT_ERR_CUDA);
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

// ---- the qd / twisted-factorisation steps and the small vector helpers ----
// (bbtsvd.cpp:54-136, 149-164, 970-978).  Each is an O(n) recurrence or an
// elementwise rotation, run on the device (one thread for a recurrence) in
// the reference's order of operations, every product and sum rounded
// separately; host arrays are staged as for the functions above.
namespace {

#define MUL __dmul_rn
#define DIV __ddiv_rn
#define ADD __dadd_rn
#define SUB __dsub_rn

// bbtsvd.cpp:73-81
__global__ void dstqds_kernel(int n, const double* l, const double* d, double tau, double* lp, double* dp,
                              double* s) {
  if (blockIdx.x || threadIdx.x) return;
  double si = -tau;
  s[0] = si;
  for (int i = 0; i + 1 < n; ++i) {
    const double dpi = ADD(d[i], si);
    dp[i] = dpi;
    const double lpi = DIV(MUL(d[i], l[i]), dpi);
    lp[i] = lpi;
    si = SUB(MUL(MUL(lpi, l[i]), si), tau);
    s[i + 1] = si;
  }
  dp[n - 1] = ADD(d[n - 1], si);
}

// bbtsvd.cpp:83-91
__global__ void dpqds_kernel(int n, const double* l, const double* d, double tau, double* up, double* rp,
                             double* p) {
  if (blockIdx.x || threadIdx.x) return;
  double pi = SUB(d[n - 1], tau);
  p[n - 1] = pi;
  for (int i = n - 2; i >= 0; --i) {
    const double r = ADD(MUL(d[i], MUL(l[i], l[i])), pi);
    rp[i + 1] = r;
    up[i] = DIV(MUL(l[i], d[i]), r);
    pi = SUB(DIV(MUL(pi, d[i]), r), tau);
    p[i] = pi;
  }
  rp[0] = pi;
}

// bbtsvd.cpp:149-164: x <- the Householder vector (x[0] = 1 after the
// scaling), *beta its coefficient; sigma summed in index order.
__global__ void house_kernel(int n, double* x, long inc, double* beta) {
  if (blockIdx.x || threadIdx.x) return;
  double sigma = 0.0;
  for (int i = 1; i < n; ++i) sigma = ADD(sigma, MUL(x[i * inc], x[i * inc]));
  const double x0 = x[0];
  x[0] = 1.0;
  if (sigma == 0.0 && x0 >= 0.0) {
    *beta = 0.0;
  } else if (sigma == 0.0 && x0 < 0.0) {
    *beta = 2.0;
  } else {
    const double mu = sqrt(ADD(MUL(x0, x0), sigma));   // pow(., 0.5): the correctly rounded square root
    const double h = (x0 <= 0.0) ? SUB(x0, mu) : DIV(-sigma, ADD(x0, mu));
    x[0] = h;
    const double h2 = MUL(h, h);
    *beta = DIV(MUL(2.0, h2), ADD(sigma, h2));
    const double r = DIV(1.0, h);   // cblas_dscal(n, 1 / x[0], x, incX)
    for (int i = 0; i < n; ++i) x[i * inc] = MUL(x[i * inc], r);
  }
}

// bbtsvd.cpp:970-978: (x, y) <- (x c + y s, x (-s) + y c), elementwise
__global__ void drot_kernel(size_t n, double* x, size_t incx, double* y, size_t incy, double c, double s) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double xi = x[i * incx], yi = y[i * incy];
    x[i * incx] = ADD(MUL(xi, c), MUL(yi, s));
    y[i * incy] = ADD(MUL(xi, -s), MUL(yi, c));
  }
}

void launched(bbt_ctx* c, const char* what) {
  c->launches++;
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) die(what, bbt::cuda_fail(c, e, "kernel launch"));
}

void sync(bbt_ctx* c, const char* what) {
  const bbt_status s = bbt_synchronize(c);
  if (s != BBT_OK) die(what, s);
}

#undef MUL
#undef DIV
#undef ADD
#undef SUB

}  // namespace

void ldl_decomposition(int n, double* x_diagonal, double* x_upper_diagonal, double* l, double* d) {
  bbt_ctx* c = ctx();
  Dev da(x_diagonal, n), db(x_upper_diagonal, n > 1 ? n - 1 : 0), dl(nullptr, n > 1 ? n - 1 : 0), dd(nullptr, n);
  bbt_status s = bbt::ldl_factor(c, n, da.p, db.p, dl.p, dd.p);
  if (s != BBT_OK) die("ldl_decomposition", s);
  sync(c, "ldl_decomposition");
  dl.back(l, n > 1 ? n - 1 : 0);
  dd.back(d, n);
}

// v (stride ldv) gets the normalised inverse-iteration vector twisted at k;
// the reference normalises with BLAS dnrm2, this library with the scaled sum
// of squares, so the two agree to rounding.
void inverse_iteration(int n, int k, double* l, double* u, double* v, int ldv) {
  bbt_ctx* c = ctx();
  const size_t span = (size_t)(n - 1) * ldv + 1;
  Dev dl(l, n > 1 ? n - 1 : 0), du(u, n > 1 ? n - 1 : 0), dv(v, span);
  bbt_status s = bbt::inverse_iteration_dev(c, n, k, dl.p, du.p, dv.p, ldv);
  if (s != BBT_OK) die("inverse_iteration", s);
  sync(c, "inverse_iteration");
  dv.back(v, span);
}

void dstqds(int n, double* l, double* d, double tau, double* l_plus, double* d_plus, double* s) {
  bbt_ctx* c = ctx();
  Dev dl(l, n > 1 ? n - 1 : 0), dd(d, n), lp(nullptr, n > 1 ? n - 1 : 0), dp(nullptr, n), ds(nullptr, n);
  dstqds_kernel<<<1, 1, 0, c->stream>>>(n, dl.p, dd.p, tau, lp.p, dp.p, ds.p);
  launched(c, "dstqds");
  sync(c, "dstqds");
  lp.back(l_plus, n > 1 ? n - 1 : 0);
  dp.back(d_plus, n);
  ds.back(s, n);
}

void dpqds(int n, double* l, double* d, double tau, double* u_plus, double* r_plus, double* p) {
  bbt_ctx* c = ctx();
  Dev dl(l, n > 1 ? n - 1 : 0), dd(d, n), up(nullptr, n > 1 ? n - 1 : 0), rp(nullptr, n), dp(nullptr, n);
  dpqds_kernel<<<1, 1, 0, c->stream>>>(n, dl.p, dd.p, tau, up.p, rp.p, dp.p);
  launched(c, "dpqds");
  sync(c, "dpqds");
  up.back(u_plus, n > 1 ? n - 1 : 0);
  rp.back(r_plus, n);
  dp.back(p, n);
}

// v (n, contiguous) and u (stride omege_count) of one singular value omega
// from the LDL^T factors l, d of B^T B (bbtsvd.cpp:93-136).
void one_pair_singular_vector_twisted_factorization(int n, int omege_count, double omega, double* l, double* d,
                                                    double* x_diagonal, double* x_upper_diagonal, double* v,
                                                    double* u) {
  bbt_ctx* c = ctx();
  const size_t uspan = (size_t)(n - 1) * omege_count + 1;
  Dev dl(l, n > 1 ? n - 1 : 0), dd(d, n), da(x_diagonal, n), db(x_upper_diagonal, n > 1 ? n - 1 : 0);
  Dev dom(&omega, 1), dv(nullptr, n), du(u, uspan), scr(nullptr, bbt::twisted_pair_scratch_doubles(n));
  bbt_status s = bbt::twisted_pair(c, n, dom.p, dl.p, dd.p, da.p, db.p, dv.p, du.p, omege_count, scr.p);
  if (s != BBT_OK) die("one_pair_singular_vector_twisted_factorization", s);
  sync(c, "one_pair_singular_vector_twisted_factorization");
  dv.back(v, n);
  du.back(u, uspan);
}

void generate_house(int n, double* x, int incX, double* beta) {
  bbt_ctx* c = ctx();
  const size_t span = n > 0 ? (size_t)(n - 1) * incX + 1 : 0;
  Dev dx(x, span), db(nullptr, 1);
  house_kernel<<<1, 1, 0, c->stream>>>(n, dx.p, incX, db.p);
  launched(c, "generate_house");
  sync(c, "generate_house");
  dx.back(x, span);
  db.back(beta, 1);
}

void mmap_drot(size_t n, double* x, size_t incX, double* y, size_t incY, double c_, double s_) {
  if (n == 0) return;
  bbt_ctx* c = ctx();
  const size_t sx = (n - 1) * incX + 1, sy = (n - 1) * incY + 1;
  Dev dx(x, sx), dy(y, sy);
  const unsigned g = (unsigned)std::min<size_t>((n + 255) / 256, 8 * (size_t)c->num_sms);
  drot_kernel<<<g, 256, 0, c->stream>>>(n, dx.p, incX, dy.p, incY, c_, s_);
  launched(c, "mmap_drot");
  sync(c, "mmap_drot");
  dx.back(x, sx);
  dy.back(y, sy);
}


// ---- random orthogonal matrices (bbtsvd.cpp:301-331, 370-395) -------------
// Normal random entries from LAPACK's dlarnv (seeded from rand(), as the
// reference seeds it) and Householder reflectors from dlarfg: the same
// library calls in the same order, so the result is the reference's bit for
// bit when the process links the same LAPACK.  This library bundles no
// LAPACK; the functions are found in the process (the reference links MKL)
// and the call aborts with a message when they are absent.
namespace {
using dlarnv_fn = int (*)(int, int*, int, double*);
using dlarfg_fn = int (*)(int, double*, double*, int, double*);
using dorgqr_fn = int (*)(int, int, int, int, double*, int, const double*);
constexpr int ROW_MAJOR = 101, COL_MAJOR = 102;   // CblasRowMajor / LAPACK_ROW_MAJOR, column-major

void* lapack_symbol(const char* name, const char* fn) {
  void* f = dlsym(RTLD_DEFAULT, name);
  if (!f) f = dlsym(RTLD_DEFAULT, (std::string("scipy_") + name).c_str());   // scipy's prefixed OpenBLAS
  if (!f) {
    fprintf(stderr, "libexcalibur_b200: %s needs %s from the LAPACK the process links; none is loaded\n", fn,
            name);
    abort();
  }
  return f;
}

void random_seed4(int (&iseed)[4]) {
  for (int r = 0; r < 4; ++r) iseed[r] = rand() % 4096;
  if (iseed[3] % 2 == 0) iseed[3] = (iseed[3] + 1) % 4096;   // dlarnv wants an odd last seed
}
}  // namespace

void generate_random_orthogonal_matrix(int matrix_layout, size_t m, double* house, double* tau, unsigned int seed) {
  const auto dlarnv = (dlarnv_fn)lapack_symbol("LAPACKE_dlarnv", "generate_random_orthogonal_matrix");
  const auto dlarfg = (dlarfg_fn)lapack_symbol("LAPACKE_dlarfg", "generate_random_orthogonal_matrix");
  srand(seed);
  int iseed[4];
  std::vector<double> h(m);
  const bool row = matrix_layout == ROW_MAJOR;
  for (size_t i = 0; i < m; ++i) {   // row-major: row i holds i + 1 entries; else column i from its diagonal
    random_seed4(iseed);
    if (row) dlarnv(3, iseed, (int)(i + 1), house + i * m);
    else dlarnv(3, iseed, (int)(m - i), house + i * m + i);
  }
  for (size_t i = 0; i + 1 < m; ++i) {   // reflector i from column i below the diagonal
    const size_t step = row ? m : 1;
    for (size_t j = 0; j < m - i; ++j) h[j] = house[i * m + i + j * step];
    dlarfg((int)(m - i), h.data(), h.data() + 1, 1, tau + i);
    for (size_t j = 0; j < m - i; ++j) house[i * m + i + j * step] = h[j];
  }
  if (m > 0) house[m * m - 1] = 1.0;
}

void generate_random_orthogonal_matrix(size_t m, size_t n, double* x, unsigned int seed) {
  const auto dlarnv = (dlarnv_fn)lapack_symbol("LAPACKE_dlarnv", "generate_random_orthogonal_matrix");
  const auto dlarfg = (dlarfg_fn)lapack_symbol("LAPACKE_dlarfg", "generate_random_orthogonal_matrix");
  const auto dorgqr = (dorgqr_fn)lapack_symbol("LAPACKE_dorgqr", "generate_random_orthogonal_matrix");
  srand(seed);
  int iseed[4];
  std::vector<double> tau(std::min(m, n));
  if (m >= n) {   // m x n row-major with orthonormal columns
    for (size_t i = 0; i < m; ++i) {
      random_seed4(iseed);
      dlarnv(3, iseed, (int)std::min(i + 1, n), x + i * n);
    }
    for (size_t i = 0; i + 1 < n; ++i) dlarfg((int)(m - i), x + i * n + i, x + i * n + i + n, (int)n, tau.data() + i);
    dorgqr(ROW_MAJOR, (int)m, (int)n, (int)n, x, (int)n, tau.data());
  } else {        // orthonormal rows: the transposed problem, column-major
    for (size_t i = 0; i < m; ++i) {
      random_seed4(iseed);
      dlarnv(3, iseed, (int)(n - i), x + i * n + i);
    }
    for (size_t i = 0; i + 1 < m; ++i) dlarfg((int)(n - i), x + i * n + i, x + i * n + i + 1, 1, tau.data() + i);
    dorgqr(COL_MAJOR, (int)n, (int)m, (int)m, x, (int)n, tau.data());
  }
}

// ---- shuffle_matrix (bbtsvd.cpp:398-427) -----------------------------------
// The permutation is drawn on the host with the reference's calls (srand,
// default_random_engine, shuffle, rand), so rand()'s state afterwards is the
// reference's; the swaps of rows (is_left) or columns run on the GPU: the
// pairs are disjoint, and the extra swap of an odd count goes first when
// unshuffling and last otherwise, as in the reference.
namespace {
__global__ void swap_lines_kernel(int npairs, const int2* __restrict__ pr, size_t len, size_t lstride,
                                  size_t estride, double* __restrict__ x) {
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < (long)npairs * (long)len;
       t += (long)gridDim.x * blockDim.x) {
    const int2 q = pr[t / (long)len];
    const size_t e = (size_t)(t % (long)len) * estride;
    double* a = x + (size_t)q.x * lstride + e;
    double* b = x + (size_t)q.y * lstride + e;
    const double ta = *a;
    *a = *b;
    *b = ta;
  }
}
}  // namespace

namespace {
// The swaps of shuffle_matrix on a device copy of x (the draws on the host,
// made even when x is empty, as the reference makes them).
void shuffle_dev(size_t m, size_t n, double* dx, unsigned int seed, bool is_left, bool unshuffle) {
  srand(seed);
  auto dre = std::default_random_engine(seed);
  const size_t k = is_left ? m : n;
  std::vector<int> idx(k);
  for (size_t i = 0; i < k; ++i) idx[i] = (int)i;
  std::shuffle(idx.begin(), idx.end(), dre);
  size_t ri = 0;
  if (k % 2 != 0) ri = k > 1 ? rand() % (k - 1) : 0;   // the reference divides by zero at k = 1
  std::vector<int2> first, pairs, last;
  if (k % 2 != 0 && unshuffle) first.push_back(make_int2((int)(k - 1), (int)ri));
  for (size_t i = 0; i < k / 2; ++i) pairs.push_back(make_int2(idx[2 * i], idx[2 * i + 1]));
  if (k % 2 != 0 && !unshuffle) last.push_back(make_int2((int)(k - 1), (int)ri));
  if (m == 0 || n == 0) return;
  bbt_ctx* c = ctx();
  const size_t len = is_left ? n : m, lstride = is_left ? n : 1, estride = is_left ? 1 : n;
  for (const auto* v : {&first, &pairs, &last}) {
    if (v->empty()) continue;
    int2* dp = nullptr;
    if (cudaMalloc(&dp, v->size() * sizeof(int2)) != cudaSuccess) die("cudaMalloc", BBT_ERR_NOMEM);
    if (cudaMemcpyAsync(dp, v->data(), v->size() * sizeof(int2), cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
      die("cudaMemcpyAsync", BBT_ERR_CUDA);
    const long work = (long)v->size() * (long)len;
    const unsigned g = (unsigned)std::min<long>((work + 255) / 256, 8L * c->num_sms);
    swap_lines_kernel<<<g, 256, 0, c->stream>>>((int)v->size(), dp, len, lstride, estride, dx);
    launched(c, "shuffle_matrix");
    sync(c, "shuffle_matrix");
    cudaFree(dp);
  }
}
}  // namespace

void shuffle_matrix(size_t m, size_t n, double* x, unsigned int seed, bool is_left, bool unshuffle) {
  if (m == 0 || n == 0) {
    shuffle_dev(m, n, nullptr, seed, is_left, unshuffle);   // the draws only
    return;
  }
  ctx();
  Dev dx(x, m * n);
  shuffle_dev(m, n, dx.p, seed, is_left, unshuffle);
  dx.back(x, m * n);
}

// ---- the other masks of bbtsvd.hpp (bbtsvd.cpp:190-299, 429-531, 670-726) ----
// Not on the path DecentralizedClient::run() takes with opt_control 1/3
// (client.cpp calls block_mask for opt_control 0/2; the rest are declared
// only).  Their random tables and reflectors are drawn on the host with the
// reference's own calls in the reference's order, so glibc's rand() state
// afterwards is the reference's; every application to x runs on the GPU.
// The Givens variants rotate with the strip kernel of the mask path, each
// product and sum rounded on its own, as the reference's scalar loops do.
// The Householder variants form the orthogonal factor Q = H_0 ... H_{k-1}
// explicitly on the GPU (the blocked reflector application to an identity)
// and multiply by it (FP64 GEMM), where the reference applies the
// reflectors with LAPACK's dormqr: the same Q to rounding.
namespace {

template <class T>
struct DevArr {   // device copy of a host array of T (freed at scope end)
  T* p = nullptr;
  explicit DevArr(const std::vector<T>& h) {
    if (cudaMalloc(&p, (h.empty() ? 1 : h.size()) * sizeof(T)) != cudaSuccess) die("cudaMalloc", BBT_ERR_NOMEM);
    if (!h.empty() &&
        cudaMemcpyAsync(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, g_ctx->stream) != cudaSuccess)
      die("cudaMemcpyAsync", BBT_ERR_CUDA);
  }
  ~DevArr() { cudaFree(p); }
};

void ensure_ws(bbt_ctx* c, size_t bytes, const char* what) {
  c->ws.reset();
  if (c->ws.cap < bytes && c->ws.reserve(bytes) != cudaSuccess) die(what, BBT_ERR_NOMEM);
}

// Rotations of a Givens mask drawn on the host, applied on the GPU: passes of
// disjoint pairs (one stage each), (c, s) with s already signed.
void rotate_dev(size_t m, size_t n, double* dx, bool is_left, size_t k, size_t passes, size_t ops,
                const std::vector<int2>& pairs, const std::vector<double2>& cs, const char* what) {
  if (k > 10000) {
    fprintf(stderr, "libexcalibur_b200: %s: rotated dimensions above 10,000 are not provided\n", what);
    abort();
  }
  bbt_ctx* c = ctx();
  DevArr<int2> dp(pairs);
  DevArr<double2> dc(cs);
  bbt::GivensDev T{k, passes, ops, 0, (int)ops, dp.p, dc.p};
  bbt_status s = bbt::apply_givens(c, T, m, n, dx, is_left);
  if (s == BBT_OK) s = bbt_synchronize(c);
  if (s != BBT_OK) die(what, s);
}

// (c, s) normalised as the reference does: c / |(c, s)|, s / |(c, s)|.
void normalise_cs(std::vector<double>& c, std::vector<double>& s) {
  for (size_t i = 0; i < c.size(); ++i) {
    const double r = pow(pow(c[i], 2) + pow(s[i], 2), 0.5);
    c[i] /= r;
    s[i] /= r;
  }
}

double random_value_pm1() { return (rand() / (double)RAND_MAX) * 2.0 + -1.0; }   // utils.hpp random_value(-1, 1)

// Q (k x k, column-major, device) = H_0 ... H_{nref-1}: reflector j is column
// j of V from row j down (unit diagonal implied), V(r, c) at V[r*rs + c*cs].
void form_q(bbt_ctx* c, int k, int nref, const double* dV, long rs, long cs, const double* dtau, double* dQ,
            const char* what) {
  bbt_status s = bbt::identity(c, k, dQ, k);
  if (s == BBT_OK && nref > 0) {
    bbt::QrPlan plan;
    ensure_ws(c, bbt::qr_workspace_bytes(k, nref, k, plan) + (1 << 20), what);
    s = bbt::ormqr_left_notrans(c, k, nref, dV, rs, cs, dtau, dQ, k, k, false, plan);
  }
  if (s == BBT_OK) s = bbt_synchronize(c);
  if (s != BBT_OK) die(what, s);
}

// X (r x cc, column-major, ld) <- op(Q) X (left, Q r x r) or X op(Q) (right,
// Q cc x cc), op(Q) = Q^T when trans; dT holds r*cc doubles of scratch.
void apply_q(bbt_ctx* c, bool left, bool trans, int r, int cc, const double* dQ, double* dX, long ld, double* dT,
             const char* what) {
  if (r < 1 || cc < 1) return;
  ensure_ws(c, bbt::dgemm_workspace_bytes(c, r, cc, left ? r : cc) + (1 << 20), what);
  bbt_status s = bbt::copy2d(c, cc, r, dX, ld, dT, r);   // cc columns of r contiguous entries
  if (s == BBT_OK)
    s = left ? bbt::dgemm(c, trans, false, r, cc, r, 1.0, dQ, r, dT, r, 0.0, dX, ld)
             : bbt::dgemm(c, false, trans, r, cc, cc, 1.0, dT, r, dQ, cc, 0.0, dX, ld);
  if (s == BBT_OK) s = bbt_synchronize(c);
  if (s != BBT_OK) die(what, s);
}

// x (m x n row-major, on the device) <- the blocks of the reference's
// block_mask / shuffle_block_mask step: per diagonal block of `bs` rows
// (is_left) or columns, the random orthogonal Q of the block's size from
// generate_random_orthogonal_matrix(row-major, size, seed) (every block
// draws from srand(seed) again), applied as op(Q) x_block (is_left) or
// x_block op(Q), op(Q) = Q for mask and Q^T otherwise.  The last of the
// block's reflectors is the identity: the reference reads its tau one past
// the tau array (a zeroed or negligible value); here it is left out.  With
// dx null only the draws are made (the reference's rand() calls on an empty x).
void block_orthogonal_dev(size_t m, size_t n, size_t bs, double* dx, bool mask, bool is_left, unsigned seed,
                          const char* what) {
  bbt_ctx* c = dx ? ctx() : nullptr;
  const size_t k = is_left ? m : n;
  std::vector<double> house, tau;
  size_t formed = 0;   // block size of the Q in dQ
  double* dQ = nullptr;
  double* dT = nullptr;
  for (size_t i = 0; i < k; i += bs) {
    const size_t rb = std::min(bs, k - i);
    house.assign(rb * rb, 0.0);
    tau.assign(rb > 1 ? rb - 1 : 1, 0.0);
    generate_random_orthogonal_matrix(ROW_MAJOR, rb, house.data(), tau.data(), seed);
    if (!dx) continue;   // an empty x: the draws only
    if (rb != formed) {
      cudaFree(dQ);
      cudaFree(dT);
      dQ = dT = nullptr;
      if (cudaMalloc(&dQ, rb * rb * sizeof(double)) != cudaSuccess ||
          cudaMalloc(&dT, rb * (is_left ? n : m) * sizeof(double)) != cudaSuccess)
        die(what, BBT_ERR_NOMEM);
      DevArr<double> dV(house), dtau(tau);
      form_q(c, (int)rb, (int)rb - 1, dV.p, (long)rb, 1, dtau.p, dQ, what);
      formed = rb;
    }
    // row-major x is the column-major n x m matrix x^T (ld n)
    if (is_left)   // x_block (rb x n) <- op(Q) x_block  <=>  x_block^T <- x_block^T op(Q)^T
      apply_q(c, false, mask, (int)n, (int)rb, dQ, dx + i * n, (long)n, dT, what);
    else           // x_block (m x rb) <- x_block op(Q)  <=>  x_block^T <- op(Q)^T x_block^T
      apply_q(c, true, mask, (int)rb, (int)m, dQ, dx + i, (long)n, dT, what);
  }
  cudaFree(dQ);
  cudaFree(dT);
}

}  // namespace

// bbtsvd.cpp:190-226.  The permutation is shuffled again for every pass
// (each pass starts from the previous one's order); pairs rotate as BLAS drot
// (x, y) <- (c x + s y, c y - s x), s negated when unmasking, which takes
// the passes in reverse order but their (c, s) in the forward order.
void naive_givens_mask_parallel(size_t m, size_t n, size_t mask_size, double* x, bool mask, bool is_left,
                                unsigned int seed) {
  srand(seed);
  auto dre = std::default_random_engine(seed);
  const int k = (int)(is_left ? m : n);
  std::vector<std::vector<int>> pmi;
  std::vector<int> tmp;
  for (int i = 0; i < k; ++i) tmp.push_back(i);
  for (int i = 0; i < (int)mask_size; ++i) {
    std::shuffle(tmp.begin(), tmp.end(), dre);
    pmi.push_back(tmp);
  }
  const int ops = (k - (k % 2)) / 2;
  const size_t cs_size = mask_size * (size_t)ops;
  std::vector<double> cc(cs_size), ss(cs_size);
  for (auto& v : cc) v = random_value_pm1();
  for (auto& v : ss) v = random_value_pm1();
  normalise_cs(cc, ss);
  if (ops == 0 || mask_size == 0 || m == 0 || n == 0) return;
  std::vector<int2> pairs(cs_size);
  std::vector<double2> cs(cs_size);
  const double sg = mask ? 1.0 : -1.0;
  for (size_t i = 0; i < mask_size; ++i) {
    const size_t pi = mask ? i : mask_size - 1 - i;
    for (int j = 0; j < ops; ++j) {
      pairs[i * ops + j] = make_int2(pmi[pi][2 * j], pmi[pi][2 * j + 1]);
      cs[i * ops + j] = make_double2(cc[i * ops + j], sg * ss[i * ops + j]);
    }
  }
  ctx();
  Dev dx(x, m * n);
  rotate_dev(m, n, dx.p, is_left, (size_t)k, mask_size, (size_t)ops, pairs, cs, "naive_givens_mask_parallel");
  dx.back(x, m * n);
}

// bbtsvd.cpp:228-299.  A fresh shuffle per pass; pairs ordered (low, high);
// unmasking reverses the passes and their (c, s) together.
void givens_mask_cache_optimized_parallel(size_t m, size_t n, size_t mask_times, double* x, bool mask,
                                          bool is_left, unsigned int seed) {
  srand(seed);
  auto dre = std::default_random_engine(seed);
  const int k = (int)(is_left ? m : n);
  std::vector<std::vector<int>> pmi;
  for (int i = 0; i < (int)mask_times; ++i) {
    std::vector<int> t;
    for (int j = 0; j < k; ++j) t.push_back(j);
    std::shuffle(t.begin(), t.end(), dre);
    pmi.push_back(t);
  }
  if (!mask) std::reverse(pmi.begin(), pmi.end());
  const int ops = (k - (k % 2)) / 2;
  const size_t cs_size = mask_times * (size_t)ops;
  std::vector<double> cc(cs_size), ss(cs_size);
  for (auto& v : cc) v = random_value_pm1();
  for (auto& v : ss) v = random_value_pm1();
  normalise_cs(cc, ss);
  if (ops == 0 || mask_times == 0 || m == 0 || n == 0) return;
  std::vector<int2> pairs(cs_size);
  std::vector<double2> cs(cs_size);
  const double sg = mask ? 1.0 : -1.0;
  for (size_t i = 0; i < mask_times; ++i) {
    const size_t ci = mask ? i : mask_times - 1 - i;
    for (int j = 0; j < ops; ++j) {
      const int a = pmi[i][2 * j], b = pmi[i][2 * j + 1];
      pairs[i * ops + j] = make_int2(std::min(a, b), std::max(a, b));
      cs[i * ops + j] = make_double2(cc[ci * ops + j], sg * ss[ci * ops + j]);
    }
  }
  ctx();
  Dev dx(x, m * n);
  rotate_dev(m, n, dx.p, is_left, (size_t)k, mask_times, (size_t)ops, pairs, cs,
             "givens_mask_cache_optimized_parallel");
  dx.back(x, m * n);
}

// bbtsvd.cpp:429-487 (blocks below 10,000; the reference's batched branch
// for larger blocks is not provided).
void block_mask(size_t m, size_t n, size_t block_size, double* x, bool mask, bool is_left, unsigned int seed) {
  if ((is_left && m <= 1) || (!is_left && n <= 1)) return;
  if (block_size == 0 || std::min(block_size, is_left ? m : n) >= 10000) {
    fprintf(stderr, "libexcalibur_b200: block_mask: block size %zu is not provided (1 .. 9,999)\n", block_size);
    abort();
  }
  if (m == 0 || n == 0) {
    block_orthogonal_dev(m, n, block_size, nullptr, mask, is_left, seed, "block_mask");
    return;
  }
  ctx();
  Dev dx(x, m * n);
  block_orthogonal_dev(m, n, block_size, dx.p, mask, is_left, seed, "block_mask");
  dx.back(x, m * n);
}

// bbtsvd.cpp:489-531: per round a shuffle (before the blocks when masking,
// after them when unmasking) and the block step with that round's seed.
void shuffle_block_mask(size_t m, size_t n, size_t block_size, int shuffle_times, double* x, bool mask,
                        bool is_left, unsigned int seed) {
  srand(seed);
  std::vector<unsigned int> shuffle_seed, mask_seed;
  for (int st = 0; st < shuffle_times; ++st) {
    shuffle_seed.push_back(rand());
    mask_seed.push_back(rand());
  }
  if (!mask) {
    std::reverse(shuffle_seed.begin(), shuffle_seed.end());
    std::reverse(mask_seed.begin(), mask_seed.end());
  }
  if (shuffle_times > 0 && block_size == 0) {
    fprintf(stderr, "libexcalibur_b200: shuffle_block_mask: block size 0\n");
    abort();
  }
  ctx();
  Dev dx(x, m * n);
  for (int st = 0; st < shuffle_times; ++st) {
    if (mask) shuffle_dev(m, n, m * n ? dx.p : nullptr, shuffle_seed[st], is_left, true);
    srand(mask_seed[st]);
    block_orthogonal_dev(m, n, block_size, m * n ? dx.p : nullptr, mask, is_left, mask_seed[st], "shuffle_block_mask");
    if (!mask) shuffle_dev(m, n, m * n ? dx.p : nullptr, shuffle_seed[st], is_left, false);
  }
  dx.back(x, m * n);
}

// bbtsvd.cpp:670-694: Q from the QR of a normal random mask_size x k matrix
// (column-major k x mask_size), applied to x as a column-major m x n matrix
// (ld m) from the left (Q m x m) or the right (Q n x n); op(Q) = Q when
// is_left equals mask, else Q^T.  The QR runs on the GPU (the library's
// Householder QR, LAPACK's sign convention).
void house_mask(size_t m, size_t n, size_t mask_size, double* x, bool mask, bool is_left, unsigned int seed) {
  const auto dlarnv = (dlarnv_fn)lapack_symbol("LAPACKE_dlarnv", "house_mask");
  srand(seed);
  const size_t k = is_left ? m : n;
  if (mask_size > k) {
    fprintf(stderr, "libexcalibur_b200: house_mask: mask size %zu above the masked dimension %zu\n", mask_size, k);
    abort();
  }
  std::vector<double> house(k * mask_size);
  int iseed[4];
  for (size_t i = 0; i < mask_size; ++i) {   // utils.cpp random_normal_matrix(house, mask_size, k)
    random_seed4(iseed);
    dlarnv(3, iseed, (int)k, house.data() + i * k);
  }
  if (mask_size == 0 || m == 0 || n == 0) return;
  bbt_ctx* c = ctx();
  Dev dx(x, m * n), dQ(nullptr, k * k), dT(nullptr, m * n), dtau(nullptr, mask_size);
  DevArr<double> dA(house);
  bbt::QrPlan plan;
  const size_t tb = (size_t)((mask_size + plan.nb - 1) / plan.nb) * plan.nb * plan.nb;
  Dev dTf(nullptr, tb);
  ensure_ws(c, bbt::qr_workspace_bytes((long)k, (int)mask_size, (int)mask_size, plan) + (1 << 20), "house_mask");
  bbt_status s = bbt::geqrf(c, (long)k, (int)mask_size, dA.p, (long)k, dtau.p, dTf.p, plan);
  if (s == BBT_OK) s = bbt_synchronize(c);
  if (s != BBT_OK) die("house_mask", s);
  form_q(c, (int)k, (int)mask_size, dA.p, 1, (long)k, dtau.p, dQ.p, "house_mask");
  const bool trans = is_left != mask;
  apply_q(c, is_left, trans, (int)m, (int)n, dQ.p, dx.p, (long)m, dT.p, "house_mask");
  dx.back(x, m * n);
}

// bbtsvd.cpp:696-726: mask_size reflectors with uniform random entries below
// a unit head, tau = 2 / ||v||^2 (the process's BLAS dnrm2, as the
// reference); x is column-major m x n when m >= n (Q on the side of is_left)
// and column-major n x m otherwise (Q on the other side).
void householder_reflector_mask(size_t m, size_t n, size_t mask_size, double* x, bool mask, bool is_left,
                                unsigned int seed) {
  using dnrm2_fn = double (*)(int, const double*, int);
  srand(seed);
  const size_t k = is_left ? m : n;
  if (mask_size > k) {
    fprintf(stderr, "libexcalibur_b200: householder_reflector_mask: mask size %zu above the masked dimension %zu\n",
            mask_size, k);
    abort();
  }
  std::vector<double> house(k * mask_size, 0.0), tau(mask_size, 0.0);
  if (mask_size > 0) {
    const auto dnrm2 = (dnrm2_fn)lapack_symbol("cblas_dnrm2", "householder_reflector_mask");
    for (size_t i = 0; i < mask_size; ++i) {
      house[i * k + i] = 1.0;
      for (size_t j = 0; j + i + 1 < k; ++j) house[i * k + i + 1 + j] = random_value_pm1();
      tau[i] = 2 / pow(dnrm2((int)(k - i), house.data() + i * k + i, 1), 2);
    }
  }
  if (mask_size == 0 || m == 0 || n == 0) return;
  bbt_ctx* c = ctx();
  Dev dx(x, m * n), dQ(nullptr, k * k), dT(nullptr, m * n);
  DevArr<double> dV(house), dtau(tau);
  form_q(c, (int)k, (int)mask_size, dV.p, 1, (long)k, dtau.p, dQ.p, "householder_reflector_mask");
  if (m >= n)   // Q on the is_left side of the column-major m x n x
    apply_q(c, is_left, is_left != mask, (int)m, (int)n, dQ.p, dx.p, (long)m, dT.p, "householder_reflector_mask");
  else          // Q on the other side of the column-major n x m x
    apply_q(c, !is_left, is_left == mask, (int)n, (int)m, dQ.p, dx.p, (long)n, dT.p,
            "householder_reflector_mask");
  dx.back(x, m * n);
}
