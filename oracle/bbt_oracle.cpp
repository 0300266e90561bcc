// ORACLE — test infrastructure, not product code.
//
// A CPU restatement of the reference's bidiagonal-SVD and data-mask
// algorithms (Excalibur `src/bbtsvd.cpp`), used only by tests/, by
// __graft_entry__.smoke() and by bench.py's cpu_baseline leg to check the
// CUDA path.  The product never links or calls this library.
//
// Parity is pinned: tests/test_oracle_golden.py checks every function here
// against golden vectors produced by the reference's own sources compiled
// in this repository's checker build (oracle/Makefile, target `ref`).
//
// Arithmetic follows the reference operation by operation and is compiled
// with -ffp-contract=off (no fused multiply-add), matching the reference's
// `-O3 -mavx2` build in which pow(x, 2) is folded to x*x and AVX2 without
// FMA rounds every product and every sum.
#include <dlfcn.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <vector>

namespace {

// The LAPACK / BLAS routines the reference's dense masks call (MKL there),
// resolved in the process at run time: the plain name, else scipy's
// prefixed OpenBLAS.  Null when none is loaded.
void* lapack(const char* name) {
  void* f = dlsym(RTLD_DEFAULT, name);
  if (!f) f = dlsym(RTLD_DEFAULT, (std::string("scipy_") + name).c_str());
  return f;
}
using dlarnv_t = int (*)(int, int*, int, double*);
using dlarfg_t = int (*)(int, double*, double*, int, double*);
using dgeqrf_t = int (*)(int, int, int, double*, int, double*);
using dnrm2_t = double (*)(int, const double*, int);

void seed4(int (&iseed)[4]) {   // the reference's dlarnv seeding (bbtsvd.cpp:305-306)
  for (int r = 0; r < 4; ++r) iseed[r] = rand() % 4096;
  if (iseed[3] % 2 == 0) iseed[3] = (iseed[3] + 1) % 4096;
}

// generate_random_orthogonal_matrix(CblasRowMajor, m, house, tau, seed),
// bbtsvd.cpp:301-331: row i of house gets i + 1 normal entries, then
// reflector i from column i below the diagonal (dlarfg), house[m*m-1] = 1.
bool orthogonal_house(size_t m, double* house, double* tau, unsigned seed) {
  const auto dlarnv = (dlarnv_t)lapack("LAPACKE_dlarnv");
  const auto dlarfg = (dlarfg_t)lapack("LAPACKE_dlarfg");
  if (!dlarnv || !dlarfg) return false;
  srand(seed);
  int iseed[4];
  std::vector<double> h(m);
  for (size_t i = 0; i < m; ++i) {
    seed4(iseed);
    dlarnv(3, iseed, (int)(i + 1), house + i * m);
  }
  for (size_t i = 0; i + 1 < m; ++i) {
    for (size_t j = 0; j < m - i; ++j) h[j] = house[i * m + i + j * m];
    dlarfg((int)(m - i), h.data(), h.data() + 1, 1, tau + i);
    for (size_t j = 0; j < m - i; ++j) house[i * m + i + j * m] = h[j];
  }
  if (m > 0) house[m * m - 1] = 1.0;
  return true;
}

// dormqr's action, by its definition: Q = H_0 ... H_{k-1}, H_j = I - tau_j
// v_j v_j^T, v_j unit at j with A(r, j) below it (A(r, c) = A[r*ars + c*acs]);
// C (rows x cols, C(r, c) = C[r*crs + c*ccs]) <- op(Q) C (left) or C op(Q).
void reflect(bool left, bool trans, size_t rows, size_t cols, size_t k, const double* A, long ars, long acs,
             const double* tau, double* C, long crs, long ccs) {
  const size_t nq = left ? rows : cols;
  std::vector<double> v(nq);
  // left N and right T apply H_{k-1} first; left T and right N apply H_0 first
  const bool backward = left != trans;
  for (size_t s = 0; s < k; ++s) {
    const size_t j = backward ? k - 1 - s : s;
    for (size_t r = 0; r < nq; ++r) v[r] = r < j ? 0.0 : (r == j ? 1.0 : A[r * ars + j * acs]);
    if (left) {
      for (size_t c = 0; c < cols; ++c) {   // C(:, c) -= tau v (v^T C(:, c))
        double w = 0.0;
        for (size_t r = j; r < rows; ++r) w += v[r] * C[r * crs + c * ccs];
        for (size_t r = j; r < rows; ++r) C[r * crs + c * ccs] -= tau[j] * v[r] * w;
      }
    } else {
      for (size_t r = 0; r < rows; ++r) {   // C(r, :) -= tau (C(r, :) v) v^T
        double w = 0.0;
        for (size_t c = j; c < cols; ++c) w += C[r * crs + c * ccs] * v[c];
        for (size_t c = j; c < cols; ++c) C[r * crs + c * ccs] -= tau[j] * w * v[c];
      }
    }
  }
}

// The block step of block_mask / shuffle_block_mask (bbtsvd.cpp:436-442,
// 463-467, 511-523) on a row-major m x n x: each block of bs rows (is_left)
// or columns gets op(Q) from its size and seed, op = Q masking and Q^T
// unmasking.  A full block's last reflector is taken as the identity (the
// reference reads its tau one past the end of the tau array).
bool block_step(size_t m, size_t n, size_t bs, double* x, int mask, int is_left, unsigned seed) {
  const size_t k = is_left ? m : n;
  std::vector<double> house, tau;
  for (size_t i = 0; i < k; i += bs) {
    const size_t rb = std::min(bs, k - i);
    house.assign(rb * rb, 0.0);
    tau.assign(rb, 0.0);
    if (!orthogonal_house(rb, house.data(), tau.data(), seed)) return false;
    tau[rb - 1] = 0.0;
    if (is_left)
      reflect(true, !mask, rb, n, rb, house.data(), (long)rb, 1, tau.data(), x + i * n, (long)n, 1);
    else
      reflect(false, !mask, m, rb, rb, house.data(), (long)rb, 1, tau.data(), x + i, (long)n, 1);
  }
  return true;
}

// shuffle_matrix, bbtsvd.cpp:396-427 (k = 1 left alone: the reference divides by zero).
void shuffle_rows(size_t m, size_t n, double* x, unsigned seed, int is_left, int unshuffle) {
  srand(seed);
  std::default_random_engine dre(seed);
  const size_t k = is_left ? m : n;
  std::vector<int> idx;
  for (size_t i = 0; i < k; ++i) idx.push_back((int)i);
  std::shuffle(idx.begin(), idx.end(), dre);
  size_t ri = 0;
  if (k % 2 != 0) ri = k > 1 ? rand() % (k - 1) : 0;
  auto sw = [&](size_t a, size_t b) {
    if (a == b) return;
    if (is_left) for (size_t e = 0; e < n; ++e) std::swap(x[a * n + e], x[b * n + e]);
    else for (size_t e = 0; e < m; ++e) std::swap(x[e * n + a], x[e * n + b]);
  };
  if (k % 2 != 0 && unshuffle) sw(k - 1, ri);
  for (size_t i = 0; i < k / 2; ++i) sw((size_t)idx[2 * i], (size_t)idx[2 * i + 1]);
  if (k % 2 != 0 && !unshuffle) sw(k - 1, ri);
}

// Stationary-qd Sturm count of B^T B - mu^2 I.  bbtsvd.cpp:7-17.
int sturm_count(int n, const double* a, const double* b, double mu) {
  const double mu2 = mu * mu;
  int neg = 0;
  double piv = 1.0, t = 0.0;
  for (int i = 0; i < n; ++i) {
    if (i == 0) {
      t = -mu2;
    } else {
      const double q = (b[i - 1] * b[i - 1]) / piv;
      t = t * q;
      t = t - mu2;
    }
    piv = a[i] * a[i] + t;
    if (piv < 0.0) ++neg;
  }
  return neg;
}

// Plain 2-norm, stride inc.  Stands in for cblas_dnrm2 (bbtsvd.cpp:69);
// agrees with BLAS to rounding, not bitwise.
double norm2(int n, const double* x, int inc) {
  double scale = 0.0, ssq = 1.0;
  for (int i = 0; i < n; ++i) {
    const double v = std::fabs(x[(size_t)i * inc]);
    if (v != 0.0) {
      if (scale < v) {
        ssq = 1.0 + ssq * (scale / v) * (scale / v);
        scale = v;
      } else {
        ssq += (v / scale) * (v / scale);
      }
    }
  }
  return scale * std::sqrt(ssq);
}

// First index of the smallest |x_i| (cblas_idamin semantics).
int argmin_abs(int n, const double* x) {
  int best = 0;
  double bv = std::fabs(x[0]);
  for (int i = 1; i < n; ++i) {
    const double v = std::fabs(x[i]);
    if (v < bv) { bv = v; best = i; }
  }
  return best;
}

// First index of the largest |x_i| (cblas_idamax semantics).
int argmax_abs(int n, const double* x, int inc) {
  int best = 0;
  double bv = std::fabs(x[0]);
  for (int i = 1; i < n; ++i) {
    const double v = std::fabs(x[(size_t)i * inc]);
    if (v > bv) { bv = v; best = i; }
  }
  return best;
}

// Twisted inverse-iteration solve: x[k] = 1, backward with lower factor,
// forward with upper factor, then normalise.  bbtsvd.cpp:65-71.
void twisted_solve(int n, int k, const double* lo, const double* up, double* x, int inc) {
  x[(size_t)k * inc] = 1.0;
  for (int i = k - 1; i >= 0; --i) x[(size_t)i * inc] = -lo[i] * x[(size_t)(i + 1) * inc];
  for (int i = k + 1; i < n; ++i) x[(size_t)i * inc] = -up[i - 1] * x[(size_t)(i - 1) * inc];
  const double r = 1.0 / norm2(n, x, inc);
  for (int i = 0; i < n; ++i) x[(size_t)i * inc] *= r;
}

// One singular triplet's vectors by twisted factorisations of B^T B - w^2 I
// and the coupled B B^T - w^2 I.  bbtsvd.cpp:73-135.
void one_triplet(int n, int ldu, double w, const double* L, const double* D,
                 const double* a, const double* b, double* v, double* u) {
  const double w2 = w * w;
  std::vector<double> lp(n > 1 ? n - 1 : 1), dp(n), s(n + 1), up(n > 1 ? n - 1 : 1),
      rp(n + 1), p(n + 1), g(n);
  // stationary qd (dstqds), bbtsvd.cpp:73-81
  s[0] = -w2;
  for (int i = 0; i + 1 < n; ++i) {
    dp[i] = D[i] + s[i];
    lp[i] = D[i] * L[i] / dp[i];
    s[i + 1] = lp[i] * L[i] * s[i] - w2;
  }
  dp[n - 1] = D[n - 1] + s[n - 1];
  // progressive qd (dpqds), bbtsvd.cpp:83-91
  p[n - 1] = D[n - 1] - w2;
  for (int i = n - 2; i >= 0; --i) {
    rp[i + 1] = D[i] * (L[i] * L[i]) + p[i + 1];
    up[i] = L[i] * D[i] / rp[i + 1];
    p[i] = p[i + 1] * D[i] / rp[i + 1] - w2;
  }
  rp[0] = p[0];
  for (int i = 0; i < n; ++i) g[i] = s[i] + p[i] + w2;
  int k = argmin_abs(n, g.data());
  twisted_solve(n, k, lp.data(), up.data(), v, 1);
  // coupling to the left factor, bbtsvd.cpp:114-126
  s[n] = -w2; p[n] = 1.0; rp[n] = 1.0;
  for (int i = 0; i < n; ++i) {
    dp[i] = s[i + 1] / s[i] * dp[i];
    g[i] = -w2 * g[i] * rp[i + 1] / (s[i] * p[i + 1]);
  }
  k = argmin_abs(n, g.data());
  for (int i = 0; i < n; ++i) rp[i] = p[i] / p[i + 1] * rp[i + 1];
  for (int i = 0; i + 1 < n; ++i) {
    lp[i] = a[i + 1] / dp[i] * b[i];
    up[i] = a[i + 1] / rp[i + 1] * b[i];
  }
  twisted_solve(n, k, lp.data(), up.data(), u, ldu);
}

}  // namespace

extern "C" {

int orc_negative_count(int n, const double* a, const double* b, double mu) {
  return sturm_count(n, a, b, mu);
}

// Depth-first bisection over [lo, hi], upper half first, until the midpoint
// no longer splits the interval (or the width is <= tol).  One value per
// converged interval, descending, at most top_k.  bbtsvd.cpp:19-52.
void orc_bisection(int n, const double* a, const double* b, double lo, double hi, double tol,
                   int top_k, double* sigma, int* count) {
  struct Node { double lo; int clo; double hi; int chi; };
  const int clo = sturm_count(n, a, b, lo), chi = sturm_count(n, a, b, hi);
  *count = 0;
  if (!(clo <= chi && top_k > 0)) return;
  std::vector<Node> st;
  st.push_back({lo, clo, hi, chi});
  while (!st.empty()) {
    Node nd = st.back();
    st.pop_back();
    const double mid = (nd.lo + nd.hi) / 2;
    if ((nd.hi - nd.lo) <= tol || mid == nd.lo || mid == nd.hi) {
      sigma[(*count)++] = mid;
      if (*count >= top_k) break;
      continue;
    }
    const int cm = sturm_count(n, a, b, mid);
    if (cm > nd.clo) st.push_back({nd.lo, nd.clo, mid, cm});
    if (nd.chi > cm) st.push_back({mid, cm, nd.hi, nd.chi});
  }
}

// LDL^T of B^T B.  bbtsvd.cpp:54-63.
void orc_ldl(int n, const double* a, const double* b, double* L, double* D) {
  D[0] = a[0] * a[0];
  for (int i = 1; i < n; ++i) {
    const double ab = a[i - 1] * b[i - 1];
    L[i - 1] = ab / D[i - 1];
    D[i] = a[i] * a[i] + b[i - 1] * b[i - 1] - (ab * ab) / D[i - 1];
  }
}

// Vectors for `cnt` singular values: v_i in row i of V (cnt x n), u_i in
// column i of U (n x cnt).  bbtsvd.cpp:138-147.
void orc_twisted_vectors(int n, int cnt, const double* sigma, const double* a, const double* b,
                         double* U, double* V) {
  std::vector<double> L(n > 1 ? n - 1 : 1), D(n);
  orc_ldl(n, a, b, L.data(), D.data());
  for (int i = 0; i < cnt; ++i)
    one_triplet(n, cnt, sigma[i], L.data(), D.data(), a, b, V + (size_t)i * n, U + i);
}

// Top-k bisection + twisted vectors + sign fixes.  bbtsvd.cpp:932-968.
// Returns 0, or -1 where the reference asserts (fewer values than top_k).
int orc_bidiagonal_svd(int k, const double* a, const double* b, double* U, double* V,
                       double* sigma, int top_k) {
  const double na = norm2(k, a, 1), nb = (k > 1) ? norm2(k - 1, b, 1) : 0.0;
  const double bound = na * na + nb * nb;
  int cnt = 0;
  orc_bisection(k, a, b, 0.0, bound, 1e-20, top_k, sigma, &cnt);
  if (cnt < top_k) return -1;
  orc_twisted_vectors(k, top_k, sigma, a, b, U, V);
  for (int i = 0; i < top_k; ++i) {
    double* vi = V + (size_t)i * k;
    const int p = argmax_abs(k, vi, 1);
    double sg;
    if (p == 0) sg = U[i] * a[0] / sigma[i];
    else sg = (U[(size_t)(p - 1) * top_k + i] * b[p - 1] + U[(size_t)p * top_k + i] * a[p]) / sigma[i];
    if (sg * vi[p] < 0)
      for (int j = 0; j < k; ++j) vi[j] = -vi[j];
  }
  for (int i = 0; i < top_k; ++i) {
    if (std::fabs(sigma[i] - a[i]) < 1e-15) {
      U[(size_t)i + (size_t)i * top_k] = 1.0;
      for (int j = i + 1; j < top_k; ++j) U[(size_t)i * top_k + j] = 0.0;
      for (int j = i + 1; j < k; ++j) U[(size_t)j * top_k + i] = 0.0;
      for (int j = 0; j < k; ++j) V[(size_t)i * k + j] = (j == i) ? 1.0 : 0.0;
    }
  }
  return 0;
}

// Random Givens tables exactly as the reference draws them
// (bbtsvd.cpp:729-779): per pass a std::shuffle of 0..k-1 with
// std::default_random_engine(seed), an extra rand() partner when k is odd,
// reversal for the inverse, pairs ordered (smaller, larger); then per pass
// c, s = random_value(-1, 1) normalised.  Output per pass: `ops` index pairs
// in application order and their c, s (s already signed for this
// direction: x1' = c x1 + s x2, x2' = -s x1 + c x2).
void orc_givens_tables(size_t k, size_t passes, int mask, unsigned seed, int32_t* pairs,
                       double* c, double* s) {
  srand(seed);
  std::default_random_engine eng(seed);
  const size_t ops = (k + (k & 1)) / 2;
  std::vector<std::vector<size_t>> perm(passes);
  for (size_t t = 0; t < passes; ++t) {
    std::vector<size_t> idx(k);
    for (size_t j = 0; j < k; ++j) idx[j] = j;
    std::shuffle(idx.begin(), idx.end(), eng);
    if (k & 1) {
      idx.push_back(rand() % k);
      while (idx[k] == idx[k - 1]) idx[k] = rand() % k;
    }
    if (!mask) std::reverse(idx.begin(), idx.end());
    for (size_t j = 0; j < 2 * ops; j += 2)
      if (idx[j] > idx[j + 1]) std::swap(idx[j], idx[j + 1]);
    perm[t] = idx;
  }
  if (!mask) std::reverse(perm.begin(), perm.end());
  std::vector<std::vector<double>> cc(passes), ss(passes);
  for (size_t t = 0; t < passes; ++t) {
    cc[t].assign(ops, 0.0);
    ss[t].assign(ops, 0.0);
    for (size_t j = 0; j < ops; ++j) {
      cc[t][j] = (rand() / (double)RAND_MAX) * 2.0 + -1.0;
      ss[t][j] = (rand() / (double)RAND_MAX) * 2.0 + -1.0;
      const double r = pow(cc[t][j] * cc[t][j] + ss[t][j] * ss[t][j], 0.5);
      cc[t][j] /= r;
      ss[t][j] /= r;
    }
    if (!mask) {
      std::reverse(cc[t].begin(), cc[t].end());
      std::reverse(ss[t].begin(), ss[t].end());
    }
  }
  if (!mask) {
    std::reverse(cc.begin(), cc.end());
    std::reverse(ss.begin(), ss.end());
  }
  for (size_t t = 0; t < passes; ++t)
    for (size_t j = 0; j < ops; ++j) {
      pairs[(t * ops + j) * 2] = (int32_t)perm[t][2 * j];
      pairs[(t * ops + j) * 2 + 1] = (int32_t)perm[t][2 * j + 1];
      c[t * ops + j] = cc[t][j];
      s[t * ops + j] = (mask ? 1.0 : -1.0) * ss[t][j];
    }
}

// Direct Givens mask of a row-major m x n matrix: rotates rows (is_left)
// or columns.  bbtsvd.cpp:727-876.
void orc_givens_mask(size_t m, size_t n, size_t passes, double* x, int mask, int is_left,
                     unsigned seed) {
  const size_t k = is_left ? m : n;
  if (k <= 1) return;
  const size_t ops = (k + (k & 1)) / 2;
  std::vector<int32_t> pr(passes * ops * 2);
  std::vector<double> c(passes * ops), s(passes * ops);
  orc_givens_tables(k, passes, mask, seed, pr.data(), c.data(), s.data());
  const size_t other = is_left ? n : m;
  std::vector<double> vec(k);
  for (size_t col = 0; col < other; ++col) {
    for (size_t i = 0; i < k; ++i) vec[i] = is_left ? x[i * n + col] : x[col * n + i];
    for (size_t t = 0; t < passes; ++t)
      for (size_t j = 0; j < ops; ++j) {
        const size_t q = t * ops + j;
        const double x1 = vec[pr[2 * q]], x2 = vec[pr[2 * q + 1]];
        const double cq = c[q], sq = s[q];
        const double n1 = x1 * cq + x2 * sq;
        const double n2 = x1 * (-sq) + x2 * cq;
        vec[pr[2 * q]] = n1;
        vec[pr[2 * q + 1]] = n2;
      }
    for (size_t i = 0; i < k; ++i) {
      if (is_left) x[i * n + col] = vec[i];
      else x[col * n + i] = vec[i];
    }
  }
}

// The two other Givens masks of bbtsvd.hpp (bbtsvd.cpp:190-299), restated:
// floor(k / 2) pairs per pass (an odd k's last index stays put), c and s
// drawn as two runs of random_value(-1, 1) after every shuffle, normalised
// by |(c, s)|.  naive (cached = 0): the permutation is shuffled again for
// every pass, pairs rotate unordered as BLAS drot (x, y) <- (c x + s y,
// c y - s x) with s negated when unmasking, which takes the passes in
// reverse order but their (c, s) forward.  cached (cached = 1): a fresh
// shuffle per pass, pairs ordered (low, high), unmasking reverses the passes
// and their (c, s) together.  Each product and sum rounded on its own.
void orc_givens_variant(size_t m, size_t n, size_t passes, double* x, int mask, int is_left, unsigned seed,
                        int cached) {
  srand(seed);
  std::default_random_engine eng(seed);
  const int k = (int)(is_left ? m : n);
  std::vector<std::vector<int>> perm;
  std::vector<int> run;
  for (int i = 0; i < k; ++i) run.push_back(i);
  for (size_t t = 0; t < passes; ++t) {
    if (cached) {
      std::vector<int> idx;
      for (int i = 0; i < k; ++i) idx.push_back(i);
      std::shuffle(idx.begin(), idx.end(), eng);
      perm.push_back(idx);
    } else {
      std::shuffle(run.begin(), run.end(), eng);
      perm.push_back(run);
    }
  }
  if (cached && !mask) std::reverse(perm.begin(), perm.end());
  const size_t ops = (size_t)((k - (k % 2)) / 2);
  std::vector<double> c(passes * ops), s(passes * ops);
  for (auto& v : c) v = (rand() / (double)RAND_MAX) * 2.0 + -1.0;
  for (auto& v : s) v = (rand() / (double)RAND_MAX) * 2.0 + -1.0;
  for (size_t q = 0; q < c.size(); ++q) {
    const double r = pow(pow(c[q], 2) + pow(s[q], 2), 0.5);
    c[q] /= r;
    s[q] /= r;
  }
  const double sg = mask ? 1.0 : -1.0;
  const size_t other = is_left ? n : m;
  std::vector<double> vec(k);
  for (size_t col = 0; col < other; ++col) {
    for (int i = 0; i < k; ++i) vec[i] = is_left ? x[i * n + col] : x[col * n + i];
    for (size_t t = 0; t < passes; ++t) {
      const std::vector<int>& pr = cached ? perm[t] : perm[mask ? t : passes - 1 - t];
      const size_t cb = (cached && !mask ? passes - 1 - t : t) * ops;
      for (size_t j = 0; j < ops; ++j) {
        int a = pr[2 * j], b = pr[2 * j + 1];
        if (cached && a > b) std::swap(a, b);
        const double cq = c[cb + j], sq = sg * s[cb + j];
        const double x1 = vec[a], x2 = vec[b];
        const double n1 = x1 * cq + x2 * sq;
        const double n2 = x1 * (-sq) + x2 * cq;
        vec[a] = n1;
        vec[b] = n2;
      }
    }
    for (int i = 0; i < k; ++i) {
      if (is_left) x[i * n + col] = vec[i];
      else x[col * n + i] = vec[i];
    }
  }
}

// Near-square factorisation k - remain = rows * cols used by the large-k
// mask path.  bbtsvd.cpp:166-188 (limit 10000, aspect ratio < 2).
void orc_square_convert(size_t k, size_t* rows, size_t* cols, size_t* remain) {
  const size_t lim = 10000;
  size_t rem = 0;
  for (;;) {
    const size_t kk = k - rem;
    size_t bm = kk, bn = 1;
    for (size_t i = lim; i > 1; --i) {
      if (kk % i) continue;
      const size_t q = kk / i;
      if (i > q && q < lim && q > 1 && (i - q) < (bm - bn) && ((double)i / (double)q) < 2) {
        bm = i;
        bn = q;
      }
    }
    if (bm < lim) { *rows = bm; *cols = bn; *remain = rem; return; }
    ++rem;
  }
}

// Block-shift mask: direct Givens mask when the rotated dimension k <= 10000,
// otherwise each vector is folded into a near-square virtual matrix
// (Givens mask on both sides, cyclic row shift, remainder pass).
// bbtsvd.cpp:533-669.
void orc_block_shift_mask(size_t m, size_t n, size_t passes, double* x, int mask, int is_left,
                          unsigned seed) {
  srand(seed);
  const size_t k = is_left ? m : n;
  if (k <= 10000) {
    orc_givens_mask(m, n, passes, x, mask, is_left, seed);
    return;
  }
  size_t vm, vn, rem;
  orc_square_convert(k, &vm, &vn, &rem);
  const size_t body = k - rem;
  const size_t nvec = is_left ? n : m;
  const size_t stride = is_left ? n : 1;  // step between elements of one vector
  std::vector<double> blk(body), sh(body), rb(rem + vm);
  auto at = [&](size_t v, size_t i) -> double& { return x[v * (is_left ? 1 : n) + i * stride]; };
  for (size_t v = 0; v < nvec; ++v) {
    if (mask) {
      for (size_t i = 0; i < body; ++i) blk[i] = at(v, i);
      if (rem) {
        for (size_t r = 0; r < vm; ++r) rb[r] = blk[r * vn];
        for (size_t r = 0; r < rem; ++r) rb[vm + r] = at(v, body + r);
        orc_givens_mask(1, rem + vm, passes, rb.data(), 1, 0, seed + 1000);
        for (size_t r = 0; r < vm; ++r) blk[r * vn] = rb[r];
      }
      orc_givens_mask(vm, vn, passes, blk.data(), 1, 1, seed + 2000);
      for (size_t r = 0; r < vm; ++r)
        for (size_t q = 0; q < vn; ++q) {
          long sft = ((long)q - (long)r) % (long)vn;
          if (sft < 0) sft += (long)vn;
          sh[r * vn + q] = blk[r * vn + (size_t)sft];
        }
      orc_givens_mask(vm, vn, passes, sh.data(), 1, 1, seed + 3000);
      orc_givens_mask(vm, vn, passes, sh.data(), 1, 0, seed + 4000);
      if (rem) {
        for (size_t r = 0; r < vm; ++r) rb[r] = sh[r * vn];
        orc_givens_mask(1, rem + vm, passes, rb.data(), 1, 0, seed + 5000);
        for (size_t r = 0; r < vm; ++r) sh[r * vn] = rb[r];
        for (size_t r = 0; r < rem; ++r) at(v, body + r) = rb[vm + r];
      }
      for (size_t i = 0; i < body; ++i) at(v, i) = sh[i];
    } else {
      for (size_t i = 0; i < body; ++i) sh[i] = at(v, i);
      if (rem) {
        for (size_t r = 0; r < rem; ++r) rb[vm + r] = at(v, body + r);
        for (size_t r = 0; r < vm; ++r) rb[r] = sh[r * vn];
        orc_givens_mask(1, rem + vm, passes, rb.data(), 0, 0, seed + 5000);
        for (size_t r = 0; r < vm; ++r) sh[r * vn] = rb[r];
      }
      orc_givens_mask(vm, vn, passes, sh.data(), 0, 1, seed + 3000);
      orc_givens_mask(vm, vn, passes, sh.data(), 0, 0, seed + 4000);
      for (size_t r = 0; r < vm; ++r)
        for (size_t q = 0; q < vn; ++q) blk[r * vn + q] = sh[r * vn + (q + r) % vn];
      orc_givens_mask(vm, vn, passes, blk.data(), 0, 1, seed + 2000);
      if (rem) {
        for (size_t r = 0; r < vm; ++r) rb[r] = blk[r * vn];
        orc_givens_mask(1, rem + vm, passes, rb.data(), 0, 0, seed + 1000);
        for (size_t r = 0; r < vm; ++r) blk[r * vn] = rb[r];
        for (size_t r = 0; r < rem; ++r) at(v, body + r) = rb[vm + r];
      }
      for (size_t i = 0; i < body; ++i) at(v, i) = blk[i];
    }
  }
}

// The dense masks of bbtsvd.hpp, restated over the process's LAPACK (each
// returns 0, or -1 when no LAPACK is loaded).  block_mask, bbtsvd.cpp:429-487
// (blocks below 10,000): every block draws its Q from srand(seed) again.
int orc_block_mask(size_t m, size_t n, size_t bs, double* x, int mask, int is_left, unsigned seed) {
  if ((is_left && m <= 1) || (!is_left && n <= 1)) return 0;
  return block_step(m, n, bs, x, mask, is_left, seed) ? 0 : -1;
}

// shuffle_block_mask, bbtsvd.cpp:489-531: per round a shuffle (before the
// blocks when masking, after them when unmasking) and the block step.
int orc_shuffle_block_mask(size_t m, size_t n, size_t bs, int rounds, double* x, int mask, int is_left,
                           unsigned seed) {
  srand(seed);
  std::vector<unsigned> ss, ms;
  for (int st = 0; st < rounds; ++st) {
    ss.push_back((unsigned)rand());
    ms.push_back((unsigned)rand());
  }
  if (!mask) {
    std::reverse(ss.begin(), ss.end());
    std::reverse(ms.begin(), ms.end());
  }
  for (int st = 0; st < rounds; ++st) {
    if (mask) shuffle_rows(m, n, x, ss[st], is_left, 1);
    srand(ms[st]);
    if (!block_step(m, n, bs, x, mask, is_left, ms[st])) return -1;
    if (!mask) shuffle_rows(m, n, x, ss[st], is_left, 0);
  }
  return 0;
}

// house_mask, bbtsvd.cpp:670-694: Q from dgeqrf of a normal random
// mask_size x k matrix (column-major k x mask_size), applied to x as a
// column-major m x n matrix; op(Q) = Q when is_left equals mask.
int orc_house_mask(size_t m, size_t n, size_t ms, double* x, int mask, int is_left, unsigned seed) {
  const auto dlarnv = (dlarnv_t)lapack("LAPACKE_dlarnv");
  const auto dgeqrf = (dgeqrf_t)lapack("LAPACKE_dgeqrf");
  if (!dlarnv || !dgeqrf) return -1;
  srand(seed);
  const size_t k = is_left ? m : n;
  std::vector<double> A(k * ms), tau(ms);
  int iseed[4];
  for (size_t i = 0; i < ms; ++i) {   // utils.cpp:214-223 random_normal_matrix
    seed4(iseed);
    dlarnv(3, iseed, (int)k, A.data() + i * k);
  }
  dgeqrf(102, (int)k, (int)ms, A.data(), (int)k, tau.data());
  reflect(is_left, is_left != mask, m, n, ms, A.data(), 1, (long)k, tau.data(), x, 1, (long)m);
  return 0;
}

// householder_reflector_mask, bbtsvd.cpp:696-726: unit-headed reflectors
// with random_value(-1, 1) entries below, tau = 2 / dnrm2(v)^2; x column-major
// m x n when m >= n (Q on the is_left side), else n x m (Q on the other side).
int orc_householder_reflector_mask(size_t m, size_t n, size_t ms, double* x, int mask, int is_left,
                                   unsigned seed) {
  const auto dnrm2 = (dnrm2_t)lapack("cblas_dnrm2");
  if (!dnrm2) return -1;
  srand(seed);
  const size_t k = is_left ? m : n;
  std::vector<double> H(k * ms, 0.0), tau(ms, 0.0);
  for (size_t i = 0; i < ms; ++i) {
    H[i * k + i] = 1.0;
    for (size_t j = 0; j + i + 1 < k; ++j) H[i * k + i + 1 + j] = (rand() / (double)RAND_MAX) * 2.0 + -1.0;
    tau[i] = 2 / pow(dnrm2((int)(k - i), H.data() + i * k + i, 1), 2);
  }
  if (m >= n)
    reflect(is_left, is_left != mask, m, n, ms, H.data(), 1, (long)k, tau.data(), x, 1, (long)m);
  else
    reflect(!is_left, is_left == mask, n, m, ms, H.data(), 1, (long)k, tau.data(), x, 1, (long)n);
  return 0;
}

// glibc srand/rand passthrough so tests can derive seeds the way the
// reference's participants do (client.cpp:196, 498, 531).
void orc_srand(unsigned s) { srand(s); }
int orc_rand(void) { return rand(); }

}  // extern "C"
