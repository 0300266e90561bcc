// CHECKER — test infrastructure, not product code.
// extern "C" wrappers over the reference's own bbtsvd.hpp functions
// (Excalibur include/bbtsvd.hpp:22-47), compiled together with the
// reference's sources into oracle/_ref/ so that tests/golden/make_golden.py
// can call them through ctypes.  Built only where the reference sources are
// present; nothing here is part of the product.
#include <cstdint>
#include <cstdlib>
#include "bbtsvd.hpp"

extern "C" {
int ref_negative_count(int n, double* a, double* b, double mu) { return negative_count(n, a, b, mu); }
void ref_bisection(int n, double* a, double* b, double lo, double hi, double tol, int top_k,
                   double* sigma, int* count) {
  bisection_singular_values(n, a, b, lo, hi, tol, top_k, sigma, count);
}
void ref_twisted_vectors(int n, int cnt, double* sigma, double* a, double* b, double* u, double* v) {
  two_side_singular_vectors_twisted_factorization(n, cnt, sigma, a, b, u, v);
}
void ref_bidiagonal_svd(int k, double* a, double* b, double* u, double* v, double* s, int top_k) {
  bidiagonal_bisection_twisted_svd(k, a, b, u, v, s, top_k);
}
void ref_givens_mask(size_t m, size_t n, size_t t, double* x, int mask, int is_left, unsigned seed) {
  givens_mask_cache_optimized_parallel_with_simd(m, n, t, x, mask != 0, is_left != 0, seed);
}
void ref_block_shift_mask(size_t m, size_t n, size_t t, double* x, int mask, int is_left, unsigned seed) {
  block_shift_mask(m, n, t, x, mask != 0, is_left != 0, seed);
}
void ref_ldl(int n, double* a, double* b, double* l, double* d) { ldl_decomposition(n, a, b, l, d); }
void ref_inverse_iteration(int n, int k, double* l, double* u, double* v, int ldv) {
  inverse_iteration(n, k, l, u, v, ldv);
}
void ref_dstqds(int n, double* l, double* d, double tau, double* lp, double* dp, double* s) {
  dstqds(n, l, d, tau, lp, dp, s);
}
void ref_dpqds(int n, double* l, double* d, double tau, double* up, double* rp, double* p) {
  dpqds(n, l, d, tau, up, rp, p);
}
void ref_one_pair(int n, int cnt, double omega, double* l, double* d, double* a, double* b, double* v, double* u) {
  one_pair_singular_vector_twisted_factorization(n, cnt, omega, l, d, a, b, v, u);
}
void ref_generate_house(int n, double* x, int inc, double* beta) { generate_house(n, x, inc, beta); }
void ref_mmap_drot(size_t n, double* x, size_t incx, double* y, size_t incy, double c, double s) {
  mmap_drot(n, x, incx, y, incy, c, s);
}
void ref_random_orthogonal_house(int layout, size_t m, double* house, double* tau, unsigned seed) {
  generate_random_orthogonal_matrix(layout, m, house, tau, seed);
}
void ref_random_orthogonal(size_t m, size_t n, double* x, unsigned seed) {
  generate_random_orthogonal_matrix(m, n, x, seed);
}
void ref_shuffle_matrix(size_t m, size_t n, double* x, unsigned seed, int is_left, int unshuffle) {
  shuffle_matrix(m, n, x, seed, is_left != 0, unshuffle != 0);
}
void ref_naive_givens(size_t m, size_t n, size_t t, double* x, int mask, int is_left, unsigned seed) {
  naive_givens_mask_parallel(m, n, t, x, mask != 0, is_left != 0, seed);
}
void ref_givens_cached(size_t m, size_t n, size_t t, double* x, int mask, int is_left, unsigned seed) {
  givens_mask_cache_optimized_parallel(m, n, t, x, mask != 0, is_left != 0, seed);
}
void ref_block_mask(size_t m, size_t n, size_t bs, double* x, int mask, int is_left, unsigned seed) {
  block_mask(m, n, bs, x, mask != 0, is_left != 0, seed);
}
void ref_shuffle_block_mask(size_t m, size_t n, size_t bs, int times, double* x, int mask, int is_left,
                            unsigned seed) {
  shuffle_block_mask(m, n, bs, times, x, mask != 0, is_left != 0, seed);
}
void ref_house_mask(size_t m, size_t n, size_t k, double* x, int mask, int is_left, unsigned seed) {
  house_mask(m, n, k, x, mask != 0, is_left != 0, seed);
}
void ref_householder_reflector_mask(size_t m, size_t n, size_t k, double* x, int mask, int is_left, unsigned seed) {
  householder_reflector_mask(m, n, k, x, mask != 0, is_left != 0, seed);
}
int ref_rand() { return rand(); }
void ref_set_threads(int n) { omp_set_num_threads(n); mkl_set_num_threads(n); }
}
