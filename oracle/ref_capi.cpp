// CHECKER — test infrastructure, not product code.
// extern "C" wrappers over the reference's own bbtsvd.hpp functions
// (Excalibur include/bbtsvd.hpp:22-47), compiled together with the
// reference's sources into oracle/_ref/ so that tests/golden/make_golden.py
// can call them through ctypes.  Built only where the reference sources are
// present; nothing here is part of the product.
#include <cstdint>
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
void ref_set_threads(int n) { omp_set_num_threads(n); mkl_set_num_threads(n); }
}
