// Build shim for compiling the reference's own sources as a CPU checker.
// Test infrastructure only: maps the MKL entry points the reference calls
// (cblas_*, LAPACKE_*, mkl_*) to the OpenBLAS bundled with scipy, which
// exports them under a "scipy_" prefix (LP64).  Nothing in the product
// includes this header.
#pragma once
#include <cstddef>
#include <cstring>
#include <cstdlib>
enum CBLAS_LAYOUT {CblasRowMajor=101, CblasColMajor=102};
enum CBLAS_TRANSPOSE {CblasNoTrans=111, CblasTrans=112};
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
extern "C" {
double scipy_cblas_dnrm2(int,const double*,int);
double scipy_cblas_ddot(int,const double*,int,const double*,int);
void scipy_cblas_daxpy(int,double,const double*,int,double*,int);
void scipy_cblas_dscal(int,double,double*,int);
size_t scipy_cblas_idamin(int,const double*,int);
size_t scipy_cblas_idamax(int,const double*,int);
void scipy_cblas_drot(int,double*,int,double*,int,double,double);
void scipy_cblas_drotg(double*,double*,double*,double*);
void scipy_cblas_dswap(int,double*,int,double*,int);
void scipy_cblas_dcopy(int,const double*,int,double*,int);
void scipy_cblas_dgemv(int,int,int,int,double,const double*,int,const double*,int,double,double*,int);
void scipy_cblas_dger(int,int,int,double,const double*,int,const double*,int,double*,int);
void scipy_cblas_dgemm(int,int,int,int,int,int,double,const double*,int,const double*,int,double,double*,int);
int scipy_LAPACKE_dlarnv(int,int*,int,double*);
int scipy_LAPACKE_dlarfg(int,double*,double*,int,double*);
int scipy_LAPACKE_dgeqrf(int,int,int,double*,int,double*);
int scipy_LAPACKE_dorgqr(int,int,int,int,double*,int,const double*);
int scipy_LAPACKE_dormqr(int,char,char,int,int,int,const double*,int,const double*,double*,int);
int scipy_LAPACKE_dbdsdc(int,char,char,int,double*,double*,double*,int,double*,int,double*,int*);
void scipy_openblas_set_num_threads(int);
}
#define cblas_dnrm2 scipy_cblas_dnrm2
#define cblas_ddot scipy_cblas_ddot
#define cblas_daxpy scipy_cblas_daxpy
#define cblas_dscal scipy_cblas_dscal
#define cblas_idamin (int)scipy_cblas_idamin
#define cblas_idamax (int)scipy_cblas_idamax
#define cblas_drot scipy_cblas_drot
#define cblas_drotg scipy_cblas_drotg
#define cblas_dswap scipy_cblas_dswap
#define cblas_dcopy scipy_cblas_dcopy
#define cblas_dgemv scipy_cblas_dgemv
#define cblas_dger scipy_cblas_dger
#define cblas_dgemm scipy_cblas_dgemm
#define LAPACKE_dlarnv scipy_LAPACKE_dlarnv
#define LAPACKE_dlarfg scipy_LAPACKE_dlarfg
#define LAPACKE_dgeqrf scipy_LAPACKE_dgeqrf
#define LAPACKE_dorgqr scipy_LAPACKE_dorgqr
#define LAPACKE_dormqr scipy_LAPACKE_dormqr
#define LAPACKE_dbdsdc scipy_LAPACKE_dbdsdc
inline void mkl_set_num_threads(int n){ scipy_openblas_set_num_threads(n); }
// Row-major transpose; the reference only calls it as ('R','T', alpha=1).
inline void mkl_dimatcopy(char, char, size_t rows, size_t cols, double, double* a, size_t lda, size_t ldb){
  double* t=(double*)malloc(rows*cols*8);
  for(size_t i=0;i<rows;i++) for(size_t j=0;j<cols;j++) t[j*rows+i]=a[i*lda+j];
  for(size_t j=0;j<cols;j++) memcpy(a+j*ldb, t+j*rows, rows*8);
  free(t);
}
