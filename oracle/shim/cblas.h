/*
 * Minimal CBLAS interface for building the reference C sources in a container
 * without a BLAS installation.  Only the routines the reference calls are
 * declared.  TEST INFRASTRUCTURE ONLY (reference build for the oracle).
 */
#pragma once

enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };

double cblas_ddot(const int n, const double* x, const int incx, const double* y, const int incy);
void   cblas_daxpy(const int n, const double alpha, const double* x, const int incx, double* y, const int incy);
void   cblas_dscal(const int n, const double alpha, double* x, const int incx);
double cblas_dnrm2(const int n, const double* x, const int incx);
double cblas_dznrm2(const int n, const void* x, const int incx);
void   cblas_zdscal(const int n, const double alpha, void* x, const int incx);
void   cblas_dgemv(const enum CBLAS_ORDER order, const enum CBLAS_TRANSPOSE trans, const int m, const int n,
                   const double alpha, const double* a, const int lda, const double* x, const int incx,
                   const double beta, double* y, const int incy);
void   cblas_zgemv(const enum CBLAS_ORDER order, const enum CBLAS_TRANSPOSE trans, const int m, const int n,
                   const void* alpha, const void* a, const int lda, const void* x, const int incx,
                   const void* beta, void* y, const int incy);
