/*
 * Straightforward loop implementations of the CBLAS routines the reference
 * calls (src/trust_region.c, src/statevector.c, test/test_target.c).
 * Summation is sequential, in index order.  TEST INFRASTRUCTURE ONLY.
 */
#include <complex.h>
#include <math.h>
#include "cblas.h"

double cblas_ddot(const int n, const double* x, const int incx, const double* y, const int incy)
{
	double s = 0;
	for (int k = 0; k < n; k++) s += x[k * incx] * y[k * incy];
	return s;
}

void cblas_daxpy(const int n, const double alpha, const double* x, const int incx, double* y, const int incy)
{
	for (int k = 0; k < n; k++) y[k * incy] += alpha * x[k * incx];
}

void cblas_dscal(const int n, const double alpha, double* x, const int incx)
{
	for (int k = 0; k < n; k++) x[k * incx] *= alpha;
}

double cblas_dnrm2(const int n, const double* x, const int incx)
{
	double s = 0;
	for (int k = 0; k < n; k++) s += x[k * incx] * x[k * incx];
	return sqrt(s);
}

double cblas_dznrm2(const int n, const void* xv, const int incx)
{
	const double complex* x = (const double complex*)xv;
	double s = 0;
	for (int k = 0; k < n; k++) { const double complex v = x[k * incx]; s += creal(v) * creal(v) + cimag(v) * cimag(v); }
	return sqrt(s);
}

void cblas_zdscal(const int n, const double alpha, void* xv, const int incx)
{
	double complex* x = (double complex*)xv;
	for (int k = 0; k < n; k++) x[k * incx] *= alpha;
}

void cblas_dgemv(const enum CBLAS_ORDER order, const enum CBLAS_TRANSPOSE trans, const int m, const int n,
                 const double alpha, const double* a, const int lda, const double* x, const int incx,
                 const double beta, double* y, const int incy)
{
	/* row-major, no transpose: the only form the reference uses */
	(void)order; (void)trans;
	for (int r = 0; r < m; r++) {
		double s = 0;
		for (int c = 0; c < n; c++) s += a[r * lda + c] * x[c * incx];
		y[r * incy] = alpha * s + (beta == 0 ? 0 : beta * y[r * incy]);
	}
}

void cblas_zgemv(const enum CBLAS_ORDER order, const enum CBLAS_TRANSPOSE trans, const int m, const int n,
                 const void* alphav, const void* av, const int lda, const void* xv, const int incx,
                 const void* betav, void* yv, const int incy)
{
	(void)order; (void)trans;
	const double complex alpha = *(const double complex*)alphav, beta = *(const double complex*)betav;
	const double complex* a = (const double complex*)av;
	const double complex* x = (const double complex*)xv;
	double complex* y = (double complex*)yv;
	for (int r = 0; r < m; r++) {
		double complex s = 0;
		for (int c = 0; c < n; c++) s += a[r * lda + c] * x[c * incx];
		y[r * incy] = alpha * s + (beta == 0 ? 0 : beta * y[r * incy]);
	}
}
