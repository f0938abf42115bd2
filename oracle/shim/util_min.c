/*
 * The distance helpers of the reference's src/util.c (lines 8-49), restated
 * so that the reference sources build without libhdf5 (the rest of util.c is
 * HDF5 file I/O, which the oracle does not need).  TEST INFRASTRUCTURE ONLY.
 */
#include <math.h>
#include "util.h"

double uniform_distance_real(long n, const double* x, const double* y)
{
	double d = 0;
	for (long i = 0; i < n; i++) d = fmax(d, fabs(x[i] - y[i]));
	return d;
}

double uniform_distance(long n, const numeric* x, const numeric* y)
{
	double d = 0;
	for (long i = 0; i < n; i++) d = fmax(d, _abs(x[i] - y[i]));
	return d;
}

double relative_distance(long n, const numeric* x, const numeric* y, double eps)
{
	double d = 0;
	for (long i = 0; i < n; i++) d = fmax(d, reldist(x[i], y[i], eps));
	return d;
}
