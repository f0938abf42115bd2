// FP64 device arithmetic of truncated CG and of the trust-region ratio test
// (src/trust_region.c:14-65, 159-217, 336-352): dot products and axpys with
// explicitly rounded multiplies and adds in index order (no fused multiply-add),
// the arithmetic of a sequential BLAS level-1 loop.  Shared by the single-problem
// optimiser and the batched one.
#pragma once
#include <math.h>

namespace rqc {

enum TcgStatus { TCG_CONTINUE = 0, TCG_BOUNDARY = 1, TCG_CONVERGED = 2 };

struct TcgState
{
	double rsq, stoptol, radius;
	int status;
};

struct RtrState
{
	double radius, rho, fx, fnext, maxradius, rho_trust;
	int accept;
};

__device__ inline double dot_seq(int n, const double* a, const double* b)
{
	double s = 0;
	for (int k = 0; k < n; k++) s = __dadd_rn(s, __dmul_rn(a[k], b[k]));
	return s;
}

// t > 0 with ||z + t d|| = radius (src/trust_region.c:14-65)
__device__ inline double to_boundary(int n, const double* z, const double* d, double radius)
{
	const double dsq = dot_seq(n, d, d);
	if (dsq == 0) return 0;
	const double p = __ddiv_rn(dot_seq(n, z, d), dsq);
	const double q = __ddiv_rn(__dsub_rn(dot_seq(n, z, z), __dmul_rn(radius, radius)), dsq);
	if (p == 0) return sqrt(-q);
	const double a = -__dadd_rn(p, copysign(1.0, p) * sqrt(__dsub_rn(__dmul_rn(p, p), q)));
	const double b = __ddiv_rn(q, a);
	return a <= b ? b : a;
}

// r = grad, rsq, stop tolerance, z = 0, d = -r (src/trust_region.c:161-175)
__device__ inline void tcg_init_dev(int n, const double* grad, double* r, double* d, double* z, TcgState* st,
                                    double radius, double abstol, double reltol)
{
	for (int k = 0; k < n; k++) { r[k] = grad[k]; z[k] = 0; d[k] = -grad[k]; }
	st->rsq = dot_seq(n, r, r);
	st->stoptol = fmax(abstol, reltol * sqrt(st->rsq));
	st->radius = radius;
	st->status = TCG_CONTINUE;
}

// One tCG step after Hd = H d (src/trust_region.c:181-209)
__device__ inline void tcg_step_dev(int n, double* d, const double* hd, double* z, double* r, TcgState* st)
{
	const double dhd = dot_seq(n, d, hd);
	const double t = to_boundary(n, z, d, st->radius);
	const double alpha = __ddiv_rn(st->rsq, dhd);
	if (dhd <= 0 || alpha > t) {
		for (int k = 0; k < n; k++) z[k] = __dadd_rn(z[k], __dmul_rn(t, d[k]));
		st->status = TCG_BOUNDARY;
		return;
	}
	for (int k = 0; k < n; k++) r[k] = __dadd_rn(r[k], __dmul_rn(alpha, hd[k]));
	for (int k = 0; k < n; k++) z[k] = __dadd_rn(z[k], __dmul_rn(alpha, d[k]));
	const double rsq_next = dot_seq(n, r, r);
	if (sqrt(rsq_next) <= st->stoptol) {
		st->status = TCG_CONVERGED;
		return;
	}
	const double beta = __ddiv_rn(rsq_next, st->rsq);
	for (int k = 0; k < n; k++) d[k] = __dadd_rn(__dmul_rn(beta, d[k]), -r[k]);
	st->rsq = rsq_next;
	st->status = TCG_CONTINUE;
}

// Ratio test and radius update (src/trust_region.c:336-352); st->fx, st->fnext set
__device__ inline void rtr_rho_dev(int n, const double* grad, const double* eta, const double* heta, RtrState* st,
                                   int on_boundary)
{
	const double den = __dadd_rn(dot_seq(n, grad, eta), __dmul_rn(0.5, dot_seq(n, eta, heta)));
	const double rho = __ddiv_rn(__dsub_rn(st->fnext, st->fx), den);
	if (rho < 0.25) st->radius = __dmul_rn(st->radius, 0.25);
	else if (rho > 0.75 && on_boundary) st->radius = fmin(2 * st->radius, st->maxradius);
	st->rho = rho;
	st->accept = rho > st->rho_trust;
}

}  // namespace rqc
