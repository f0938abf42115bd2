// Truncated CG, Riemannian trust region and the circuit optimisers
// (src/trust_region.c:14-65, 83-141, 159-217, 230-293, 306-368;
// src/brickwall_opt.c:22-186; src/circuit_opt.c:22-124).
//
// The vector algebra and every scalar decision of tCG and of the ratio test run
// in FP64 on the device, in single-thread kernels whose dot products and axpys
// use explicitly rounded multiplies and adds in index order (no fused
// multiply-add), the arithmetic of a sequential BLAS level-1 loop.  The host
// only reads the resulting status flags to decide whether to launch the next
// Hessian-vector product.  In the optimisers every evaluation (f, gradient,
// HVP), the tangent conversion and the polar retraction run on the device as
// well; the gates cross to the host only as kernel arguments of the passes.
#include <math.h>
#include <stdio.h>
#include <string.h>
#include <vector>

#include "engine.h"
#include "hess.h"
#include "manifold.cuh"
#include "rqc_runtime.h"
#include "rqcopt_gpu.h"
#include "sampling.h"
#include "target_problem.h"
#include "trust_region.cuh"

using namespace rqc;

namespace {

// r = grad, rsq, stop tolerance, z = 0, d = -r
__global__ void k_tcg_init(int n, const double* grad, double* r, double* d, double* z, TcgState* st, double radius,
                           double abstol, double reltol)
{
	if (threadIdx.x | blockIdx.x) return;
	tcg_init_dev(n, grad, r, d, z, st, radius, abstol, reltol);
}

// One tCG step after Hd = H d
__global__ void k_tcg_step(int n, double* d, const double* hd, double* z, double* r, TcgState* st)
{
	if (threadIdx.x | blockIdx.x) return;
	tcg_step_dev(n, d, hd, z, r, st);
}

// Ratio test and radius update; fx / fnext read from the given device doubles unless null.
__global__ void k_rtr_rho(int n, const double* grad, const double* eta, const double* heta, const double* fx_dev,
                          const double* fnext_dev, RtrState* st, int on_boundary)
{
	if (threadIdx.x | blockIdx.x) return;
	if (fx_dev) st->fx = *fx_dev;
	if (fnext_dev) st->fnext = *fnext_dev;
	rtr_rho_dev(n, grad, eta, heta, st, on_boundary);
}

// Z_u = V_u A(vec_u) for every unit (src/matrix.c:309-314)
__global__ void k_real_to_tangent(int nunits, const double* vec, const double2* x, double2* dirs)
{
	const int u = blockIdx.x * blockDim.x + threadIdx.x;
	if (u >= nunits) return;
	M4 v, z;
	for (int e = 0; e < 16; e++) v.a[e] = x[16 * u + e];
	m4_real_to_tangent(vec + 16 * u, v, z);
	for (int e = 0; e < 16; e++) dirs[16 * u + e] = z.a[e];
}

// polar retraction of every unit (src/matrix.c:517-531)
__global__ void k_retract(int nunits, const double2* x, const double* eta, double2* xs)
{
	const int u = blockIdx.x * blockDim.x + threadIdx.x;
	if (u >= nunits) return;
	M4 v, w;
	for (int e = 0; e < 16; e++) v.a[e] = x[16 * u + e];
	m4_retract(v, eta + 16 * u, w);
	for (int e = 0; e < 16; e++) xs[16 * u + e] = w.a[e];
}

int launched(Runtime& rt)
{
	rt.launches++;
	return RQC_CUDA(cudaGetLastError());
}

template <typename S>
int read_state(Runtime& rt, const S* d, S* h)
{
	int ret = RQC_CUDA(cudaMemcpyAsync(h, d, sizeof(S), cudaMemcpyDeviceToHost, rt.stream));
	return ret ? ret : sync(rt);
}

// ----------------------------------------------------------------------------- generic API

struct DevVecs
{
	double *r, *d, *hd, *z, *grad, *eta, *heta;
	TcgState* tcg;
	RtrState* rtr;
};

int alloc_vecs(Runtime& rt, int n, DevVecs& v, Buffer& buf)
{
	const size_t bytes = 7 * (size_t)n * sizeof(double) + 256 + sizeof(TcgState) + sizeof(RtrState);
	int ret = ensure_device(buf, bytes);
	if (ret) return ret;
	double* p = reinterpret_cast<double*>(buf.ptr);
	v.r = p; v.d = p + n; v.hd = p + 2 * n; v.z = p + 3 * n; v.grad = p + 4 * n; v.eta = p + 5 * n; v.heta = p + 6 * n;
	char* s = reinterpret_cast<char*>(p + 7 * n);
	s = reinterpret_cast<char*>(((uintptr_t)s + 127) & ~(uintptr_t)127);
	v.tcg = reinterpret_cast<TcgState*>(s);
	v.rtr = reinterpret_cast<RtrState*>(s + 128);
	return OK;
}

// tCG with a host callback; grad already in v.grad; solution in v.z; returns <0 on error
int tcg_host_callback(Runtime& rt, const double* x, hessian_vector_product_func f_hvp, void* fdata, int n, double radius,
                      const struct truncated_cg_params* params, DevVecs& v, std::vector<double>& hbuf, bool* on_boundary)
{
	k_tcg_init<<<1, 1, 0, rt.stream>>>(n, v.grad, v.r, v.d, v.z, v.tcg, radius, params->abstol, params->reltol);
	int ret = launched(rt);
	*on_boundary = false;
	hbuf.resize(2 * (size_t)n);
	for (int it = 0; it < params->maxiter && !ret; it++) {
		if ((ret = RQC_CUDA(cudaMemcpyAsync(hbuf.data(), v.d, n * sizeof(double), cudaMemcpyDeviceToHost, rt.stream)))) break;
		if ((ret = sync(rt))) break;
		f_hvp(x, fdata, hbuf.data(), hbuf.data() + n);
		if ((ret = RQC_CUDA(cudaMemcpyAsync(v.hd, hbuf.data() + n, n * sizeof(double), cudaMemcpyHostToDevice, rt.stream)))) break;
		k_tcg_step<<<1, 1, 0, rt.stream>>>(n, v.d, v.hd, v.z, v.r, v.tcg);
		if ((ret = launched(rt))) break;
		TcgState st;
		if ((ret = read_state(rt, v.tcg, &st))) break;
		if (st.status == TCG_BOUNDARY) { *on_boundary = true; break; }
		if (st.status == TCG_CONVERGED) break;
	}
	return ret;
}

}  // namespace

extern "C" bool truncated_cg_hvp(const double* x, const double* grad, const hessian_vector_product_func f_hvp, void* fdata,
                                 const int n, const double radius, const struct truncated_cg_params* params, double* z)
{
	Runtime* rt = runtime();
	if (!rt || n < 1) {
		set_last_error(rt ? E_ARG : E_CUDA);
		return false;
	}
	DevVecs v;
	int ret = alloc_vecs(*rt, n, v, rt->opt);
	if (!ret) ret = RQC_CUDA(cudaMemcpyAsync(v.grad, grad, n * sizeof(double), cudaMemcpyHostToDevice, rt->stream));
	std::vector<double> hbuf;
	bool boundary = false;
	if (!ret) ret = tcg_host_callback(*rt, x, f_hvp, fdata, n, radius, params, v, hbuf, &boundary);
	if (!ret) ret = RQC_CUDA(cudaMemcpyAsync(z, v.z, n * sizeof(double), cudaMemcpyDeviceToHost, rt->stream));
	if (!ret) ret = sync(*rt);
	if (ret) set_last_error(ret);
	return boundary;
}

extern "C" void riemannian_trust_region_optimize_hvp(const target_func f, const target_gradient_func f_deriv,
                                                     const hessian_vector_product_func f_hvp, void* fdata,
                                                     retract_func retract_fn, void* rdata, const int n,
                                                     const double* x_init, const int m, const struct rtr_params* params,
                                                     const int niter, double* f_iter, double* x_final)
{
	Runtime* rt = runtime();
	if (!rt || n < 1 || m < 1 || !(params->rho_trust >= 0 && params->rho_trust < 0.25)) {
		fail_arg("riemannian_trust_region_optimize_hvp", "invalid arguments");
		return;
	}
	DevVecs v;
	int ret = alloc_vecs(*rt, n, v, rt->opt);
	std::vector<double> x(x_init, x_init + m), xn(m), hgrad(n), heta(n), hheta(n), hbuf;
	RtrState rs = {};
	rs.radius = params->radius_init;
	rs.maxradius = params->maxradius;
	rs.rho_trust = params->rho_trust;
	if (params->g_func) params->g_iter[0] = params->g_func(x.data(), params->g_data);
	for (int k = 0; k < niter && !ret; k++) {
		const double fx = f_deriv(x.data(), fdata, hgrad.data());
		if ((ret = RQC_CUDA(cudaMemcpyAsync(v.grad, hgrad.data(), n * sizeof(double), cudaMemcpyHostToDevice, rt->stream)))) break;
		bool boundary = false;
		if ((ret = tcg_host_callback(*rt, x.data(), f_hvp, fdata, n, rs.radius, &params->tcg_params, v, hbuf, &boundary))) break;
		if ((ret = RQC_CUDA(cudaMemcpyAsync(heta.data(), v.z, n * sizeof(double), cudaMemcpyDeviceToHost, rt->stream)))) break;
		if ((ret = sync(*rt))) break;
		retract_fn(x.data(), heta.data(), rdata, xn.data());
		f_iter[k] = fx;
		f_hvp(x.data(), fdata, heta.data(), hheta.data());
		rs.fx = fx;
		rs.fnext = f(xn.data(), fdata);
		if ((ret = RQC_CUDA(cudaMemcpyAsync(v.heta, hheta.data(), n * sizeof(double), cudaMemcpyHostToDevice, rt->stream)))) break;
		if ((ret = RQC_CUDA(cudaMemcpyAsync(v.rtr, &rs, sizeof(rs), cudaMemcpyHostToDevice, rt->stream)))) break;
		k_rtr_rho<<<1, 1, 0, rt->stream>>>(n, v.grad, v.z, v.heta, nullptr, nullptr, v.rtr, boundary ? 1 : 0);
		if ((ret = launched(*rt))) break;
		if ((ret = read_state(*rt, v.rtr, &rs))) break;
		if (rs.accept) x.swap(xn);
		if (params->g_func) params->g_iter[k + 1] = params->g_func(x.data(), params->g_data);
	}
	if (ret) {
		set_last_error(ret);
		return;
	}
	memcpy(x_final, x.data(), m * sizeof(double));
	f_iter[niter] = f(x_final, fdata);
}

// ----------------------------------------------------------------------------- dense Hessian

extern "C" bool truncated_cg_hmat(const double* grad, const double* hess, int n, double radius,
                                  const struct truncated_cg_params* params, double* z)
{
	Runtime* rt = runtime();
	if (!rt || n < 1 || !grad || !hess || !params || !z) {
		if (rt) fail_arg("truncated_cg_hmat", "invalid arguments");
		else set_last_error(E_CUDA);
		return false;
	}
	// device: grad n | hess n^2 | work 3n | z n | status
	const size_t nd = (size_t)n * n + 5 * (size_t)n;
	int ret = ensure_device(rt->opt, nd * sizeof(double) + 64);
	double* d_grad = static_cast<double*>(rt->opt.ptr);
	double* d_hess = d_grad + n;
	double* d_work = d_hess + (size_t)n * n;
	double* d_z = d_work + 3 * (size_t)n;
	int* d_status = reinterpret_cast<int*>(d_z + n);
	int status = 0;
	if (!ret) ret = RQC_CUDA(cudaMemcpyAsync(d_grad, grad, n * sizeof(double), cudaMemcpyHostToDevice, rt->stream));
	if (!ret) ret = RQC_CUDA(cudaMemcpyAsync(d_hess, hess, (size_t)n * n * sizeof(double), cudaMemcpyHostToDevice, rt->stream));
	if (!ret) ret = tcg_hmat_device(*rt, n, d_grad, d_hess, radius, params->maxiter, params->abstol, params->reltol, d_work,
	                                d_z, d_status);
	if (!ret) ret = RQC_CUDA(cudaMemcpyAsync(z, d_z, n * sizeof(double), cudaMemcpyDeviceToHost, rt->stream));
	if (!ret) ret = RQC_CUDA(cudaMemcpyAsync(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost, rt->stream));
	if (!ret) ret = sync(*rt);
	if (ret) set_last_error(ret);
	return status != 0;
}

extern "C" void riemannian_trust_region_optimize_hmat(target_func f, target_gradient_hessian_func f_deriv_hess, void* fdata,
                                                      retract_func retract_fn, void* rdata, const int n,
                                                      const double* x_init, const int m, const struct rtr_params* params,
                                                      const int niter, double* f_iter, double* x_final)
{
	Runtime* rt = runtime();
	if (!rt || n < 1 || m < 1 || !f || !f_deriv_hess || !retract_fn || !params ||
	    !(params->rho_trust >= 0 && params->rho_trust < 0.25)) {
		if (rt) fail_arg("riemannian_trust_region_optimize_hmat", "invalid arguments");
		else set_last_error(E_CUDA);
		return;
	}
	DevVecs v;
	int ret = alloc_vecs(*rt, n, v, rt->opt);
	// dense Hessian, tCG work and status
	if (!ret) ret = ensure_device(rt->arrays, ((size_t)n * n + 3 * (size_t)n) * sizeof(double) + 64);
	double* d_hess = static_cast<double*>(rt->arrays.ptr);
	double* d_work = d_hess + (size_t)n * n;
	int* d_status = reinterpret_cast<int*>(d_work + 3 * (size_t)n);
	std::vector<double> x(x_init, x_init + m), xn(m), hgrad(n), hhess((size_t)n * n), heta(n);
	RtrState rs = {};
	rs.radius = params->radius_init;
	rs.maxradius = params->maxradius;
	rs.rho_trust = params->rho_trust;
	if (params->g_func) params->g_iter[0] = params->g_func(x.data(), params->g_data);
	for (int k = 0; k < niter && !ret; k++) {
		const double fx = f_deriv_hess(x.data(), fdata, hgrad.data(), hhess.data());
		if ((ret = RQC_CUDA(cudaMemcpyAsync(v.grad, hgrad.data(), n * sizeof(double), cudaMemcpyHostToDevice, rt->stream)))) break;
		if ((ret = RQC_CUDA(cudaMemcpyAsync(d_hess, hhess.data(), (size_t)n * n * sizeof(double), cudaMemcpyHostToDevice,
		                                    rt->stream))))
			break;
		if ((ret = tcg_hmat_device(*rt, n, v.grad, d_hess, rs.radius, params->tcg_params.maxiter, params->tcg_params.abstol,
		                           params->tcg_params.reltol, d_work, v.z, d_status)))
			break;
		int boundary = 0;
		if ((ret = RQC_CUDA(cudaMemcpyAsync(heta.data(), v.z, n * sizeof(double), cudaMemcpyDeviceToHost, rt->stream)))) break;
		if ((ret = RQC_CUDA(cudaMemcpyAsync(&boundary, d_status, sizeof(int), cudaMemcpyDeviceToHost, rt->stream)))) break;
		if ((ret = gemv_device(*rt, n, d_hess, v.z, v.heta))) break;
		if ((ret = sync(*rt))) break;
		retract_fn(x.data(), heta.data(), rdata, xn.data());
		f_iter[k] = fx;
		rs.fx = fx;
		rs.fnext = f(xn.data(), fdata);
		if ((ret = RQC_CUDA(cudaMemcpyAsync(v.rtr, &rs, sizeof(rs), cudaMemcpyHostToDevice, rt->stream)))) break;
		k_rtr_rho<<<1, 1, 0, rt->stream>>>(n, v.grad, v.z, v.heta, nullptr, nullptr, v.rtr, boundary);
		if ((ret = launched(*rt))) break;
		if ((ret = read_state(*rt, v.rtr, &rs))) break;
		if (rs.accept) x.swap(xn);
		if (params->g_func) params->g_iter[k + 1] = params->g_func(x.data(), params->g_data);
	}
	if (ret) {
		set_last_error(ret);
		return;
	}
	memcpy(x_final, x.data(), m * sizeof(double));
	f_iter[niter] = f(x_final, fdata);
}

// ----------------------------------------------------------------------------- device-resident optimiser

namespace rqc {

// Optimisation of a brickwall or general circuit with all vectors on the device.
struct DeviceOptimizer
{
	Runtime& rt;
	Problem& pb;
	const TargetHolder& th;
	int n;
	DevVecs v;
	double2 *x, *xn, *dirs, *res, *ug;
	double* scratch;   // projected-gradient output of HVP evaluations
	std::vector<double2> hx;
	int hvp_prec;
	long evals_hvp = 0, evals_grad = 0, evals_f = 0;

	DeviceOptimizer(Runtime& r, Problem& p, const TargetHolder& t) : rt(r), pb(p), th(t), n(16 * p.nunits) {}

	int init(const double2* x0)
	{
		const size_t nu = pb.nunits;
		const size_t nres = result_count(pb.G);
		const size_t bytes = 7 * (size_t)n * sizeof(double) + 512 + (4 * 16 * nu + nres) * sizeof(double2) + (n + 8) * sizeof(double);
		int ret = ensure_device(rt.opt, bytes);
		if (ret) return ret;
		if ((ret = alloc_vecs(rt, n, v, rt.opt))) return ret;
		char* base = reinterpret_cast<char*>(rt.opt.ptr) + 7 * (size_t)n * sizeof(double) + 512;
		x = reinterpret_cast<double2*>(base);
		xn = x + 16 * nu;
		dirs = xn + 16 * nu;
		ug = dirs + 16 * nu;
		res = ug + 16 * nu;
		scratch = reinterpret_cast<double*>(res + nres);
		hx.assign(x0, x0 + 16 * nu);
		return RQC_CUDA(cudaMemcpyAsync(x, x0, 16 * nu * sizeof(double2), cudaMemcpyHostToDevice, rt.stream));
	}

	// gates of the device array `src` become the kernel arguments of the next passes
	int load_gates(const double2* src)
	{
		int ret = RQC_CUDA(cudaMemcpyAsync(hx.data(), src, hx.size() * sizeof(double2), cudaMemcpyDeviceToHost, rt.stream));
		if (!ret) ret = sync(rt);
		if (!ret) pb.set_gates_from_units(hx.data());
		if (!ret) ret = RQC_CUDA(cudaMemcpyAsync(ug, src, hx.size() * sizeof(double2), cudaMemcpyDeviceToDevice, rt.stream));
		return ret;
	}

	CircuitSpec spec(bool with_dirs) const
	{
		CircuitSpec cs;
		cs.L = pb.L;
		cs.ngates = pb.G;
		cs.gates = pb.gates.data();
		cs.dirs = with_dirs ? pb.dirs.data() : nullptr;
		cs.wires = pb.wires.data();
		return cs;
	}

	// f at the loaded gates -> res[0]
	int eval_f(int prec)
	{
		evals_f++;
		return evaluate(rt, spec(false), th.spec, EVAL_F, prec, res);
	}

	// f and projected gradient at the loaded gates -> res[0], v.grad
	int eval_grad(int prec)
	{
		evals_grad++;
		int ret = evaluate(rt, spec(false), th.spec, EVAL_GRAD, prec, res);
		if (!ret) ret = post_launch(rt, res, pb, ug, nullptr, 0, nullptr, nullptr, v.grad, nullptr);
		return ret;
	}

	// projected HVP at the loaded gates in direction vec (device, 16 per unit) -> out
	int eval_hvp(const double* vec, double* out, int prec)
	{
		evals_hvp++;
		const int threads = 64, blocks = (pb.nunits + threads - 1) / threads;
		k_real_to_tangent<<<blocks, threads, 0, rt.stream>>>(pb.nunits, vec, ug, dirs);
		int ret = launched(rt);
		std::vector<double2> hd(16 * (size_t)pb.nunits);
		if (!ret) ret = RQC_CUDA(cudaMemcpyAsync(hd.data(), dirs, hd.size() * sizeof(double2), cudaMemcpyDeviceToHost, rt.stream));
		if (!ret) ret = sync(rt);
		if (ret) return ret;
		pb.set_dirs_from_units(hd.data());
		if ((ret = evaluate(rt, spec(true), th.spec, EVAL_HVP, prec, res))) return ret;
		return post_launch(rt, res, pb, ug, dirs, 1, nullptr, nullptr, scratch, out);
	}

	int run(const struct rtr_params* params, int niter, double* f_iter, double2* x_final, int precision)
	{
		RtrState rs = {};
		rs.radius = params->radius_init;
		rs.maxradius = params->maxradius;
		rs.rho_trust = params->rho_trust;
		int ret = RQC_CUDA(cudaMemcpyAsync(v.rtr, &rs, sizeof(rs), cudaMemcpyHostToDevice, rt.stream));
		// precision policy: f and gradient (the ratio test) in complex128 unless plain
		// complex64 was asked for; HVPs in complex64 until the gradient norm falls
		// below the refinement threshold (mixed mode)
		const int fprec = precision == PREC_C64 ? PREC_C64 : PREC_C128;
		hvp_prec = precision == PREC_C128 ? PREC_C128 : PREC_C64;
		double* fx_slot = scratch + n;
		const int threads = 64, blocks = (pb.nunits + threads - 1) / threads;
		rt.opt_trace.clear();
		for (int k = 0; k < niter && !ret; k++) {
			// f and gradient at x (src/trust_region.c:328)
			if ((ret = load_gates(x))) break;
			if ((ret = eval_grad(fprec))) break;
			if ((ret = RQC_CUDA(cudaMemcpyAsync(fx_slot, res, sizeof(double), cudaMemcpyDeviceToDevice, rt.stream)))) break;
			if ((ret = RQC_CUDA(cudaMemcpyAsync(&rs, v.rtr, sizeof(rs), cudaMemcpyDeviceToHost, rt.stream)))) break;
			if ((ret = sync(rt))) break;
			// tCG (src/trust_region.c:159-217)
			k_tcg_init<<<1, 1, 0, rt.stream>>>(n, v.grad, v.r, v.d, v.z, v.tcg, rs.radius, params->tcg_params.abstol,
			                                   params->tcg_params.reltol);
			if ((ret = launched(rt))) break;
			TcgState st;
			if ((ret = read_state(rt, v.tcg, &st))) break;
			if (precision == PREC_MIXED && hvp_prec != PREC_C128 && sqrt(st.rsq) < rt.refine_threshold) hvp_prec = PREC_C128;
			bool boundary = false;
			int inner = 0;
			for (int it = 0; it < params->tcg_params.maxiter; it++) {
				if ((ret = eval_hvp(v.d, v.hd, hvp_prec))) break;
				k_tcg_step<<<1, 1, 0, rt.stream>>>(n, v.d, v.hd, v.z, v.r, v.tcg);
				if ((ret = launched(rt))) break;
				if ((ret = read_state(rt, v.tcg, &st))) break;
				inner = it + 1;
				if (st.status == TCG_BOUNDARY) { boundary = true; break; }
				if (st.status == TCG_CONVERGED) break;
			}
			if (ret) break;
			// candidate point, model decrease and ratio test (src/trust_region.c:330-352)
			k_retract<<<blocks, threads, 0, rt.stream>>>(pb.nunits, x, v.z, xn);
			if ((ret = launched(rt))) break;
			if ((ret = eval_hvp(v.z, v.heta, hvp_prec))) break;
			if ((ret = load_gates(xn))) break;
			if ((ret = eval_f(fprec))) break;
			k_rtr_rho<<<1, 1, 0, rt.stream>>>(n, v.grad, v.z, v.heta, fx_slot, reinterpret_cast<const double*>(res), v.rtr,
			                                   boundary ? 1 : 0);
			if ((ret = launched(rt))) break;
			if ((ret = read_state(rt, v.rtr, &rs))) break;
			f_iter[k] = rs.fx;
			rt.opt_trace.push_back({rs.accept, boundary ? 1 : 0, inner, hvp_prec == PREC_C128 ? 1 : 0});
			if (rs.accept) std::swap(x, xn);
		}
		if (ret) return ret;
		if ((ret = RQC_CUDA(cudaMemcpyAsync(x_final, x, hx.size() * sizeof(double2), cudaMemcpyDeviceToHost, rt.stream)))) return ret;
		if ((ret = load_gates(x))) return ret;
		if ((ret = eval_f(fprec))) return ret;
		double2 ff;
		if ((ret = RQC_CUDA(cudaMemcpyAsync(&ff, res, sizeof(double2), cudaMemcpyDeviceToHost, rt.stream)))) return ret;
		if ((ret = sync(rt))) return ret;
		f_iter[niter] = ff.x;
		return OK;
	}

	// f at the loaded gates from nsamples Haar-random states of rng's stream -> res[0]
	int eval_f_sampled(struct rng_state* rng, long nsamples)
	{
		evals_f++;
		int ret = sampled_f_device(rt, pb.L, pb.G, pb.gates.data(), pb.wires.data(), th.spec, sample_spec(rng, nsamples), res);
		if (!ret) advance_rng(rng, nsamples, pb.L);
		return ret;
	}

	// Trust region with the dense Riemannian Hessian of a brickwall (src/trust_region.c:230-293,
	// src/brickwall_opt.c:85-100, 159-186): every evaluation in complex128.  With rng, f and
	// the Hessian are the sampling estimates of src/brickwall_opt.c:189-265, drawing from
	// rng's stream in the reference's order (f_deriv_hess at x, f at the candidate, ...,
	// f at the result).
	int run_hmat(const struct rtr_params* params, int niter, double* f_iter, double2* x_final,
	             struct rng_state* rng = nullptr, long nsamples = 0)
	{
		const int nl = pb.nunits;
		const size_t nrec = hess_record_count(nl);
		// record | dense Hessian | tCG work | fx | status
		int ret = ensure_device(rt.arrays, nrec * sizeof(double2) + ((size_t)n * n + 3 * (size_t)n + 2) * sizeof(double) + 64);
		if (ret) return ret;
		double2* rec = static_cast<double2*>(rt.arrays.ptr);
		double* d_hess = reinterpret_cast<double*>(rec + nrec);
		double* d_work = d_hess + (size_t)n * n;
		double* fx_slot = d_work + 3 * (size_t)n;
		int* d_status = reinterpret_cast<int*>(fx_slot + 2);
		RtrState rs = {};
		rs.radius = params->radius_init;
		rs.maxradius = params->maxradius;
		rs.rho_trust = params->rho_trust;
		if ((ret = RQC_CUDA(cudaMemcpyAsync(v.rtr, &rs, sizeof(rs), cudaMemcpyHostToDevice, rt.stream)))) return ret;
		HessCircuit c;
		c.L = pb.L;
		c.nlayers = nl;
		c.wires = pb.wires.data();
		const int threads = 64, blocks = (nl + threads - 1) / threads;
		for (int k = 0; k < niter && !ret; k++) {
			// f, gradient vector and Hessian matrix at x (src/trust_region.c:263)
			if ((ret = load_gates(x))) break;
			c.ugates = hx.data();
			if (rng) {
				const SampleSpec sp = sample_spec(rng, nsamples);
				if ((ret = hessian_target_device(rt, c, th.spec, rec, &sp))) break;
				advance_rng(rng, nsamples, pb.L);
			} else if ((ret = hessian_target_device(rt, c, th.spec, rec))) {
				break;
			}
			if ((ret = project_hessian_device(rt, nl, ug, rec, v.grad, d_hess))) break;
			if ((ret = RQC_CUDA(cudaMemcpyAsync(fx_slot, rec, sizeof(double), cudaMemcpyDeviceToDevice, rt.stream)))) break;
			// tCG on the dense Hessian (src/trust_region.c:264)
			if ((ret = tcg_hmat_device(rt, n, v.grad, d_hess, rs.radius, params->tcg_params.maxiter,
			                           params->tcg_params.abstol, params->tcg_params.reltol, d_work, v.z, d_status)))
				break;
			int boundary = 0;
			if ((ret = RQC_CUDA(cudaMemcpyAsync(&boundary, d_status, sizeof(int), cudaMemcpyDeviceToHost, rt.stream)))) break;
			// candidate, model decrease and ratio test (src/trust_region.c:265-281)
			k_retract<<<blocks, threads, 0, rt.stream>>>(nl, x, v.z, xn);
			if ((ret = launched(rt))) break;
			if ((ret = gemv_device(rt, n, d_hess, v.z, v.heta))) break;
			if ((ret = load_gates(xn))) break;   // synchronises: boundary is valid after this
			if ((ret = rng ? eval_f_sampled(rng, nsamples) : eval_f(PREC_C128))) break;
			k_rtr_rho<<<1, 1, 0, rt.stream>>>(n, v.grad, v.z, v.heta, fx_slot, reinterpret_cast<const double*>(res), v.rtr,
			                                   boundary);
			if ((ret = launched(rt))) break;
			if ((ret = read_state(rt, v.rtr, &rs))) break;
			f_iter[k] = rs.fx;
			if (rs.accept) std::swap(x, xn);
		}
		if (ret) return ret;
		if ((ret = RQC_CUDA(cudaMemcpyAsync(x_final, x, hx.size() * sizeof(double2), cudaMemcpyDeviceToHost, rt.stream)))) return ret;
		if ((ret = load_gates(x))) return ret;
		if ((ret = rng ? eval_f_sampled(rng, nsamples) : eval_f(PREC_C128))) return ret;
		double2 ff;
		if ((ret = RQC_CUDA(cudaMemcpyAsync(&ff, res, sizeof(double2), cudaMemcpyDeviceToHost, rt.stream)))) return ret;
		if ((ret = sync(rt))) return ret;
		f_iter[niter] = ff.x;
		return OK;
	}
};

}  // namespace rqc

namespace {

void run_optimizer(const char* fn, Problem& pb, linear_func ufunc, void* udata, struct rtr_params* params, int niter,
                   double* f_iter, const struct mat4x4* start, struct mat4x4* out, bool hmat = false,
                   struct rng_state* rng = nullptr, long nsamples = 0)
{
	TargetHolder th;
	if (!th.set(ufunc, udata, pb.L)) {
		fail_arg(fn, "invalid target");
		return;
	}
	Runtime* rt = runtime();
	if (!rt) { set_last_error(E_CUDA); return; }
	// the drivers disable the per-iteration callback (src/brickwall_opt.c:141-143)
	params->g_func = NULL;
	params->g_data = NULL;
	params->g_iter = NULL;
	DeviceOptimizer opt(*rt, pb, th);
	int ret = opt.init(reinterpret_cast<const double2*>(start));
	if (!ret)
		ret = hmat ? opt.run_hmat(params, niter, f_iter, reinterpret_cast<double2*>(out), rng, nsamples)
		           : opt.run(params, niter, f_iter, reinterpret_cast<double2*>(out), rt->precision);
	if (ret) set_last_error(ret);
}

}  // namespace

extern "C" void optimize_brickwall_circuit_hvp(linear_func ufunc, void* udata, const struct mat4x4 vlist_start[],
                                               const int nlayers, const int nqubits, const int* perms[],
                                               struct rtr_params* params, const int niter, double* f_iter,
                                               struct mat4x4 vlist_opt[])
{
	Problem pb;
	if (!pb.set_brickwall(nqubits, nlayers, vlist_start, nullptr, perms)) {
		fail_arg("optimize_brickwall_circuit_hvp", "invalid arguments");
		return;
	}
	run_optimizer("optimize_brickwall_circuit_hvp", pb, ufunc, udata, params, niter, f_iter, vlist_start, vlist_opt);
}

extern "C" void optimize_quantum_circuit(linear_func ufunc, void* udata, const struct mat4x4 gates_start[],
                                         const int ngates, const int nqubits, const int wires[], struct rtr_params* params,
                                         const int niter, double* f_iter, struct mat4x4 gates_opt[])
{
	Problem pb;
	if (!pb.set_circuit(nqubits, ngates, gates_start, nullptr, wires)) {
		fail_arg("optimize_quantum_circuit", "invalid arguments");
		return;
	}
	run_optimizer("optimize_quantum_circuit", pb, ufunc, udata, params, niter, f_iter, gates_start, gates_opt);
}

extern "C" void optimize_brickwall_circuit_hmat(linear_func ufunc, void* udata, const struct mat4x4 vlist_start[],
                                                const int nlayers, const int nqubits, const int* perms[],
                                                struct rtr_params* params, const int niter, double* f_iter,
                                                struct mat4x4 vlist_opt[])
{
	Problem pb;
	if (!params || !f_iter || !vlist_opt || !pb.set_brickwall(nqubits, nlayers, vlist_start, nullptr, perms)) {
		fail_arg("optimize_brickwall_circuit_hmat", "invalid arguments");
		return;
	}
	run_optimizer("optimize_brickwall_circuit_hmat", pb, ufunc, udata, params, niter, f_iter, vlist_start, vlist_opt, true);
}

extern "C" void optimize_brickwall_circuit_hmat_sampling(linear_func ufunc, void* udata, const struct mat4x4 vlist_start[],
                                                         const int nlayers, const int nqubits, const int* perms[],
                                                         const long nsamples, struct rng_state* rng,
                                                         struct rtr_params* params, const int niter, double* f_iter,
                                                         struct mat4x4 vlist_opt[])
{
	Problem pb;
	if (!params || !f_iter || !vlist_opt || !rng || nsamples < 1 ||
	    !pb.set_brickwall(nqubits, nlayers, vlist_start, nullptr, perms)) {
		fail_arg("optimize_brickwall_circuit_hmat_sampling", "invalid arguments");
		return;
	}
	run_optimizer("optimize_brickwall_circuit_hmat_sampling", pb, ufunc, udata, params, niter, f_iter, vlist_start,
	              vlist_opt, true, rng, nsamples);
}
