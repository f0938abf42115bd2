// Exported target functions (src/target.h:10-67): f = -tr(U^H C), gradients and
// Hessian-vector products summed over all basis columns on the GPU, plus the
// device-native target callbacks.  Per-layer folding (brickwall) and the
// Riemannian projections run in FP64 on the device (k_post).
#include <stdio.h>
#include <string.h>
#include <vector>

#include "engine.h"
#include "manifold.cuh"
#include "rqc_runtime.h"
#include "rqcopt_gpu.h"
#include "target_problem.h"

using namespace rqc;

// ------------------------------------------------------------------ device-native targets

extern "C" int rqcopt_brickwall_ufunc(const struct statevector* psi, void* udata, struct statevector* psi_out)
{
	const struct rqcopt_brickwall_target* t = static_cast<const struct rqcopt_brickwall_target*>(udata);
	return apply_brickwall_unitary(t->vlist, t->nlayers, const_cast<const int**>(t->perms), psi, psi_out);
}

extern "C" int rqcopt_circuit_ufunc(const struct statevector* psi, void* udata, struct statevector* psi_out)
{
	const struct rqcopt_circuit_target* t = static_cast<const struct rqcopt_circuit_target*>(udata);
	return apply_quantum_circuit(t->gates, t->ngates, t->wires, psi, psi_out);
}

extern "C" int rqcopt_dense_ufunc(const struct statevector* psi, void* udata, struct statevector* psi_out)
{
	const struct rqcopt_dense_target* t = static_cast<const struct rqcopt_dense_target*>(udata);
	if (!t || !t->u || !psi || !psi_out || psi->nqubits != t->nqubits || psi_out->nqubits != t->nqubits) return -1;
	const int64_t n = (int64_t)1 << t->nqubits;
	const double2* u = reinterpret_cast<const double2*>(t->u);
	const double2* x = reinterpret_cast<const double2*>(psi->data);
	double2* y = reinterpret_cast<double2*>(psi_out->data);
	// at most two nonzero entries (a basis vector, or a paired column e_b + i e_b'): only
	// their columns of U enter, in the same order and arithmetic as the full product
	int64_t nz[2] = { -1, -1 };
	int cnt = 0;
	for (int64_t j = 0; j < n && cnt <= 2; j++)
		if (x[j].x != 0 || x[j].y != 0) {
			if (cnt < 2) nz[cnt] = j;
			cnt++;
		}
	if (cnt == 1 && x[nz[0]].x == 1 && x[nz[0]].y == 0) {
		for (int64_t r = 0; r < n; r++) y[r] = u[r * n + nz[0]];
		return 0;
	}
	if (cnt <= 2) {
		for (int64_t r = 0; r < n; r++) {
			double sx = 0, sy = 0;
			for (int k = 0; k < cnt; k++) {
				const double2 a = u[r * n + nz[k]], b = x[nz[k]];
				sx += a.x * b.x - a.y * b.y;
				sy += a.x * b.y + a.y * b.x;
			}
			y[r] = make_double2(sx, sy);
		}
		return 0;
	}
	for (int64_t r = 0; r < n; r++) {
		double sx = 0, sy = 0;
		for (int64_t c = 0; c < n; c++) {
			const double2 a = u[r * n + c], b = x[c];
			sx += a.x * b.x - a.y * b.y;
			sy += a.x * b.y + a.y * b.x;
		}
		y[r] = make_double2(sx, sy);
	}
	return 0;
}

namespace rqc {

bool Problem::set_brickwall(int L_, int nlayers, const struct mat4x4* vlist, const struct mat4x4* vdirs,
                            const int* const* perms)
{
	L = L_;
	if (L < 2 || L % 2 || nlayers < 1 || !perms || !vlist) return false;
	per = L / 2;
	nunits = nlayers;
	G = nunits * per;
	gates.assign(16 * (size_t)G, make_double2(0, 0));
	dirs.assign(vdirs ? 16 * (size_t)G : 0, make_double2(0, 0));
	wires.resize(2 * (size_t)G);
	ugates.assign(reinterpret_cast<const double2*>(vlist), reinterpret_cast<const double2*>(vlist) + 16 * nunits);
	udirs.clear();
	if (vdirs) udirs.assign(reinterpret_cast<const double2*>(vdirs), reinterpret_cast<const double2*>(vdirs) + 16 * nunits);
	for (int l = 0; l < nlayers; l++) {
		if (!perms[l]) return false;
		for (int p = 0; p < per; p++) {
			const int k = l * per + p;
			wires[2 * k] = perms[l][2 * p];
			wires[2 * k + 1] = perms[l][2 * p + 1];
			memcpy(&gates[16 * (size_t)k], &ugates[16 * (size_t)l], 16 * sizeof(double2));
			if (vdirs) memcpy(&dirs[16 * (size_t)k], &udirs[16 * (size_t)l], 16 * sizeof(double2));
		}
	}
	return valid();
}

bool Problem::set_circuit(int L_, int ngates, const struct mat4x4* g, const struct mat4x4* z, const int* w)
{
	L = L_;
	if (L < 2 || ngates < 1 || !g || !w) return false;
	per = 1;
	nunits = G = ngates;
	gates.assign(reinterpret_cast<const double2*>(g), reinterpret_cast<const double2*>(g) + 16 * (size_t)G);
	dirs.clear();
	if (z) dirs.assign(reinterpret_cast<const double2*>(z), reinterpret_cast<const double2*>(z) + 16 * (size_t)G);
	wires.assign(w, w + 2 * (size_t)G);
	ugates = gates;
	udirs = dirs;
	return valid();
}

bool Problem::valid() const
{
	for (int k = 0; k < G; k++) {
		const int i = wires[2 * k], j = wires[2 * k + 1];
		if (i < 0 || j < 0 || i >= L || j >= L || i == j) return false;
	}
	return true;
}

void Problem::set_gates_from_units(const double2* u)
{
	memcpy(ugates.data(), u, 16 * (size_t)nunits * sizeof(double2));
	for (int k = 0; k < G; k++) memcpy(&gates[16 * (size_t)k], &ugates[16 * (size_t)(k / per)], 16 * sizeof(double2));
}

void Problem::set_dirs_from_units(const double2* z)
{
	udirs.assign(z, z + 16 * (size_t)nunits);
	dirs.resize(16 * (size_t)G);
	for (int k = 0; k < G; k++) memcpy(&dirs[16 * (size_t)k], &udirs[16 * (size_t)(k / per)], 16 * sizeof(double2));
}

bool TargetHolder::set(linear_func ufunc, void* udata, int L)
{
	spec = TargetSpec();
	if (!ufunc) return false;
	if (ufunc == rqcopt_brickwall_ufunc) {
		const struct rqcopt_brickwall_target* t = static_cast<const struct rqcopt_brickwall_target*>(udata);
		Problem p;
		if (!t || !p.set_brickwall(L, t->nlayers, t->vlist, nullptr, t->perms)) return false;
		gates = p.gates;
		wires = p.wires;
	} else if (ufunc == rqcopt_circuit_ufunc) {
		const struct rqcopt_circuit_target* t = static_cast<const struct rqcopt_circuit_target*>(udata);
		Problem p;
		if (!t || !p.set_circuit(L, t->ngates, t->gates, nullptr, t->wires)) return false;
		gates = p.gates;
		wires = p.wires;
	} else {
		spec.ufunc = reinterpret_cast<void*>(ufunc);
		spec.udata = udata;
		return true;
	}
	spec.ngates = (int)(wires.size() / 2);
	spec.gates = gates.data();
	spec.wires = wires.data();
	return true;
}

// Fold per-gate sums into per-unit sums and project (src/target.c:410-430, 526-535, 652-672).
// res: engine record; outputs (device): dunits/hunits [nunits][16] unprojected sums,
// grad_vec/hvp_vec [16 nunits] (either may be null).
__global__ void k_post(const double2* __restrict__ res, int G, int nunits, int per, const double2* __restrict__ ugates,
                       const double2* __restrict__ udirs, int with_hvp, double2* __restrict__ dunits,
                       double2* __restrict__ hunits, double* __restrict__ grad_vec, double* __restrict__ hvp_vec)
{
	const int u = blockIdx.x * blockDim.x + threadIdx.x;
	if (u >= nunits) return;
	M4 dg, hg;
	for (int e = 0; e < 16; e++) { dg.a[e] = c_(0, 0); hg.a[e] = c_(0, 0); }
	for (int p = 0; p < per; p++) {
		const int k = u * per + p;
		for (int e = 0; e < 16; e++) {
			dg.a[e] = c_add(dg.a[e], res[1 + 16 * (size_t)k + e]);
			if (with_hvp) hg.a[e] = c_add(hg.a[e], res[1 + 16 * (size_t)G + 16 * (size_t)k + e]);
		}
	}
	for (int e = 0; e < 16; e++) {
		if (dunits) dunits[16 * (size_t)u + e] = dg.a[e];
		if (hunits && with_hvp) hunits[16 * (size_t)u + e] = hg.a[e];
	}
	if (grad_vec) {
		M4 g, z;
		for (int e = 0; e < 16; e++) g.a[e] = ugates[16 * (size_t)u + e];
		if (with_hvp && hvp_vec)
			for (int e = 0; e < 16; e++) z.a[e] = udirs[16 * (size_t)u + e];
		m4_project_grad_hvp(g, (with_hvp && hvp_vec) ? &z : nullptr, dg, (with_hvp && hvp_vec) ? &hg : nullptr,
		                    grad_vec + 16 * (size_t)u, (with_hvp && hvp_vec) ? hvp_vec + 16 * (size_t)u : nullptr);
	}
}

int post_launch(Runtime& rt, const double2* d_res, const Problem& pb, const double2* d_ugates, const double2* d_udirs,
                int with_hvp, double2* d_dunits, double2* d_hunits, double* d_grad, double* d_hvp)
{
	const int threads = 64;
	const int blocks = (pb.nunits + threads - 1) / threads;
	k_post<<<blocks, threads, 0, rt.stream>>>(d_res, pb.G, pb.nunits, pb.per, d_ugates, d_udirs, with_hvp, d_dunits,
	                                          d_hunits, d_grad, d_hvp);
	rt.launches++;
	return RQC_CUDA(cudaGetLastError());
}

// One evaluation of a target function through the engine, with host outputs.
int run_target(const Problem& pb, const TargetHolder& th, int mode, numeric* fval, struct mat4x4* dunits,
               struct mat4x4* hunits, double* grad_vec, double* hvp_vec)
{
	Runtime* rt = runtime();
	if (!rt) return E_CUDA;
	CircuitSpec cs;
	cs.L = pb.L;
	cs.ngates = pb.G;
	cs.gates = pb.gates.data();
	cs.dirs = mode == EVAL_HVP ? pb.dirs.data() : nullptr;
	cs.wires = pb.wires.data();
	const int prec = rt->precision == PREC_C128 ? PREC_C128 : PREC_C64;
	const size_t nres = result_count(pb.G);
	const size_t nu = (size_t)pb.nunits;
	// device layout in rt.opt: res | ugates | udirs | dunits | hunits | grad | hvp
	const size_t bytes = (nres + 4 * 16 * nu) * sizeof(double2) + 2 * 16 * nu * sizeof(double);
	int ret = ensure_device(rt->result, bytes);
	if (ret) return ret;
	double2* d_res = reinterpret_cast<double2*>(rt->result.ptr);
	double2* d_ug = d_res + nres;
	double2* d_uz = d_ug + 16 * nu;
	double2* d_du = d_uz + 16 * nu;
	double2* d_hu = d_du + 16 * nu;
	double* d_gv = reinterpret_cast<double*>(d_hu + 16 * nu);
	double* d_hv = d_gv + 16 * nu;
	// evaluate() may use rt->result for nothing else; the record goes to d_res
	if ((ret = RQC_CUDA(cudaMemcpyAsync(d_ug, pb.ugates.data(), 16 * nu * sizeof(double2), cudaMemcpyHostToDevice, rt->stream))))
		return ret;
	if (mode == EVAL_HVP &&
	    (ret = RQC_CUDA(cudaMemcpyAsync(d_uz, pb.udirs.data(), 16 * nu * sizeof(double2), cudaMemcpyHostToDevice, rt->stream))))
		return ret;
	if ((ret = evaluate(*rt, cs, th.spec, mode, prec, d_res))) return ret;
	if ((ret = post_launch(*rt, d_res, pb, d_ug, d_uz, mode == EVAL_HVP, d_du, d_hu, grad_vec ? d_gv : nullptr,
	                       hvp_vec ? d_hv : nullptr)))
		return ret;
	auto d2h = [&](void* dst, const void* src, size_t n) {
		return RQC_CUDA(cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, rt->stream));
	};
	if (fval && (ret = d2h(fval, d_res, sizeof(double2)))) return ret;
	if (dunits && (ret = d2h(dunits, d_du, 16 * nu * sizeof(double2)))) return ret;
	if (hunits && mode == EVAL_HVP && (ret = d2h(hunits, d_hu, 16 * nu * sizeof(double2)))) return ret;
	if (grad_vec && (ret = d2h(grad_vec, d_gv, 16 * nu * sizeof(double)))) return ret;
	if (hvp_vec && mode == EVAL_HVP && (ret = d2h(hvp_vec, d_hv, 16 * nu * sizeof(double)))) return ret;
	return sync(*rt);
}

}  // namespace rqc

// ------------------------------------------------------------------ exported target functions

namespace {

int report(const char* fn, int ret)
{
	if (ret == E_ARG) fprintf(stderr, "rqcopt_gpu: %s: invalid arguments\n", fn);
	return ret;
}

}  // namespace

extern "C" int circuit_unitary_target(linear_func ufunc, void* udata, const struct mat4x4 gates[], const int ngates,
                                      const int wires[], const int nqubits, numeric* fval)
{
	Problem pb;
	TargetHolder th;
	if (!pb.set_circuit(nqubits, ngates, gates, nullptr, wires) || !th.set(ufunc, udata, nqubits))
		return report("circuit_unitary_target", E_ARG);
	return run_target(pb, th, EVAL_F, fval, nullptr, nullptr, nullptr, nullptr);
}

extern "C" int circuit_unitary_target_and_gradient(linear_func ufunc, void* udata, const struct mat4x4 gates[],
                                                   const int ngates, const int wires[], const int nqubits, numeric* fval,
                                                   struct mat4x4 dgates[])
{
	Problem pb;
	TargetHolder th;
	if (!pb.set_circuit(nqubits, ngates, gates, nullptr, wires) || !th.set(ufunc, udata, nqubits))
		return report("circuit_unitary_target_and_gradient", E_ARG);
	return run_target(pb, th, EVAL_GRAD, fval, dgates, nullptr, nullptr, nullptr);
}

extern "C" int circuit_unitary_target_and_projected_gradient(linear_func ufunc, void* udata, const struct mat4x4 gates[],
                                                             const int ngates, const int wires[], const int nqubits,
                                                             numeric* fval, double* grad_vec)
{
	Problem pb;
	TargetHolder th;
	if (!pb.set_circuit(nqubits, ngates, gates, nullptr, wires) || !th.set(ufunc, udata, nqubits))
		return report("circuit_unitary_target_and_projected_gradient", E_ARG);
	return run_target(pb, th, EVAL_GRAD, fval, nullptr, nullptr, grad_vec, nullptr);
}

extern "C" int circuit_unitary_target_hessian_vector_product(linear_func ufunc, void* udata, const struct mat4x4 gates[],
                                                             const struct mat4x4 gatedirs[], const int ngates,
                                                             const int wires[], const int nqubits, numeric* fval,
                                                             struct mat4x4 dgates[], struct mat4x4 hess_gatedirs[])
{
	Problem pb;
	TargetHolder th;
	if (!gatedirs || !pb.set_circuit(nqubits, ngates, gates, gatedirs, wires) || !th.set(ufunc, udata, nqubits))
		return report("circuit_unitary_target_hessian_vector_product", E_ARG);
	return run_target(pb, th, EVAL_HVP, fval, dgates, hess_gatedirs, nullptr, nullptr);
}

extern "C" int circuit_unitary_target_projected_hessian_vector_product(linear_func ufunc, void* udata,
                                                                       const struct mat4x4 gates[],
                                                                       const struct mat4x4 gatedirs[], const int ngates,
                                                                       const int wires[], const int nqubits,
                                                                       numeric* fval, double* grad_vec, double* hvp_vec)
{
	Problem pb;
	TargetHolder th;
	if (!gatedirs || !pb.set_circuit(nqubits, ngates, gates, gatedirs, wires) || !th.set(ufunc, udata, nqubits))
		return report("circuit_unitary_target_projected_hessian_vector_product", E_ARG);
	const int ret = run_target(pb, th, EVAL_HVP, fval, nullptr, nullptr, grad_vec, hvp_vec);
	return ret < 0 ? (ret == E_ARG ? ret : -2) : 0;
}

extern "C" int brickwall_unitary_target(linear_func ufunc, void* udata, const struct mat4x4 vlist[], const int nlayers,
                                        const int nqubits, const int* perms[], numeric* fval)
{
	Problem pb;
	TargetHolder th;
	if (!pb.set_brickwall(nqubits, nlayers, vlist, nullptr, perms) || !th.set(ufunc, udata, nqubits))
		return report("brickwall_unitary_target", E_ARG);
	return run_target(pb, th, EVAL_F, fval, nullptr, nullptr, nullptr, nullptr);
}

extern "C" int brickwall_unitary_target_and_gradient(linear_func ufunc, void* udata, const struct mat4x4 vlist[],
                                                     const int nlayers, const int nqubits, const int* perms[],
                                                     numeric* fval, struct mat4x4 dvlist[])
{
	Problem pb;
	TargetHolder th;
	if (!pb.set_brickwall(nqubits, nlayers, vlist, nullptr, perms) || !th.set(ufunc, udata, nqubits))
		return report("brickwall_unitary_target_and_gradient", E_ARG);
	return run_target(pb, th, EVAL_GRAD, fval, dvlist, nullptr, nullptr, nullptr);
}

extern "C" int brickwall_unitary_target_and_projected_gradient(linear_func ufunc, void* udata, const struct mat4x4 vlist[],
                                                               const int nlayers, const int nqubits, const int* perms[],
                                                               numeric* fval, double* grad_vec)
{
	Problem pb;
	TargetHolder th;
	if (!pb.set_brickwall(nqubits, nlayers, vlist, nullptr, perms) || !th.set(ufunc, udata, nqubits))
		return report("brickwall_unitary_target_and_projected_gradient", E_ARG);
	return run_target(pb, th, EVAL_GRAD, fval, nullptr, nullptr, grad_vec, nullptr);
}

extern "C" int brickwall_unitary_target_hessian_vector_product(linear_func ufunc, void* udata, const struct mat4x4 vlist[],
                                                               const struct mat4x4 vdirs[], const int nlayers,
                                                               const int* perms[], const int nqubits, numeric* fval,
                                                               struct mat4x4 dvlist[], struct mat4x4 hess_vdirs[])
{
	Problem pb;
	TargetHolder th;
	if (!vdirs || !pb.set_brickwall(nqubits, nlayers, vlist, vdirs, perms) || !th.set(ufunc, udata, nqubits))
		return report("brickwall_unitary_target_hessian_vector_product", E_ARG);
	return run_target(pb, th, EVAL_HVP, fval, dvlist, hess_vdirs, nullptr, nullptr);
}

extern "C" int brickwall_unitary_target_projected_hessian_vector_product(linear_func ufunc, void* udata,
                                                                         const struct mat4x4 vlist[],
                                                                         const struct mat4x4 vdirs[], const int nlayers,
                                                                         const int* perms[], const int nqubits,
                                                                         numeric* fval, double* grad_vec, double* hvp_vec)
{
	Problem pb;
	TargetHolder th;
	if (!vdirs || !pb.set_brickwall(nqubits, nlayers, vlist, vdirs, perms) || !th.set(ufunc, udata, nqubits))
		return report("brickwall_unitary_target_projected_hessian_vector_product", E_ARG);
	const int ret = run_target(pb, th, EVAL_HVP, fval, nullptr, nullptr, grad_vec, hvp_vec);
	return ret < 0 ? (ret == E_ARG ? ret : -2) : 0;
}
