// Exported functions of the full-Hessian path with the reference's signatures:
// statevector arrays (src/statevector.h:39-49), the array gate kernels
// (src/gate.h:13-19), the brickwall backward pass with Hessian and the gate
// placeholder circuit (src/brickwall_circuit.h:17-22), the Hessian targets
// (src/target.h:70-83), the random-state sampling estimators with their
// generator (src/target.h:14-17, 46-49, 74-77, 85-88; src/rng.h:21;
// src/statevector.h:29) and the block-encoding target (src/target.h:96-126).  Host buffers are staged through HBM; every call
// synchronises before returning.
#include <stdio.h>
#include <string.h>
#include <vector>

#include "hess.h"
#include "rqc_runtime.h"
#include "rqcopt_gpu.h"
#include "sampling.h"
#include "target_problem.h"

using namespace rqc;

namespace {

inline size_t sv_bytes(int L) { return ((size_t)1 << L) * sizeof(double2); }
inline const double2* d2(const numeric* p) { return reinterpret_cast<const double2*>(p); }

bool wires_ok(int L, int i, int j) { return L >= 2 && L <= 40 && i >= 0 && j >= 0 && i < L && j < L && i != j; }

// layer gates and sequential wires of a brickwall (src/target.c:443-458 order)
bool brickwall_of(int L, int nlayers, const struct mat4x4* vlist, const int* const* perms, std::vector<double2>& ug,
                  std::vector<int>& wires)
{
	if (L < 2 || L % 2 || L > 40 || nlayers < 1 || !vlist || !perms) return false;
	const int per = L / 2;
	ug.assign(d2(vlist[0].data), d2(vlist[0].data) + 16 * (size_t)nlayers);
	wires.resize(2 * (size_t)nlayers * per);
	for (int l = 0; l < nlayers; l++) {
		if (!perms[l]) return false;
		for (int p = 0; p < per; p++) {
			const int k = l * per + p;
			wires[2 * k] = perms[l][2 * p];
			wires[2 * k + 1] = perms[l][2 * p + 1];
			if (!wires_ok(L, wires[2 * k], wires[2 * k + 1])) return false;
		}
	}
	return true;
}

int fail(const char* fn, int code)
{
	if (code == E_ARG) fprintf(stderr, "rqcopt_gpu: %s: invalid arguments\n", fn);
	return code;
}

void fail_void(const char* fn, int code)
{
	if (code == E_ARG) fail_arg(fn, "invalid arguments");
	else set_last_error(code);
}

int d2h(Runtime& rt, void* dst, const void* src, size_t bytes)
{
	return RQC_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, rt.stream));
}

}  // namespace

// ------------------------------------------------------------------ statevector arrays

extern "C" int allocate_statevector_array(int nqubits, int nstates, struct statevector_array* psi_list)
{
	psi_list->nqubits = nqubits;
	psi_list->nstates = nstates;
	psi_list->data = nullptr;
	if (nqubits < 0 || nqubits > 40 || nstates < 1) {
		fprintf(stderr, "rqcopt_gpu: allocate_statevector_array: invalid size (%d qubits, %d states)\n", nqubits, nstates);
		return -1;
	}
	if (!runtime()) return -1;
	void* p = nullptr;
	const size_t bytes = ((size_t)1 << nqubits) * (size_t)nstates * sizeof(numeric);
	if (cudaMallocManaged(&p, bytes, cudaMemAttachGlobal) != cudaSuccess) {
		cudaGetLastError();
		fprintf(stderr, "allocating statevector array memory (%zu bytes) failed\n", bytes);
		return -1;
	}
	psi_list->data = static_cast<numeric*>(p);
	return 0;
}

extern "C" void free_statevector_array(struct statevector_array* psi_list)
{
	if (psi_list->data) {
		if (is_device_pointer(psi_list->data)) cudaFree(psi_list->data);
		else fprintf(stderr, "rqcopt_gpu: free_statevector_array: pointer was not allocated by allocate_statevector_array\n");
	}
	psi_list->data = nullptr;
	psi_list->nqubits = 0;
	psi_list->nstates = 0;
}

// ------------------------------------------------------------------ array gate kernels

extern "C" void apply_gate_to_array(const struct mat4x4* gate, const int i, const int j,
                                    const struct statevector_array* psi, struct statevector_array* psi_out)
{
	const char* fn = "apply_gate_to_array";
	if (!gate || !psi || !psi_out || !psi->data || !psi_out->data || psi->nqubits != psi_out->nqubits ||
	    psi->nstates != psi_out->nstates || psi->nstates < 1 || !wires_ok(psi->nqubits, i, j))
		return fail_void(fn, E_ARG);
	Runtime* rt = runtime();
	if (!rt) return fail_void(fn, E_CUDA);
	const size_t bytes = sv_bytes(psi->nqubits) * psi->nstates;
	DeviceSpan in, out;
	int ret = span_in(*rt, psi->data, bytes, 0, in);
	if (!ret) ret = span_out(*rt, psi_out->data, bytes, 1, out);
	if (!ret) ret = gate_to_array_device(*rt, psi->nqubits, psi->nstates, d2(gate->data), i, j,
	                                     static_cast<const double2*>(in.dev), static_cast<double2*>(out.dev));
	if (!ret) ret = span_finish(*rt, out);
	if (!ret) ret = sync(*rt);
	if (ret) fail_void(fn, ret);
}

extern "C" void apply_gate_backward_array(const struct mat4x4* gate, const int i, const int j,
                                          const struct statevector_array* psi, const struct statevector* dpsi_out,
                                          struct mat4x4* dgates)
{
	const char* fn = "apply_gate_backward_array";
	// the gate itself does not enter the gate gradients (src/gate.c:269-377)
	if (!gate || !psi || !dpsi_out || !dgates || !psi->data || !dpsi_out->data || psi->nqubits != dpsi_out->nqubits ||
	    psi->nstates < 1 || !wires_ok(psi->nqubits, i, j))
		return fail_void(fn, E_ARG);
	Runtime* rt = runtime();
	if (!rt) return fail_void(fn, E_CUDA);
	const int L = psi->nqubits, ns = psi->nstates;
	DeviceSpan in, dout;
	int ret = span_in(*rt, psi->data, sv_bytes(L) * ns, 0, in);
	if (!ret) ret = span_in(*rt, dpsi_out->data, sv_bytes(L), 1, dout);
	if (!ret) ret = ensure_device(rt->result, 16 * (size_t)ns * sizeof(double2));
	double2* d_dg = static_cast<double2*>(rt->result.ptr);
	if (!ret) ret = gate_backward_array_device(*rt, L, ns, i, j, static_cast<const double2*>(in.dev),
	                                           static_cast<const double2*>(dout.dev), d_dg);
	if (!ret) ret = d2h(*rt, dgates, d_dg, 16 * (size_t)ns * sizeof(double2));
	if (!ret) ret = sync(*rt);
	if (ret) fail_void(fn, ret);
}

extern "C" void apply_gate_placeholder(const int i, const int j, const struct statevector* psi,
                                       struct statevector_array* psi_out)
{
	const char* fn = "apply_gate_placeholder";
	if (!psi || !psi_out || !psi->data || !psi_out->data || psi->nqubits != psi_out->nqubits || psi_out->nstates != 16 ||
	    !wires_ok(psi->nqubits, i, j))
		return fail_void(fn, E_ARG);
	Runtime* rt = runtime();
	if (!rt) return fail_void(fn, E_CUDA);
	const int L = psi->nqubits;
	DeviceSpan in, out;
	int ret = span_in(*rt, psi->data, sv_bytes(L), 0, in);
	if (!ret) ret = span_out(*rt, psi_out->data, sv_bytes(L) * 16, 1, out);
	if (!ret) ret = gate_placeholder_device(*rt, L, i, j, static_cast<const double2*>(in.dev), static_cast<double2*>(out.dev));
	if (!ret) ret = span_finish(*rt, out);
	if (!ret) ret = sync(*rt);
	if (ret) fail_void(fn, ret);
}

// ------------------------------------------------------------------ brickwall with Hessian

extern "C" int brickwall_unitary_backward_hessian(const struct mat4x4 vlist[], int nlayers, const int* perms[],
                                                  const struct quantum_circuit_cache* cache,
                                                  const struct statevector* dpsi_out, struct statevector* dpsi,
                                                  struct mat4x4 dvlist[], numeric* hess)
{
	const char* fn = "brickwall_unitary_backward_hessian";
	std::vector<double2> ug;
	std::vector<int> wires;
	if (!dpsi || !dpsi_out || !cache || !dvlist || !hess || !dpsi->data || !dpsi_out->data ||
	    dpsi_out->nqubits != dpsi->nqubits || !brickwall_of(dpsi->nqubits, nlayers, vlist, perms, ug, wires) ||
	    cache->nqubits != dpsi->nqubits || cache->ngates != nlayers * (dpsi->nqubits / 2) || !cache->psi_list)
		return fail(fn, E_ARG);
	Runtime* rt = runtime();
	if (!rt) return E_CUDA;
	const int L = dpsi->nqubits, G = cache->ngates, m = 16 * nlayers;
	const size_t N = (size_t)1 << L;
	for (int k = 0; k < G; k++)
		if (!cache->psi_list[k].data || cache->psi_list[k].nqubits != L) return fail(fn, E_ARG);
	int ret = ensure_device(rt->arrays, (size_t)G * N * sizeof(double2));
	if (ret) return ret;
	double2* d_cache = static_cast<double2*>(rt->arrays.ptr);
	for (int k = 0; k < G && !ret; k++)
		ret = RQC_CUDA(cudaMemcpyAsync(d_cache + (size_t)k * N, cache->psi_list[k].data, N * sizeof(double2),
		                               cudaMemcpyDefault, rt->stream));
	DeviceSpan dout, dp;
	if (!ret) ret = span_in(*rt, dpsi_out->data, sv_bytes(L), 0, dout);
	if (!ret) ret = span_out(*rt, dpsi->data, sv_bytes(L), 1, dp);
	if (!ret) ret = ensure_device(rt->result, hess_record_count(nlayers) * sizeof(double2));
	double2* rec = static_cast<double2*>(rt->result.ptr);
	HessCircuit c;
	c.L = L;
	c.nlayers = nlayers;
	c.ugates = ug.data();
	c.wires = wires.data();
	if (!ret) ret = hessian_single_device(*rt, c, d_cache, static_cast<const double2*>(dout.dev),
	                                      static_cast<double2*>(dp.dev), rec);
	if (!ret) ret = span_finish(*rt, dp);
	if (!ret) ret = d2h(*rt, dvlist, rec + 1, 16 * (size_t)nlayers * sizeof(double2));
	if (!ret) ret = d2h(*rt, hess, rec + 1 + 16 * nlayers, (size_t)m * m * sizeof(double2));
	if (!ret) ret = sync(*rt);
	return ret;
}

extern "C" int apply_brickwall_unitary_gate_placeholder(const struct mat4x4 vlist[], int nlayers, const int* perms[],
                                                        int l, const struct quantum_circuit_cache* cache,
                                                        struct statevector_array* psi_out)
{
	const char* fn = "apply_brickwall_unitary_gate_placeholder";
	std::vector<double2> ug;
	std::vector<int> wires;
	if (!cache || !psi_out || !psi_out->data || psi_out->nstates != 16 || cache->nqubits != psi_out->nqubits ||
	    !brickwall_of(cache->nqubits, nlayers, vlist, perms, ug, wires) || cache->ngates != nlayers * (cache->nqubits / 2) ||
	    l < 0 || l >= nlayers || !cache->psi_list)
		return fail(fn, E_ARG);
	Runtime* rt = runtime();
	if (!rt) return E_CUDA;
	const int L = cache->nqubits, per = L / 2, G = cache->ngates;
	const size_t N = (size_t)1 << L;
	for (int p = 0; p < per; p++)
		if (!cache->psi_list[l * per + p].data || cache->psi_list[l * per + p].nqubits != L) return fail(fn, E_ARG);
	// device: two 16-state arrays and one input state
	int ret = ensure_device(rt->arrays, (32 * N + N) * sizeof(double2));
	if (ret) return ret;
	double2* t[2] = { static_cast<double2*>(rt->arrays.ptr), static_cast<double2*>(rt->arrays.ptr) + 16 * N };
	double2* d_psi = t[1] + 16 * N;
	DeviceSpan out;
	if ((ret = span_out(*rt, psi_out->data, 16 * N * sizeof(double2), 0, out))) return ret;
	double2* acc = static_cast<double2*>(out.dev);
	for (int p = 0; p < per && !ret; p++) {
		const int k = l * per + p;
		ret = RQC_CUDA(cudaMemcpyAsync(d_psi, cache->psi_list[k].data, N * sizeof(double2), cudaMemcpyDefault, rt->stream));
		if (!ret) ret = gate_placeholder_device(*rt, L, wires[2 * k], wires[2 * k + 1], d_psi, t[0]);
		int cur = 0;
		for (int q = k + 1; q < G && !ret; q++) {
			ret = gate_to_array_device(*rt, L, 16, &ug[16 * (size_t)(q / per)], wires[2 * q], wires[2 * q + 1], t[cur],
			                           t[1 - cur]);
			cur = 1 - cur;
		}
		if (!ret) ret = p == 0 ? RQC_CUDA(cudaMemcpyAsync(acc, t[cur], 16 * N * sizeof(double2), cudaMemcpyDeviceToDevice,
		                                                  rt->stream))
		                       : add_device(*rt, acc, t[cur], acc, (long)(16 * N));
	}
	if (!ret) ret = span_finish(*rt, out);
	if (!ret) ret = sync(*rt);
	return ret;
}

// ------------------------------------------------------------------ Hessian targets

namespace {

int hessian_target(const char* fn, linear_func ufunc, void* udata, const struct mat4x4 vlist[], int nlayers,
                   int nqubits, const int* perms[], numeric* fval, struct mat4x4* dvlist, numeric* hess,
                   double* grad_vec, double* H, const SampleSpec* samp = nullptr)
{
	std::vector<double2> ug;
	std::vector<int> wires;
	TargetHolder th;
	if (!brickwall_of(nqubits, nlayers, vlist, perms, ug, wires) || !th.set(ufunc, udata, nqubits))
		return fail(fn, E_ARG);
	Runtime* rt = runtime();
	if (!rt) return E_CUDA;
	const int m = 16 * nlayers;
	const size_t nrec = hess_record_count(nlayers);
	// device: record | layer gates | gradient vector | real Hessian
	int ret = ensure_device(rt->result, (nrec + 16 * (size_t)nlayers) * sizeof(double2) + ((size_t)m + (size_t)m * m) * sizeof(double));
	if (ret) return ret;
	double2* rec = static_cast<double2*>(rt->result.ptr);
	double2* d_ug = rec + nrec;
	double* d_grad = reinterpret_cast<double*>(d_ug + 16 * nlayers);
	double* d_H = d_grad + m;
	HessCircuit c;
	c.L = nqubits;
	c.nlayers = nlayers;
	c.ugates = ug.data();
	c.wires = wires.data();
	if ((ret = hessian_target_device(*rt, c, th.spec, rec, samp))) return ret;
	if (H) {
		if ((ret = RQC_CUDA(cudaMemcpyAsync(d_ug, ug.data(), 16 * (size_t)nlayers * sizeof(double2), cudaMemcpyHostToDevice,
		                                    rt->stream))))
			return ret;
		if ((ret = project_hessian_device(*rt, nlayers, d_ug, rec, d_grad, d_H))) return ret;
		if ((ret = d2h(*rt, grad_vec, d_grad, m * sizeof(double)))) return ret;
		if ((ret = d2h(*rt, H, d_H, (size_t)m * m * sizeof(double)))) return ret;
	} else {
		if ((ret = d2h(*rt, dvlist, rec + 1, 16 * (size_t)nlayers * sizeof(double2)))) return ret;
		if ((ret = d2h(*rt, hess, rec + 1 + 16 * nlayers, (size_t)m * m * sizeof(double2)))) return ret;
	}
	if ((ret = d2h(*rt, fval, rec, sizeof(double2)))) return ret;
	return sync(*rt);
}

}  // namespace

extern "C" int brickwall_unitary_target_gradient_hessian(linear_func ufunc, void* udata, const struct mat4x4 vlist[],
                                                         const int nlayers, const int nqubits, const int* perms[],
                                                         numeric* fval, struct mat4x4 dvlist[], numeric* hess)
{
	if (!fval || !dvlist || !hess) return fail("brickwall_unitary_target_gradient_hessian", E_ARG);
	return hessian_target("brickwall_unitary_target_gradient_hessian", ufunc, udata, vlist, nlayers, nqubits, perms,
	                      fval, dvlist, hess, nullptr, nullptr);
}

extern "C" int brickwall_unitary_target_gradient_vector_hessian_matrix(linear_func ufunc, void* udata,
                                                                       const struct mat4x4 vlist[], const int nlayers,
                                                                       const int nqubits, const int* perms[],
                                                                       numeric* fval, double* grad_vec, double* H)
{
	if (!fval || !grad_vec || !H) return fail("brickwall_unitary_target_gradient_vector_hessian_matrix", E_ARG);
	return hessian_target("brickwall_unitary_target_gradient_vector_hessian_matrix", ufunc, udata, vlist, nlayers,
	                      nqubits, perms, fval, nullptr, nullptr, grad_vec, H);
}

extern "C" int brickwall_unitary_target_gradient_hessian_sampling(linear_func ufunc, void* udata,
                                                                  const struct mat4x4 vlist[], const int nlayers,
                                                                  const int nqubits, const int* perms[],
                                                                  const long nsamples, struct rng_state* rng,
                                                                  numeric* fval, struct mat4x4 dvlist[], numeric* hess)
{
	const char* fn = "brickwall_unitary_target_gradient_hessian_sampling";
	if (!fval || !dvlist || !hess || !rng || nsamples < 1) return fail(fn, E_ARG);
	const SampleSpec sp = sample_spec(rng, nsamples);
	const int ret = hessian_target(fn, ufunc, udata, vlist, nlayers, nqubits, perms, fval, dvlist, hess, nullptr,
	                               nullptr, &sp);
	if (!ret) advance_rng(rng, nsamples, nqubits);
	return ret;
}

extern "C" int brickwall_unitary_target_gradient_vector_hessian_matrix_sampling(linear_func ufunc, void* udata,
                                                                                const struct mat4x4 vlist[],
                                                                                const int nlayers, const int nqubits,
                                                                                const int* perms[], const long nsamples,
                                                                                struct rng_state* rng, numeric* fval,
                                                                                double* grad_vec, double* H)
{
	const char* fn = "brickwall_unitary_target_gradient_vector_hessian_matrix_sampling";
	if (!fval || !grad_vec || !H || !rng || nsamples < 1) return fail(fn, E_ARG);
	const SampleSpec sp = sample_spec(rng, nsamples);
	const int ret = hessian_target(fn, ufunc, udata, vlist, nlayers, nqubits, perms, fval, nullptr, nullptr, grad_vec, H,
	                               &sp);
	if (!ret) advance_rng(rng, nsamples, nqubits);
	return ret;
}

// ------------------------------------------------------------------ generator and sampled target values

namespace {

int sampled_value(const char* fn, linear_func ufunc, void* udata, const std::vector<double2>& gates,
                  const std::vector<int>& wires, int nqubits, long nsamples, struct rng_state* rng, numeric* fval)
{
	TargetHolder th;
	if (!th.set(ufunc, udata, nqubits)) return fail(fn, E_ARG);
	Runtime* rt = runtime();
	if (!rt) return E_CUDA;
	int ret = ensure_device(rt->result, sizeof(double2));
	if (ret) return ret;
	double2* d_f = static_cast<double2*>(rt->result.ptr);
	if ((ret = sampled_f_device(*rt, nqubits, (int)(wires.size() / 2), gates.data(), wires.data(), th.spec,
	                            sample_spec(rng, nsamples), d_f)))
		return ret;
	if ((ret = d2h(*rt, fval, d_f, sizeof(double2)))) return ret;
	if ((ret = sync(*rt))) return ret;
	advance_rng(rng, nsamples, nqubits);
	return OK;
}

}  // namespace

extern "C" void haar_random_statevector(struct statevector* psi, struct rng_state* rng)
{
	const char* fn = "haar_random_statevector";
	if (!psi || !psi->data || !rng || psi->nqubits < 0 || psi->nqubits > 40) return fail_void(fn, E_ARG);
	Runtime* rt = runtime();
	if (!rt) return fail_void(fn, E_CUDA);
	const int L = psi->nqubits;
	DeviceSpan out;
	int ret = span_out(*rt, psi->data, sv_bytes(L), 0, out);
	if (!ret) ret = haar_states_device(*rt, sample_spec(rng, 1), L, 0, 1, static_cast<double2*>(out.dev));
	if (!ret) ret = span_finish(*rt, out);
	if (!ret) ret = sync(*rt);
	if (ret) return fail_void(fn, ret);
	advance_rng(rng, 1, L);
}

extern "C" int circuit_unitary_target_sampling(linear_func ufunc, void* udata, const struct mat4x4 gates[],
                                               const int ngates, const int wires[], const int nqubits,
                                               const long nsamples, struct rng_state* rng, numeric* fval)
{
	const char* fn = "circuit_unitary_target_sampling";
	if (!gates || !wires || !rng || !fval || ngates < 1 || nsamples < 1 || nqubits < 2 || nqubits > 40)
		return fail(fn, E_ARG);
	for (int k = 0; k < ngates; k++)
		if (!wires_ok(nqubits, wires[2 * k], wires[2 * k + 1])) return fail(fn, E_ARG);
	std::vector<double2> g(d2(gates[0].data), d2(gates[0].data) + 16 * (size_t)ngates);
	std::vector<int> w(wires, wires + 2 * (size_t)ngates);
	return sampled_value(fn, ufunc, udata, g, w, nqubits, nsamples, rng, fval);
}

extern "C" int brickwall_unitary_target_sampling(linear_func ufunc, void* udata, const struct mat4x4 vlist[],
                                                 const int nlayers, const int nqubits, const int* perms[],
                                                 const long nsamples, struct rng_state* rng, numeric* fval)
{
	const char* fn = "brickwall_unitary_target_sampling";
	std::vector<double2> ug;
	std::vector<int> wires;
	if (!rng || !fval || nsamples < 1 || !brickwall_of(nqubits, nlayers, vlist, perms, ug, wires)) return fail(fn, E_ARG);
	const int per = nqubits / 2;
	std::vector<double2> g(16 * (size_t)nlayers * per);
	for (int k = 0; k < nlayers * per; k++)
		memcpy(&g[16 * (size_t)k], &ug[16 * (size_t)(k / per)], 16 * sizeof(double2));
	return sampled_value(fn, ufunc, udata, g, wires, nqubits, nsamples, rng, fval);
}

// ------------------------------------------------------------------ block-encoding target

namespace {

// mode 0: f; 1: f, dvlist / grad_vec; 2: f, dvlist, hess1, hess2 / grad_vec, H
int blockenc(const char* fn, linear_func hfunc, void* hdata, const struct mat4x4 vlist[], int nlayers, int nqubits,
             const int* perms[], int mode, double* fval, struct mat4x4* dvlist, double* grad_vec, numeric* hess1,
             numeric* hess2, double* H)
{
	std::vector<double2> ug;
	std::vector<int> wires;
	TargetHolder th;
	if (!fval || !brickwall_of(nqubits, nlayers, vlist, perms, ug, wires) || !th.set(hfunc, hdata, nqubits / 2))
		return fail(fn, E_ARG);
	Runtime* rt = runtime();
	if (!rt) return E_CUDA;
	const int m = 16 * nlayers;
	const size_t nrec = hess_record_count(nlayers);
	// device: record | hess2 | layer gates | gradient vector | real Hessian
	int ret = ensure_device(rt->result, (nrec + (size_t)m * m + 16 * (size_t)nlayers) * sizeof(double2) +
	                                        ((size_t)m + (size_t)m * m) * sizeof(double));
	if (ret) return ret;
	double2* rec = static_cast<double2*>(rt->result.ptr);
	double2* d_h2 = rec + nrec;
	double2* d_ug = d_h2 + (size_t)m * m;
	double* d_grad = reinterpret_cast<double*>(d_ug + 16 * nlayers);
	double* d_H = d_grad + m;
	HessCircuit c;
	c.L = nqubits;
	c.nlayers = nlayers;
	c.ugates = ug.data();
	c.wires = wires.data();
	if ((ret = blockenc_device(*rt, c, th.spec, mode, rec, d_h2))) return ret;
	if (grad_vec) {
		if ((ret = RQC_CUDA(cudaMemcpyAsync(d_ug, ug.data(), 16 * (size_t)nlayers * sizeof(double2), cudaMemcpyHostToDevice,
		                                    rt->stream))))
			return ret;
		if ((ret = project_hessian_device(*rt, nlayers, d_ug, rec, d_grad, d_H, mode == 2 ? d_h2 : nullptr))) return ret;
		if ((ret = d2h(*rt, grad_vec, d_grad, m * sizeof(double)))) return ret;
		if (H && (ret = d2h(*rt, H, d_H, (size_t)m * m * sizeof(double)))) return ret;
	}
	if (dvlist && (ret = d2h(*rt, dvlist, rec + 1, 16 * (size_t)nlayers * sizeof(double2)))) return ret;
	if (hess1 && (ret = d2h(*rt, hess1, rec + 1 + 16 * nlayers, (size_t)m * m * sizeof(double2)))) return ret;
	if (hess2 && (ret = d2h(*rt, hess2, d_h2, (size_t)m * m * sizeof(double2)))) return ret;
	double2 f;
	if ((ret = d2h(*rt, &f, rec, sizeof(double2)))) return ret;
	if ((ret = sync(*rt))) return ret;
	*fval = f.x;
	return OK;
}

}  // namespace

extern "C" int brickwall_blockenc_target(linear_func hfunc, void* hdata, const struct mat4x4 vlist[], const int nlayers,
                                         const int nqubits, const int* perms[], double* fval)
{
	return blockenc("brickwall_blockenc_target", hfunc, hdata, vlist, nlayers, nqubits, perms, 0, fval, nullptr, nullptr,
	                nullptr, nullptr, nullptr);
}

extern "C" int brickwall_blockenc_target_and_gradient(linear_func hfunc, void* hdata, const struct mat4x4 vlist[],
                                                      const int nlayers, const int nqubits, const int* perms[],
                                                      double* fval, struct mat4x4 dvlist[])
{
	if (!dvlist) return fail("brickwall_blockenc_target_and_gradient", E_ARG);
	return blockenc("brickwall_blockenc_target_and_gradient", hfunc, hdata, vlist, nlayers, nqubits, perms, 1, fval,
	                dvlist, nullptr, nullptr, nullptr, nullptr);
}

extern "C" int brickwall_blockenc_target_and_gradient_vector(linear_func hfunc, void* hdata, const struct mat4x4 vlist[],
                                                             const int nlayers, const int nqubits, const int* perms[],
                                                             double* fval, double* grad_vec)
{
	if (!grad_vec) return fail("brickwall_blockenc_target_and_gradient_vector", E_ARG);
	return blockenc("brickwall_blockenc_target_and_gradient_vector", hfunc, hdata, vlist, nlayers, nqubits, perms, 1,
	                fval, nullptr, grad_vec, nullptr, nullptr, nullptr);
}

extern "C" int brickwall_blockenc_target_gradient_hessian(linear_func hfunc, void* hdata, const struct mat4x4 vlist[],
                                                          const int nlayers, const int nqubits, const int* perms[],
                                                          double* fval, struct mat4x4 dvlist[], numeric* hess1,
                                                          numeric* hess2)
{
	if (!dvlist || !hess1 || !hess2) return fail("brickwall_blockenc_target_gradient_hessian", E_ARG);
	return blockenc("brickwall_blockenc_target_gradient_hessian", hfunc, hdata, vlist, nlayers, nqubits, perms, 2, fval,
	                dvlist, nullptr, hess1, hess2, nullptr);
}

extern "C" int brickwall_blockenc_target_gradient_vector_hessian_matrix(linear_func hfunc, void* hdata,
                                                                        const struct mat4x4 vlist[], const int nlayers,
                                                                        const int nqubits, const int* perms[],
                                                                        double* fval, double* grad_vec, double* H)
{
	if (!grad_vec || !H) return fail("brickwall_blockenc_target_gradient_vector_hessian_matrix", E_ARG);
	return blockenc("brickwall_blockenc_target_gradient_vector_hessian_matrix", hfunc, hdata, vlist, nlayers, nqubits,
	                perms, 2, fval, nullptr, grad_vec, nullptr, nullptr, H);
}
