// Exported statevector, gate, quantum-circuit and brickwall-circuit functions
// with the reference's signatures (src/statevector.h, src/gate.h,
// src/quantum_circuit.h, src/brickwall_circuit.h).  Every call stages host
// buffers through HBM as needed, runs its passes on the library stream and
// synchronises before returning.
#include <stdio.h>
#include <string.h>
#include <vector>

#include "engine.h"
#include "rqc_runtime.h"
#include "rqcopt_gpu.h"

using namespace rqc;

namespace {

inline size_t sv_bytes(int L) { return ((size_t)1 << L) * sizeof(double2); }
inline const double2* d2(const numeric* p) { return reinterpret_cast<const double2*>(p); }
inline double2* d2(numeric* p) { return reinterpret_cast<double2*>(p); }

bool valid_wires(int L, int i, int j) { return L >= 2 && i >= 0 && j >= 0 && i < L && j < L && i != j; }

bool valid_circuit(int L, int ngates, const int* wires)
{
	if (L < 2 || ngates < 1 || !wires) return false;
	for (int k = 0; k < ngates; k++)
		if (!valid_wires(L, wires[2 * k], wires[2 * k + 1])) return false;
	return true;
}

// Sequential gates and wires of a brickwall (src/target.c:443-458 layout).
bool expand_brickwall(int L, int nlayers, const struct mat4x4* vlist, const int* const* perms,
                      std::vector<double2>* gates, std::vector<int>& wires)
{
	if (L < 2 || L % 2 != 0 || nlayers < 1 || !perms) return false;
	const int per = L / 2;
	wires.resize(2 * (size_t)nlayers * per);
	if (gates) gates->resize(16 * (size_t)nlayers * per);
	for (int l = 0; l < nlayers; l++) {
		if (!perms[l]) return false;
		for (int p = 0; p < per; p++) {
			const int k = l * per + p;
			wires[2 * k] = perms[l][2 * p];
			wires[2 * k + 1] = perms[l][2 * p + 1];
			if (gates) memcpy(&(*gates)[16 * (size_t)k], vlist[l].data, 16 * sizeof(double2));
		}
	}
	return valid_circuit(L, nlayers * per, wires.data());
}

}  // namespace

// ------------------------------------------------------------------------- statevector

extern "C" int allocate_statevector(int nqubits, struct statevector* psi)
{
	psi->nqubits = nqubits;
	psi->data = nullptr;
	if (nqubits < 0 || nqubits > 40) {
		fprintf(stderr, "rqcopt_gpu: allocate_statevector: invalid number of qubits %d\n", nqubits);
		return -1;
	}
	if (!runtime()) return -1;
	void* p = nullptr;
	const size_t bytes = ((size_t)1 << nqubits) * sizeof(numeric);
	if (cudaMallocManaged(&p, bytes, cudaMemAttachGlobal) != cudaSuccess) {
		cudaGetLastError();
		fprintf(stderr, "allocating statevector memory (%zu bytes) failed\n", bytes);
		return -1;
	}
	psi->data = static_cast<numeric*>(p);
	return 0;
}

extern "C" void free_statevector(struct statevector* psi)
{
	if (psi->data) {
		if (is_device_pointer(psi->data)) cudaFree(psi->data);
		else fprintf(stderr, "rqcopt_gpu: free_statevector: pointer was not allocated by allocate_statevector\n");
		psi->data = nullptr;
	}
	psi->nqubits = 0;
}

extern "C" void add_statevectors(const struct statevector* psi1, const struct statevector* psi2, struct statevector* psi_sum)
{
	if (psi1->nqubits != psi2->nqubits || psi1->nqubits != psi_sum->nqubits) {
		fail_arg("add_statevectors", "statevectors differ in qubit count");
		return;
	}
	Runtime* rt = runtime();
	if (!rt) { set_last_error(E_CUDA); return; }
	const int L = psi1->nqubits;
	DeviceSpan a, b, c;
	int ret = span_in(*rt, psi1->data, sv_bytes(L), 0, a);
	if (!ret) ret = span_in(*rt, psi2->data, sv_bytes(L), 1, b);
	if (!ret) ret = span_out(*rt, psi_sum->data, sv_bytes(L), 2, c);
	if (!ret) ret = add_device(*rt, (const double2*)a.dev, (const double2*)b.dev, (double2*)c.dev, 1L << L);
	if (!ret) ret = span_finish(*rt, c);
	if (!ret) ret = sync(*rt);
	if (ret) set_last_error(ret);
}

// psi_trans[j] = psi[k], k the index j with qubit i moved to qubit perm[i]
// (src/statevector.c:72-98).  A wire permutation, not on the optimisation path: it
// runs on the host, with device-memory statevectors copied through host memory.
extern "C" void transpose_statevector(const struct statevector* psi, const int* perm, struct statevector* psi_trans)
{
	if (!psi || !psi_trans || !perm || !psi->data || !psi_trans->data || psi->nqubits != psi_trans->nqubits ||
	    psi->nqubits < 0 || psi->nqubits > 40) {
		fail_arg("transpose_statevector", "invalid statevectors");
		return;
	}
	const int L = psi->nqubits;
	std::vector<int64_t> strides(L > 0 ? L : 1);
	std::vector<char> seen(L > 0 ? L : 1, 0);
	for (int i = 0; i < L; i++) {
		if (perm[i] < 0 || perm[i] >= L || seen[perm[i]]) {
			fail_arg("transpose_statevector", "'perm' is not a permutation of the qubits");
			return;
		}
		seen[perm[i]] = 1;
		strides[L - 1 - i] = (int64_t)1 << (L - 1 - perm[i]);
	}
	// device statevectors are permuted in host copies (host and managed memory in place)
	auto on_device = [](const void* p) {
		cudaPointerAttributes a;
		if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
			cudaGetLastError();
			return false;
		}
		return a.type == cudaMemoryTypeDevice;
	};
	const int64_t n = (int64_t)1 << L;
	const bool din = on_device(psi->data), dout = on_device(psi_trans->data);
	std::vector<double2> hin(din ? n : 0), hout(dout ? n : 0);
	if (din && RQC_CUDA(cudaMemcpy(hin.data(), psi->data, n * sizeof(double2), cudaMemcpyDeviceToHost))) {
		set_last_error(E_CUDA);
		return;
	}
	const double2* src = din ? hin.data() : reinterpret_cast<const double2*>(psi->data);
	double2* dst = dout ? hout.data() : reinterpret_cast<double2*>(psi_trans->data);
	for (int64_t j = 0; j < n; j++) {
		int64_t k = 0;
		for (int i = 0; i < L; i++) k += ((j >> i) & 1) * strides[i];
		dst[j] = src[k];
	}
	if (dout && RQC_CUDA(cudaMemcpy(psi_trans->data, hout.data(), n * sizeof(double2), cudaMemcpyHostToDevice)))
		set_last_error(E_CUDA);
}

// ------------------------------------------------------------------------- gates

extern "C" void apply_gate(const struct mat4x4* gate, const int i, const int j, const struct statevector* psi,
                           struct statevector* psi_out)
{
	const int L = psi->nqubits;
	if (psi_out->nqubits != L || !valid_wires(L, i, j)) {
		fail_arg("apply_gate", "invalid wires or mismatching statevectors");
		return;
	}
	Runtime* rt = runtime();
	if (!rt) { set_last_error(E_CUDA); return; }
	DeviceSpan in, out;
	int ret = span_in(*rt, psi->data, sv_bytes(L), 0, in);
	if (!ret) ret = span_out(*rt, psi_out->data, sv_bytes(L), 1, out);
	if (!ret) ret = gate_apply_device(*rt, L, d2(gate->data), i, j, (const double2*)in.dev, (double2*)out.dev, 1);
	if (!ret) ret = span_finish(*rt, out);
	if (!ret) ret = sync(*rt);
	if (ret) set_last_error(ret);
}

extern "C" void apply_gate_backward(const struct mat4x4* gate, const int i, const int j, const struct statevector* psi,
                                    const struct statevector* dpsi_out, struct statevector* dpsi, struct mat4x4* dgate)
{
	const int L = psi->nqubits;
	if (dpsi_out->nqubits != L || dpsi->nqubits != L || !valid_wires(L, i, j)) {
		fail_arg("apply_gate_backward", "invalid wires or mismatching statevectors");
		return;
	}
	Runtime* rt = runtime();
	if (!rt) { set_last_error(E_CUDA); return; }
	DeviceSpan x, d, dx;
	int ret = span_in(*rt, psi->data, sv_bytes(L), 0, x);
	if (!ret) ret = span_in(*rt, dpsi_out->data, sv_bytes(L), 1, d);
	if (!ret) ret = span_out(*rt, dpsi->data, sv_bytes(L), 2, dx);
	if (!ret) ret = ensure_device(rt->small, 16 * sizeof(double2));
	double2* dg = (double2*)rt->small.ptr;
	if (!ret) ret = gate_backward_device(*rt, L, d2(gate->data), i, j, (const double2*)x.dev, (const double2*)d.dev,
	                                     (double2*)dx.dev, dg);
	if (!ret) ret = span_finish(*rt, dx);
	if (!ret) ret = RQC_CUDA(cudaMemcpyAsync(dgate->data, dg, 16 * sizeof(double2), cudaMemcpyDeviceToHost, rt->stream));
	if (!ret) ret = sync(*rt);
	if (ret) set_last_error(ret);
}

// ------------------------------------------------------------------------- quantum circuits

extern "C" int apply_quantum_circuit(const struct mat4x4 gates[], const int ngates, const int wires[],
                                     const struct statevector* psi, struct statevector* psi_out)
{
	const int L = psi->nqubits;
	if (psi_out->nqubits != L || !valid_circuit(L, ngates, wires)) {
		fprintf(stderr, "rqcopt_gpu: apply_quantum_circuit: invalid arguments\n");
		return E_ARG;
	}
	Runtime* rt = runtime();
	if (!rt) return E_CUDA;
	DeviceSpan in, out;
	int ret = span_in(*rt, psi->data, sv_bytes(L), 0, in);
	if (!ret) ret = span_out(*rt, psi_out->data, sv_bytes(L), 1, out);
	if (!ret) ret = apply_circuit_device(*rt, L, ngates, d2(gates[0].data), wires, (const double2*)in.dev, (double2*)out.dev, 1);
	if (!ret) ret = span_finish(*rt, out);
	if (!ret) ret = sync(*rt);
	return ret;
}

extern "C" int allocate_quantum_circuit_cache(const int nqubits, const int ngates, struct quantum_circuit_cache* cache)
{
	cache->nqubits = nqubits;
	cache->ngates = ngates;
	cache->psi_list = nullptr;
	if (ngates < 1) return -1;
	cache->psi_list = static_cast<struct statevector*>(calloc(ngates, sizeof(struct statevector)));
	if (!cache->psi_list) {
		fprintf(stderr, "allocating memory for statevector array failed\n");
		return -1;
	}
	for (int k = 0; k < ngates; k++) {
		const int ret = allocate_statevector(nqubits, &cache->psi_list[k]);
		if (ret < 0) return ret;
	}
	return 0;
}

extern "C" void free_quantum_circuit_cache(struct quantum_circuit_cache* cache)
{
	if (cache->psi_list) {
		for (int k = 0; k < cache->ngates; k++) free_statevector(&cache->psi_list[k]);
		free(cache->psi_list);
	}
	cache->psi_list = nullptr;
	cache->nqubits = 0;
	cache->ngates = 0;
}

extern "C" int quantum_circuit_forward(const struct mat4x4 gates[], const int ngates, const int wires[],
                                       const struct statevector* psi, struct quantum_circuit_cache* cache,
                                       struct statevector* psi_out)
{
	const int L = psi->nqubits;
	if (psi_out->nqubits != L || cache->ngates != ngates || cache->nqubits != L || !valid_circuit(L, ngates, wires)) {
		fprintf(stderr, "rqcopt_gpu: quantum_circuit_forward: invalid arguments\n");
		return E_ARG;
	}
	Runtime* rt = runtime();
	if (!rt) return E_CUDA;
	const size_t bytes = sv_bytes(L);
	// cache[0] = psi; cache[k + 1] = G_k cache[k]; psi_out = G_{n-1} cache[n-1]
	DeviceSpan src, dst;
	int ret = span_in(*rt, psi->data, bytes, 0, src);
	if (!ret) ret = span_out(*rt, cache->psi_list[0].data, bytes, 1, dst);
	if (!ret) ret = RQC_CUDA(cudaMemcpyAsync(dst.dev, src.dev, bytes, cudaMemcpyDeviceToDevice, rt->stream));
	if (!ret) ret = span_finish(*rt, dst);
	for (int k = 0; k < ngates && !ret; k++) {
		struct statevector* next = k + 1 < ngates ? &cache->psi_list[k + 1] : psi_out;
		DeviceSpan a, b;
		ret = span_in(*rt, cache->psi_list[k].data, bytes, 0, a);
		if (!ret) ret = span_out(*rt, next->data, bytes, 1, b);
		if (!ret) ret = gate_apply_device(*rt, L, d2(gates[k].data), wires[2 * k], wires[2 * k + 1], (const double2*)a.dev,
		                                  (double2*)b.dev, 1);
		if (!ret) ret = span_finish(*rt, b);
		if (!ret && (a.host || b.host)) ret = sync(*rt);   // staging slots are reused by the next gate
	}
	if (!ret) ret = sync(*rt);
	return ret;
}

extern "C" int quantum_circuit_backward(const struct mat4x4 gates[], const int ngates, const int wires[],
                                        const struct quantum_circuit_cache* cache, const struct statevector* dpsi_out,
                                        struct statevector* dpsi, struct mat4x4 dgates[])
{
	const int L = dpsi->nqubits;
	if (dpsi_out->nqubits != L || cache->nqubits != L || cache->ngates != ngates || !valid_circuit(L, ngates, wires)) {
		fprintf(stderr, "rqcopt_gpu: quantum_circuit_backward: invalid arguments\n");
		return E_ARG;
	}
	Runtime* rt = runtime();
	if (!rt) return E_CUDA;
	const size_t bytes = sv_bytes(L);
	int ret = ensure_device(rt->stage[3], 2 * bytes);
	if (!ret) ret = ensure_device(rt->small, 16 * (size_t)ngates * sizeof(double2));
	if (ret) return ret;
	double2* tmp[2] = { (double2*)rt->stage[3].ptr, (double2*)rt->stage[3].ptr + ((size_t)1 << L) };
	double2* dg = (double2*)rt->small.ptr;
	DeviceSpan d;
	ret = span_in(*rt, dpsi_out->data, bytes, 1, d);
	const double2* cur = (const double2*)d.dev;
	for (int k = ngates - 1; k >= 0 && !ret; k--) {
		DeviceSpan x;
		ret = span_in(*rt, cache->psi_list[k].data, bytes, 0, x);
		double2* nxt = tmp[k & 1];
		if (!ret) ret = gate_backward_device(*rt, L, d2(gates[k].data), wires[2 * k], wires[2 * k + 1],
		                                     (const double2*)x.dev, cur, nxt, dg + 16 * (size_t)k);
		if (!ret && x.host) ret = sync(*rt);
		cur = nxt;
	}
	DeviceSpan out;
	if (!ret) ret = span_out(*rt, dpsi->data, bytes, 2, out);
	if (!ret) ret = RQC_CUDA(cudaMemcpyAsync(out.dev, cur, bytes, cudaMemcpyDeviceToDevice, rt->stream));
	if (!ret) ret = span_finish(*rt, out);
	if (!ret) ret = RQC_CUDA(cudaMemcpyAsync(dgates[0].data, dg, 16 * (size_t)ngates * sizeof(double2),
	                                         cudaMemcpyDeviceToHost, rt->stream));
	if (!ret) ret = sync(*rt);
	return ret;
}

extern "C" int quantum_circuit_gates_hessian_vector_product(const struct mat4x4 gates[], const struct mat4x4 gatedirs[],
                                                            const int ngates, const int wires[],
                                                            const struct statevector* psi, const struct statevector* phi,
                                                            struct statevector* psi_out, struct mat4x4 dgates[],
                                                            struct mat4x4 hess_gatedirs[])
{
	const int L = psi->nqubits;
	if (phi->nqubits != L || psi_out->nqubits != L || !valid_circuit(L, ngates, wires)) {
		fprintf(stderr, "rqcopt_gpu: quantum_circuit_gates_hessian_vector_product: invalid arguments\n");
		return E_ARG;
	}
	Runtime* rt = runtime();
	if (!rt) return E_CUDA;
	const size_t bytes = sv_bytes(L);
	int ret = ensure_device(rt->small, 32 * (size_t)ngates * sizeof(double2));
	if (ret) return ret;
	double2* dg = (double2*)rt->small.ptr;
	double2* hg = dg + 16 * (size_t)ngates;
	DeviceSpan a, b, c;
	ret = span_in(*rt, psi->data, bytes, 0, a);
	if (!ret) ret = span_in(*rt, phi->data, bytes, 1, b);
	if (!ret) ret = span_out(*rt, psi_out->data, bytes, 2, c);
	if (!ret) ret = column_passes_device(*rt, L, ngates, d2(gates[0].data), d2(gatedirs[0].data), wires,
	                                     (const double2*)a.dev, (const double2*)b.dev, (double2*)c.dev, dg, hg);
	if (!ret) ret = span_finish(*rt, c);
	if (!ret) ret = RQC_CUDA(cudaMemcpyAsync(dgates[0].data, dg, 16 * (size_t)ngates * sizeof(double2), cudaMemcpyDeviceToHost, rt->stream));
	if (!ret) ret = RQC_CUDA(cudaMemcpyAsync(hess_gatedirs[0].data, hg, 16 * (size_t)ngates * sizeof(double2), cudaMemcpyDeviceToHost, rt->stream));
	if (!ret) ret = sync(*rt);
	return ret < 0 ? ret : 0;
}

// ------------------------------------------------------------------------- brickwall circuits

extern "C" int apply_brickwall_unitary(const struct mat4x4 vlist[], const int nlayers, const int* perms[],
                                       const struct statevector* psi, struct statevector* psi_out)
{
	std::vector<double2> gates;
	std::vector<int> wires;
	if (psi_out->nqubits != psi->nqubits || !expand_brickwall(psi->nqubits, nlayers, vlist, perms, &gates, wires)) {
		fprintf(stderr, "rqcopt_gpu: apply_brickwall_unitary: invalid arguments\n");
		return E_ARG;
	}
	return apply_quantum_circuit(reinterpret_cast<const struct mat4x4*>(gates.data()), (int)(wires.size() / 2),
	                             wires.data(), psi, psi_out);
}

extern "C" int brickwall_unitary_forward(const struct mat4x4 vlist[], int nlayers, const int* perms[],
                                         const struct statevector* psi, struct quantum_circuit_cache* cache,
                                         struct statevector* psi_out)
{
	std::vector<double2> gates;
	std::vector<int> wires;
	if (!expand_brickwall(psi->nqubits, nlayers, vlist, perms, &gates, wires)) {
		fprintf(stderr, "rqcopt_gpu: brickwall_unitary_forward: invalid arguments\n");
		return E_ARG;
	}
	return quantum_circuit_forward(reinterpret_cast<const struct mat4x4*>(gates.data()), (int)(wires.size() / 2),
	                               wires.data(), psi, cache, psi_out);
}

extern "C" int brickwall_unitary_backward(const struct mat4x4 vlist[], int nlayers, const int* perms[],
                                          const struct quantum_circuit_cache* cache, const struct statevector* dpsi_out,
                                          struct statevector* dpsi, struct mat4x4 dvlist[])
{
	std::vector<double2> gates;
	std::vector<int> wires;
	if (!expand_brickwall(dpsi->nqubits, nlayers, vlist, perms, &gates, wires)) {
		fprintf(stderr, "rqcopt_gpu: brickwall_unitary_backward: invalid arguments\n");
		return E_ARG;
	}
	const int G = (int)(wires.size() / 2), per = dpsi->nqubits / 2;
	std::vector<struct mat4x4> dg(G);
	const int ret = quantum_circuit_backward(reinterpret_cast<const struct mat4x4*>(gates.data()), G, wires.data(), cache,
	                                         dpsi_out, dpsi, dg.data());
	if (ret) return ret;
	// per-layer gradient: sum over the layer's gate copies (src/brickwall_circuit.c:102-119)
	for (int l = 0; l < nlayers; l++) {
		for (int e = 0; e < 16; e++) dvlist[l].data[e] = 0;
		for (int p = per - 1; p >= 0; p--)
			for (int e = 0; e < 16; e++) dvlist[l].data[e] += dg[l * per + p].data[e];
	}
	return 0;
}
