// Gate application to single statevectors with several gates per HBM round trip.
//
// Consecutive gates are grouped into passes of up to four gates (at most eight
// qubits).  A pass streams the state once: each block loads a tile of 2^NB
// amplitudes spanning the pass's qubits plus the lowest amplitude bits (so that
// every row of the tile is a contiguous run of at least 64 bytes), applies the
// pass's gates in shared memory, and writes the tile back.  Used by
// apply_quantum_circuit / apply_brickwall_unitary for large states; the
// arithmetic per gate is the one of src/gate.c:10-76.
#include <stdio.h>
#include <string.h>
#include <algorithm>
#include <vector>

#include "engine.h"
#include "rqc_common.cuh"
#include "rqcopt_gpu.h"

namespace rqc {

namespace {

constexpr int SV_TPB = 256;
constexpr int SV_MAXK = 4;
constexpr int SV_MAXNB = 10;   // 1024 amplitudes per tile

struct SvPass
{
	int K, NB, L;
	int tbit[SV_MAXNB];            // state bits of the tile bits (ascending)
	int gi[SV_MAXK], gj[SV_MAXK];  // tile-local bits of each gate's wires
	uint32_t rest_mask;            // state bits outside the tile
	int64_t ntiles;
	int first;                     // first gate of the pass
};

template <typename T> struct SvGates { Gate4<T> g[SV_MAXK]; };

__device__ __forceinline__ int64_t sv_deposit(int64_t v, uint32_t mask)
{
	int64_t r = 0;
	for (int b = 0; mask; b++) {
		const uint32_t low = mask & (0u - mask);
		if ((v >> b) & 1) r |= (int64_t)low;
		mask &= mask - 1;
	}
	return r;
}

template <typename T>
__global__ void __launch_bounds__(SV_TPB) k_sv_pass(const cplx<T>* __restrict__ in, cplx<T>* __restrict__ out, SvPass ps,
                                                    SvGates<T> gates)
{
	using V = cplx<T>;
	__shared__ V S[1 << SV_MAXNB];
	__shared__ int64_t off[1 << SV_MAXNB];
	const int A = 1 << ps.NB;
	for (int r = threadIdx.x; r < A; r += blockDim.x) {
		int64_t o = 0;
#pragma unroll
		for (int b = 0; b < SV_MAXNB; b++)
			if (b < ps.NB && ((r >> b) & 1)) o |= (int64_t)1 << ps.tbit[b];
		off[r] = o;
	}
	__syncthreads();
	for (int64_t tile = blockIdx.x; tile < ps.ntiles; tile += gridDim.x) {
		const int64_t base = sv_deposit(tile, ps.rest_mask);
		for (int r = threadIdx.x; r < A; r += blockDim.x) S[r] = in[base + off[r]];
		__syncthreads();
#pragma unroll
		for (int k = 0; k < SV_MAXK; k++) {
			if (k >= ps.K) break;
			const int bi = ps.gi[k], bj = ps.gj[k];
			const int lo = bi < bj ? bi : bj, hi = bi < bj ? bj : bi;
			for (int g = threadIdx.x; g < A / 4; g += blockDim.x) {
				int b = g;
				b = ((b >> lo) << (lo + 1)) | (b & ((1 << lo) - 1));
				b = ((b >> hi) << (hi + 1)) | (b & ((1 << hi) - 1));
				const int r0 = b, r1 = b | (1 << bj), r2 = b | (1 << bi), r3 = b | (1 << bi) | (1 << bj);
				V x[4] = { S[r0], S[r1], S[r2], S[r3] }, y[4];
				gate_apply(gates.g[k], x, y);
				S[r0] = y[0];
				S[r1] = y[1];
				S[r2] = y[2];
				S[r3] = y[3];
			}
			__syncthreads();
		}
		for (int r = threadIdx.x; r < A; r += blockDim.x) out[base + off[r]] = S[r];
		__syncthreads();
	}
}

std::vector<SvPass> sv_schedule(int L, int G, const int* wires, int maxk)
{
	std::vector<SvPass> out;
	// the two lowest amplitude bits ride along so that every tile row is >= 64 bytes long
	const uint32_t low = L >= 2 ? 3u : 1u;
	for (int i = 0; i < G;) {
		const int K = std::min(maxk, G - i);
		uint32_t bits = low;
		for (int k = 0; k < K; k++) {
			bits |= 1u << (L - 1 - wires[2 * (i + k)]);
			bits |= 1u << (L - 1 - wires[2 * (i + k) + 1]);
		}
		SvPass p;
		memset(&p, 0, sizeof(p));
		p.K = K;
		p.L = L;
		p.first = i;
		int local[32];
		int n = 0;
		for (int b = 0; b < L; b++)
			if ((bits >> b) & 1) { local[b] = n; p.tbit[n++] = b; }
		p.NB = n;
		for (int k = 0; k < K; k++) {
			p.gi[k] = local[L - 1 - wires[2 * (i + k)]];
			p.gj[k] = local[L - 1 - wires[2 * (i + k) + 1]];
		}
		const uint32_t all = L >= 32 ? 0xffffffffu : ((1u << L) - 1);
		p.rest_mask = all & ~bits;
		p.ntiles = (int64_t)1 << (L - n);
		out.push_back(p);
		i += K;
	}
	return out;
}

}  // namespace

template <typename T>
int apply_circuit_fused_t(Runtime& rt, int L, int ngates, const double2* gates, const int* wires, const cplx<T>* d_in,
                          cplx<T>* d_out, int maxk)
{
	maxk = std::max(1, std::min(SV_MAXK, maxk));
	std::vector<SvPass> passes = sv_schedule(L, ngates, wires, maxk);
	const int P = (int)passes.size();
	const size_t bytes = ((size_t)1 << L) * sizeof(cplx<T>);
	int ret;
	if (P > 1 && (ret = ensure_device(rt.stage[3], bytes))) return ret;
	cplx<T>* tmp = reinterpret_cast<cplx<T>*>(rt.stage[3].ptr);
	const cplx<T>* src = d_in;
	for (int p = 0; p < P; p++) {
		cplx<T>* dst = ((P - 1 - p) % 2 == 0) ? d_out : tmp;
		SvGates<T> sg;
		for (int k = 0; k < passes[p].K; k++)
			for (int e = 0; e < 16; e++) {
				const double2 g = gates[16 * (passes[p].first + k) + e];
				sg.g[k].m[e].x = (T)g.x;
				sg.g[k].m[e].y = (T)g.y;
			}
		const int grid = (int)std::min<int64_t>(passes[p].ntiles, (int64_t)rt.num_sms * 8);
		cudaEvent_t ev;
		launch_begin(rt, KC_FUSED, &ev);
		k_sv_pass<T><<<grid, SV_TPB, 0, rt.stream>>>(src, dst, passes[p], sg);
		launch_end(rt, KC_FUSED, ev);
		if ((ret = RQC_CUDA(cudaGetLastError()))) return ret;
		src = dst;
	}
	return OK;
}

// out = C in for one statevector (complex128), maxk gates per pass; in and out may not alias.
int apply_circuit_fused_device(Runtime& rt, int L, int ngates, const double2* gates, const int* wires,
                               const double2* d_in, double2* d_out, int maxk)
{
	return apply_circuit_fused_t<double>(rt, L, ngates, gates, wires, d_in, d_out, maxk);
}

int apply_circuit_fused_device_c64(Runtime& rt, int L, int ngates, const double2* gates, const int* wires,
                                   const float2* d_in, float2* d_out, int maxk)
{
	return apply_circuit_fused_t<float>(rt, L, ngates, gates, wires, d_in, d_out, maxk);
}

}  // namespace rqc

using namespace rqc;

// The complex64 form of apply_quantum_circuit (src/quantum_circuit.c:13-35) on
// device-resident complex64 states; gates stay complex128 on the host and are
// rounded to complex64 for the passes.
extern "C" int rqcopt_apply_quantum_circuit_c64(const struct mat4x4 gates[], int ngates, const int wires[],
                                                const void* psi, void* psi_out, int nqubits)
{
	if (nqubits < 2 || nqubits > 34 || ngates < 1 || !gates || !wires || !psi || !psi_out || psi == psi_out) return E_ARG;
	for (int k = 0; k < ngates; k++)
		if (wires[2 * k] < 0 || wires[2 * k] >= nqubits || wires[2 * k + 1] < 0 || wires[2 * k + 1] >= nqubits ||
		    wires[2 * k] == wires[2 * k + 1])
			return E_ARG;
	Runtime* rt = runtime();
	if (!rt) return E_CUDA;
	if (!is_device_pointer(psi) || !is_device_pointer(psi_out)) return E_ARG;
	int ret = apply_circuit_device_c64(*rt, nqubits, ngates, reinterpret_cast<const double2*>(gates), wires,
	                                   static_cast<const float2*>(psi), static_cast<float2*>(psi_out));
	if (!ret) ret = sync(*rt);
	return ret;
}
