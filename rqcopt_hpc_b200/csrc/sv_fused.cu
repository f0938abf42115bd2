// Gate application to single statevectors with several gates per HBM round trip.
//
// Consecutive gates are grouped into passes of up to four gates (at most eight
// qubits).  A pass streams the state once: each block stages a tile spanning the
// pass's qubits plus the lowest amplitude bits in shared memory, applies the pass's
// gates there, and writes the tile back.  Used by apply_quantum_circuit /
// apply_brickwall_unitary for large states; the arithmetic per gate is the one of
// src/gate.c:10-76.
//
// Tiles of 64 KiB (4096 complex128 or 8192 complex64 amplitudes) take as many of the
// lowest state bits as fit beside the pass qubits, so a tile is a set of contiguous
// runs of 2^m amplitudes (m >= 4: runs of 256 B or more), one per combination of the
// pass qubits above the run.  The runs move between HBM and shared memory as TMA bulk
// copies (cp.async.bulk, completion on an mbarrier for loads, bulk groups for stores),
// issued by one warp; three blocks per SM overlap their load, gate and store phases.
// States whose address is not 16-byte aligned take a tile kernel with plain loads.
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

// ------------------------------------------------------------------ TMA bulk tiles

constexpr int SVT_TPB = 256;
constexpr int SVT_TILE_BYTES = 64 * 1024;
constexpr int SVT_MAXRUNS = 256;      // runs per tile: 2^(pass qubits above the run) <= 2^8

template <typename T> struct SvtBits;
template <> struct SvtBits<double> { static constexpr int v = 12; };   // 4096 x 16 B
template <> struct SvtBits<float>  { static constexpr int v = 13; };   // 8192 x 8 B

struct SvTile
{
	int K, NB, m, L;               // tile bits; tile bits 0..m-1 are the state bits 0..m-1 (the run)
	int hbit[8];                   // state bits of tile bits m..NB-1 (ascending)
	int gi[SV_MAXK], gj[SV_MAXK];  // tile-local bits of each gate's wires
	uint32_t rest_mask;            // state bits outside the tile
	int64_t ntiles;
	int first;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t global_ns()
{
	uint64_t t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}

// Wait for phase `parity` of the mbarrier, for at most ~2 s; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
	const uint32_t a = smem_u32(bar);
	const uint64_t t0 = global_ns();
	for (int it = 0;; it++) {
		uint32_t done;
		asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
		             "selp.u32 %0, 1, 0, p;\n\t}"
		             : "=r"(done) : "r"(a), "r"(parity) : "memory");
		if (done) return true;
		if ((it & 63) == 63 && global_ns() - t0 > 2000000000ull) return false;
		if (it > 16) __nanosleep(32);
	}
}

template <typename T>
__global__ void __launch_bounds__(SVT_TPB, 3) k_sv_tile(const cplx<T>* __restrict__ in, cplx<T>* __restrict__ out, SvTile ps,
                                                     SvGates<T> gates, int* __restrict__ err)
{
	using V = cplx<T>;
	extern __shared__ __align__(128) unsigned char sm_raw[];
	V* S = reinterpret_cast<V*>(sm_raw);
	int64_t* roff = reinterpret_cast<int64_t*>(sm_raw + SVT_TILE_BYTES);
	uint64_t* bar = reinterpret_cast<uint64_t*>(roff + SVT_MAXRUNS);
	Gate4<T>* sgate = reinterpret_cast<Gate4<T>*>(bar + 2);
	const int A = 1 << ps.NB, nruns = 1 << (ps.NB - ps.m);
	const uint32_t run_bytes = (uint32_t)(sizeof(V) << ps.m);
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	for (int r = threadIdx.x; r < nruns; r += blockDim.x) {
		int64_t o = 0;
		for (int b = 0; b < ps.NB - ps.m; b++)
			if ((r >> b) & 1) o |= (int64_t)1 << ps.hbit[b];
		roff[r] = o;
	}
	for (int e = threadIdx.x; e < SV_MAXK * 16; e += blockDim.x) sgate[e / 16].m[e % 16] = gates.g[e / 16].m[e % 16];
	if (threadIdx.x == 0) {
		asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	__syncthreads();
	uint32_t parity = 0;
	bool ok = true;
	for (int64_t tile = blockIdx.x; tile < ps.ntiles && ok; tile += gridDim.x) {
		const int64_t base = sv_deposit(tile, ps.rest_mask);
		if (warp == 0) {
			asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
			if (lane == 0)
				asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
				             "r"((uint32_t)(A * sizeof(V))) : "memory");
			__syncwarp();
			for (int r = lane; r < nruns; r += 32)
				asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
				             ::"r"(smem_u32(S + ((size_t)r << ps.m))), "l"(in + base + roff[r]), "r"(run_bytes),
				             "r"(smem_u32(bar)) : "memory");
		}
		// the block decides together, so that no thread leaves while others wait at a barrier
		if (!__syncthreads_and(mbar_wait(bar, parity) ? 1 : 0)) {
			ok = false;
			if (threadIdx.x == 0) atomicExch(err, 1);
			break;
		}
		parity ^= 1;
#pragma unroll 1
		for (int k = 0; k < ps.K; k++) {
			const int bi = ps.gi[k], bj = ps.gj[k];
			const int lo = bi < bj ? bi : bj, hi = bi < bj ? bj : bi;
			const Gate4<T>& gk = sgate[k];
			for (int g = threadIdx.x; g < A / 4; g += blockDim.x) {
				int b = g;
				b = ((b >> lo) << (lo + 1)) | (b & ((1 << lo) - 1));
				b = ((b >> hi) << (hi + 1)) | (b & ((1 << hi) - 1));
				const int r0 = b, r1 = b | (1 << bj), r2 = b | (1 << bi), r3 = b | (1 << bi) | (1 << bj);
				V x[4] = { S[r0], S[r1], S[r2], S[r3] }, y[4];
				gate_apply(gk, x, y);
				S[r0] = y[0];
				S[r1] = y[1];
				S[r2] = y[2];
				S[r3] = y[3];
			}
			__syncthreads();
		}
		// the tile's stores (generic proxy) become visible to the bulk copies (async proxy)
		asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
		__syncthreads();
		if (warp == 0) {
			for (int r = lane; r < nruns; r += 32)
				asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;"
				             ::"l"(out + base + roff[r]), "r"(smem_u32(S + ((size_t)r << ps.m))), "r"(run_bytes)
				             : "memory");
			asm volatile("cp.async.bulk.commit_group;" ::: "memory");
			asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");   // the tile may be overwritten
		}
		__syncthreads();
	}
	if (warp == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
	if (!ok && warp == 0) {
		// the loads of the tile that timed out may still land: wait (bounded) before the block exits
		mbar_wait(bar, parity);
	}
}

// Tile bits: the pass qubits plus the lowest state bits 0..m-1, m as large as the tile allows.
template <typename T>
std::vector<SvTile> sv_tile_schedule(int L, int G, const int* wires, int maxk)
{
	std::vector<SvTile> out;
	const int nbmax = std::min(SvtBits<T>::v, L);
	for (int i = 0; i < G;) {
		const int K = std::min(maxk, G - i);
		uint32_t pass = 0;
		for (int k = 0; k < K; k++) {
			pass |= 1u << (L - 1 - wires[2 * (i + k)]);
			pass |= 1u << (L - 1 - wires[2 * (i + k) + 1]);
		}
		int m = 0;
		while (m < L && __builtin_popcount(pass | ((2u << m) - 1)) <= nbmax) m++;
		const uint32_t bits = pass | (m > 0 ? ((1u << m) - 1) : 0u);
		SvTile p;
		memset(&p, 0, sizeof(p));
		p.K = K;
		p.L = L;
		p.first = i;
		p.m = m;
		int local[32];
		int n = 0, nh = 0;
		for (int b = 0; b < L; b++)
			if ((bits >> b) & 1) {
				local[b] = n++;
				if (b >= m) p.hbit[nh++] = b;
			}
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
	const size_t bytes = ((size_t)1 << L) * sizeof(cplx<T>);
	int ret;
	int P;
	if (ngates > maxk && (ret = ensure_device(rt.stage[3], bytes))) return ret;
	cplx<T>* tmp = reinterpret_cast<cplx<T>*>(rt.stage[3].ptr);
	auto gates_of = [&](int first, int K) {
		SvGates<T> sg;
		memset(&sg, 0, sizeof(sg));
		for (int k = 0; k < K; k++)
			for (int e = 0; e < 16; e++) {
				const double2 g = gates[16 * (first + k) + e];
				sg.g[k].m[e].x = (T)g.x;
				sg.g[k].m[e].y = (T)g.y;
			}
		return sg;
	};
	// TMA bulk tiles: 16-byte aligned states of at least 2^12 amplitudes
	const bool bulk = L >= 12 && ((uintptr_t)d_in % 16) == 0 && ((uintptr_t)d_out % 16) == 0;
	if (bulk) {
		std::vector<SvTile> passes = sv_tile_schedule<T>(L, ngates, wires, maxk);
		P = (int)passes.size();
		static int per_sm = 0;
		const size_t smem = SVT_TILE_BYTES + SVT_MAXRUNS * sizeof(int64_t) + 16 + SV_MAXK * sizeof(Gate4<T>);
		if (!per_sm) {
			if ((ret = RQC_CUDA(cudaFuncSetAttribute(k_sv_tile<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem))))
				return ret;
			if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sv_tile<T>, SVT_TPB, smem) != cudaSuccess ||
			    per_sm < 1) {
				cudaGetLastError();
				per_sm = 1;
			}
		}
		if ((ret = ensure_device(rt.status, sizeof(int)))) return ret;
		int* d_err = static_cast<int*>(rt.status.ptr);
		if ((ret = RQC_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), rt.stream)))) return ret;
		const cplx<T>* src = d_in;
		for (int p = 0; p < P; p++) {
			cplx<T>* dst = ((P - 1 - p) % 2 == 0) ? d_out : tmp;
			const int grid = (int)std::min<int64_t>(passes[p].ntiles, (int64_t)rt.num_sms * per_sm);
			cudaEvent_t ev;
			launch_begin(rt, KC_FUSED, &ev);
			k_sv_tile<T><<<grid, SVT_TPB, smem, rt.stream>>>(src, dst, passes[p], gates_of(passes[p].first, passes[p].K),
			                                                 d_err);
			launch_end(rt, KC_FUSED, ev);
			if ((ret = RQC_CUDA(cudaGetLastError()))) return ret;
			src = dst;
		}
		int herr = 0;
		if ((ret = RQC_CUDA(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, rt.stream)))) return ret;
		if ((ret = RQC_CUDA(cudaStreamSynchronize(rt.stream)))) return ret;
		if (herr) {
			fprintf(stderr, "rqcopt_gpu: a tile copy of the fused gate pass did not complete\n");
			return E_CUDA;
		}
		return OK;
	}
	std::vector<SvPass> passes = sv_schedule(L, ngates, wires, maxk);
	P = (int)passes.size();
	const cplx<T>* src = d_in;
	for (int p = 0; p < P; p++) {
		cplx<T>* dst = ((P - 1 - p) % 2 == 0) ? d_out : tmp;
		const int grid = (int)std::min<int64_t>(passes[p].ntiles, (int64_t)rt.num_sms * 8);
		cudaEvent_t ev;
		launch_begin(rt, KC_FUSED, &ev);
		k_sv_pass<T><<<grid, SV_TPB, 0, rt.stream>>>(src, dst, passes[p], gates_of(passes[p].first, passes[p].K));
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
