// Allocation-free variant of the gate backward pass (apply_gate_backward):
// dpsi = G^T dpsi_out and dG = sum dpsi_out (x) psi.
//
// Some callers cannot allocate device memory at the point where they need the
// pass: code that runs while its process has handed all device memory to its
// own pool, code on a latency-critical thread that must not take the
// device-wide synchronisation a cudaMalloc/cudaFree can imply, or host
// callbacks such as a target's linear_func, which another library's column
// loop calls on an ordinary host thread while that library holds the device
// memory.  This entry point therefore uses no allocator at all: the only
// memory it needs beyond the
// caller's inputs and outputs -- the per-tile partial sums of dG and the reduced
// dG -- lives in the file-scope array below, which every GPU that loads the
// library holds until the process exits (2 MiB + 256 B).
//
// Limits and sharing:
//   - states of at most 2^25 amplitudes (25 qubits); larger states are rejected;
//   - statevector data must be managed memory or device memory of the current
//     device (nothing is staged);
//   - every call shares the array, and each call overwrites what it uses before
//     reading it; calls whose work overlaps on the GPU (different streams or
//     host threads) race on it.
#include <stdio.h>

#include "rqc_common.cuh"
#include "rqcopt_gpu.h"

namespace {

constexpr int NA_TPB = 256;
constexpr int NA_TILE_GROUPS = 1024;   // amplitude groups per block (4 per thread)
constexpr int NA_MAX_TILES = 8192;     // 2^13 tiles x 2^10 groups x 4 amplitudes = 2^25 amplitudes
constexpr int NA_VALS = 32;            // doubles per tile: 16 complex dG entries
constexpr int NA_MAX_DEVICES = 128;

// per-tile partial sums [NA_MAX_TILES][NA_VALS], then the reduced dG [NA_VALS]
static __device__ __align__(256) double g_noalloc_scratch[NA_MAX_TILES * NA_VALS + NA_VALS];

// device address of g_noalloc_scratch, resolved once per device
static void* g_scratch_addr[NA_MAX_DEVICES];

__global__ void __launch_bounds__(NA_TPB) k_noalloc_backward(const double2* __restrict__ psi,
                                                             const double2* __restrict__ dout,
                                                             double2* __restrict__ dpsi, rqc::Gate4<double> g,
                                                             rqc::WirePair w, int64_t ngroups,
                                                             double* __restrict__ partials)
{
	double acc[NA_VALS];
#pragma unroll
	for (int k = 0; k < NA_VALS; k++) acc[k] = 0;
	int64_t off[4];
	rqc::group_offsets(w, off);
	const int64_t first = (int64_t)blockIdx.x * NA_TILE_GROUPS;
#pragma unroll
	for (int k = 0; k < NA_TILE_GROUPS / NA_TPB; k++) {
		const int64_t gi = first + k * NA_TPB + threadIdx.x;
		if (gi >= ngroups) break;
		const int64_t base = rqc::group_base(gi, w);
		double2 x[4], d[4], y[4];
#pragma unroll
		for (int m = 0; m < 4; m++) {
			x[m] = psi[base + off[m]];
			d[m] = dout[base + off[m]];
		}
#pragma unroll
		for (int r = 0; r < 4; r++)
#pragma unroll
			for (int c = 0; c < 4; c++) {
				const int e = 2 * (4 * r + c);
				acc[e]     = fma(d[r].x, x[c].x, fma(-d[r].y, x[c].y, acc[e]));
				acc[e + 1] = fma(d[r].x, x[c].y, fma(d[r].y, x[c].x, acc[e + 1]));
			}
		rqc::gate_apply_t(g, d, y);
#pragma unroll
		for (int m = 0; m < 4; m++) dpsi[base + off[m]] = y[m];
	}
	__shared__ double red[NA_TPB / 32][NA_VALS];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
	for (int k = 0; k < NA_VALS; k++) {
		const double v = rqc::warp_sum(acc[k]);
		if (lane == 0) red[warp][k] = v;
	}
	__syncthreads();
	if (threadIdx.x < NA_VALS) {
		double s = 0;
		for (int wi = 0; wi < NA_TPB / 32; wi++) s += red[wi][threadIdx.x];
		partials[(int64_t)blockIdx.x * NA_VALS + threadIdx.x] = s;   // written, so stale contents never leak in
	}
}

__global__ void k_noalloc_reduce(const double* __restrict__ partials, int ntiles, double* __restrict__ out)
{
	const int t = threadIdx.x;
	if (t >= NA_VALS) return;
	double sum = 0, comp = 0;
	for (int b = 0; b < ntiles; b++) {
		const double y = partials[(int64_t)b * NA_VALS + t] - comp;
		const double u = sum + y;
		comp = (u - sum) - y;
		sum = u;
	}
	out[t] = sum;
}

// Managed memory, or device memory of device `dev` (the device the kernels run
// on).  Device memory of another GPU is refused: the kernels would read it over
// a peer mapping that may not exist, and the scratch they use belongs to `dev`.
bool device_accessible(const void* p, int dev)
{
	cudaPointerAttributes a;
	if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
		cudaGetLastError();
		return false;
	}
	if (a.type == cudaMemoryTypeManaged) return true;
	return a.type == cudaMemoryTypeDevice && a.device == dev;
}

int report(cudaError_t e, const char* what)
{
	if (e == cudaSuccess) return 0;
	fprintf(stderr, "rqcopt_apply_gate_backward_noalloc: %s: %s\n", what, cudaGetErrorString(e));
	return -5;
}

}  // namespace

extern "C" int rqcopt_apply_gate_backward_noalloc(const struct mat4x4* gate, const int i, const int j,
                                                  const struct statevector* psi, const struct statevector* dpsi_out,
                                                  struct statevector* dpsi, struct mat4x4* dgate, void* stream)
{
	const char* fn = "rqcopt_apply_gate_backward_noalloc";
	if (!gate || !psi || !dpsi_out || !dpsi || !dgate || !psi->data || !dpsi_out->data || !dpsi->data) {
		fprintf(stderr, "%s: null argument\n", fn);
		return -6;
	}
	const int L = psi->nqubits;
	if (dpsi_out->nqubits != L || dpsi->nqubits != L || L < 2 || i < 0 || j < 0 || i >= L || j >= L || i == j) {
		fprintf(stderr, "%s: invalid wires or mismatching statevectors\n", fn);
		return -6;
	}
	if (L > RQCOPT_NOALLOC_MAX_QUBITS) {
		fprintf(stderr, "%s: %d qubits exceed the maximum of %d (the static scratch holds partial sums for at most "
		        "2^%d amplitudes)\n", fn, L, RQCOPT_NOALLOC_MAX_QUBITS, RQCOPT_NOALLOC_MAX_QUBITS);
		return -6;
	}
	int dev = -1;
	int ret = report(cudaGetDevice(&dev), "cudaGetDevice");
	if (ret) return ret;
	if (dev < 0 || dev >= NA_MAX_DEVICES) {
		fprintf(stderr, "%s: device ordinal %d out of range\n", fn, dev);
		return -6;
	}
	if (!device_accessible(psi->data, dev) || !device_accessible(dpsi_out->data, dev) ||
	    !device_accessible(dpsi->data, dev)) {
		fprintf(stderr, "%s: statevector data must be managed memory or device memory of the current device %d "
		        "(no staging without allocation)\n", fn, dev);
		return -6;
	}

	// one-time set-up per device: the device address of the static scratch
	if (!g_scratch_addr[dev]) {
		void* p = nullptr;
		if ((ret = report(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress"))) return ret;
		g_scratch_addr[dev] = p;
	}
	double* partials = static_cast<double*>(g_scratch_addr[dev]);
	double* result = partials + (size_t)NA_MAX_TILES * NA_VALS;

	cudaStream_t s = static_cast<cudaStream_t>(stream);
	const int64_t ngroups = (int64_t)1 << (L - 2);
	const int ntiles = (int)((ngroups + NA_TILE_GROUPS - 1) / NA_TILE_GROUPS);
	rqc::Gate4<double> g;
	for (int k = 0; k < 16; k++) g.m[k] = reinterpret_cast<const double2*>(gate->data)[k];
	k_noalloc_backward<<<ntiles, NA_TPB, 0, s>>>(reinterpret_cast<const double2*>(psi->data),
	                                              reinterpret_cast<const double2*>(dpsi_out->data),
	                                              reinterpret_cast<double2*>(dpsi->data), g, rqc::make_pair_(L, i, j),
	                                              ngroups, partials);
	if ((ret = report(cudaGetLastError(), "launch"))) return ret;
	k_noalloc_reduce<<<1, NA_VALS, 0, s>>>(partials, ntiles, result);
	if ((ret = report(cudaGetLastError(), "launch"))) return ret;
	if ((ret = report(cudaMemcpyAsync(dgate->data, result, 16 * sizeof(double2), cudaMemcpyDefault, s), "copy dgate")))
		return ret;
	return report(cudaStreamSynchronize(s), "synchronize");
}
