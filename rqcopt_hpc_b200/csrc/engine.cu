// Basis-column evaluation engine (see engine.h).
//
// Layout: a chunk of C basis columns is stored as C statevectors of 2^L
// amplitudes one after another ([C][2^L], complex128 or complex64).  Each gate
// pass is one kernel over all C * 2^(L-2) amplitude groups of the chunk, so a
// launch streams C * 2^L amplitudes per state it touches.
//
// Per column b the engine computes, for the circuit C = G_{n-1} ... G_0 and the
// target column phi = -conj(U e_b) (src/target.c:41-53):
//   forward  psi_{k+1} = G_k psi_k,   dpsi_{k+1} = G_k dpsi_k + Z_k psi_k
//            (psi_0 = e_b, dpsi_0 = 0; psi_k and dpsi_k are cached per gate)
//   f       += <phi, psi_n>                                   (no conjugation)
//   reverse  from phi_{n-1} = phi, dphi_{n-1} = 0, for k = n-1 .. 0:
//            dG_k += phi_k (x) psi_k
//            HZ_k += phi_k (x) dpsi_k + dphi_k (x) psi_k
//            phi_{k-1} = G_k^T phi_k,  dphi_{k-1} = G_k^T dphi_k + Z_k^T phi_k
// which is the per-column forward / reverse / forward-over-reverse scheme of
// src/quantum_circuit.c:147-236 with the two tangent sweeps folded into one
// forward and one reverse pass.  Column sums are formed per thread in FP64
// (complex64 passes accumulate FP32 products in short runs that are added into
// FP64), then per block, then over blocks with compensated summation.
#include "engine.h"
#include "engine_fused.h"

#include <stdio.h>
#include <string.h>
#include <algorithm>
#include <vector>

#include "rqc_common.cuh"
#include "rqcopt_gpu.h"

namespace rqc {

constexpr int TPB = 256;
constexpr int NPART = 64;   // doubles of partial sums per block and gate: 16 complex grad + 16 complex HVP

// ---------------------------------------------------------------------------------- helpers

// Paired basis columns (real-orthogonal problems): with c_pair_half = N/2 the column
// with basis index b (< N/2) is e_b + i e_{b + N/2}; 0 selects plain basis columns.
__constant__ int64_t c_pair_half = 0;

template <typename T>
__device__ __forceinline__ cplx<T> basis_amp(int64_t loc, int64_t b)
{
	return mk<T>(loc == b ? T(1) : T(0), (c_pair_half != 0 && loc == b + c_pair_half) ? T(1) : T(0));
}

__device__ __forceinline__ void block_add_f(double fx, double fy, double2* __restrict__ fpart)
{
	__shared__ double red[2][TPB / 32];
	fx = warp_sum(fx);
	fy = warp_sum(fy);
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	if (lane == 0) { red[0][warp] = fx; red[1][warp] = fy; }
	__syncthreads();
	if (threadIdx.x == 0) {
		double sx = 0, sy = 0;
		for (int k = 0; k < (int)(blockDim.x >> 5); k++) { sx += red[0][k]; sy += red[1][k]; }
		fpart[blockIdx.x].x += sx;
		fpart[blockIdx.x].y += sy;
	}
}

// ---------------------------------------------------------------------------------- kernels

// out = G in over all groups of a chunk.
//   IN  0: read `in`; 1: column c of the chunk is the basis vector e_{b0 + c}
//   OUT 0: store; 1: store -conj(.); 2: no store, accumulate f += <phi, out> into fpart
template <typename T, int IN, int OUT>
__global__ void __launch_bounds__(TPB) k_apply(const cplx<T>* __restrict__ in, cplx<T>* __restrict__ out,
                                               const cplx<T>* __restrict__ phi, Gate4<T> g, WirePair w, int L,
                                               int64_t ngroups, int64_t b0, double2* __restrict__ fpart)
{
	using V = cplx<T>;
	const int lg = L - 2;
	const int64_t gmask = ((int64_t)1 << lg) - 1;
	int64_t off[4];
	group_offsets(w, off);
	double fx = 0, fy = 0;
	for (int64_t gi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; gi < ngroups; gi += (int64_t)gridDim.x * blockDim.x) {
		const int64_t c = gi >> lg;
		const int64_t loc = group_base(gi & gmask, w);
		const int64_t base = (c << L) + loc;
		V x[4], y[4];
#pragma unroll
		for (int m = 0; m < 4; m++) x[m] = IN == 0 ? in[base + off[m]] : basis_amp<T>(loc + off[m], b0 + c);
		gate_apply(g, x, y);
#pragma unroll
		for (int m = 0; m < 4; m++) {
			if (OUT == 2) {
				const V p = phi[base + off[m]];
				fx += (double)p.x * y[m].x - (double)p.y * y[m].y;
				fy += (double)p.x * y[m].y + (double)p.y * y[m].x;
			} else if (OUT == 1) {
				out[base + off[m]] = cneg_conj(y[m]);
			} else {
				out[base + off[m]] = y[m];
			}
		}
	}
	if (OUT == 2) block_add_f(fx, fy, fpart);
}

// Forward pass of one gate with its tangent: psi_o = G psi, dpsi_o = G dpsi + Z psi.
// FIRST: psi is the basis column, dpsi = 0.  LAST: no stores, f += <phi, G psi>.
template <typename T, bool FIRST, bool LAST>
__global__ void __launch_bounds__(TPB) k_forward(const cplx<T>* __restrict__ psi, const cplx<T>* __restrict__ dpsi,
                                                 cplx<T>* __restrict__ psi_o, cplx<T>* __restrict__ dpsi_o,
                                                 const cplx<T>* __restrict__ phi, Gate4<T> g, Gate4<T> z, WirePair w,
                                                 int L, int64_t ngroups, int64_t b0, double2* __restrict__ fpart)
{
	using V = cplx<T>;
	const int lg = L - 2;
	const int64_t gmask = ((int64_t)1 << lg) - 1;
	int64_t off[4];
	group_offsets(w, off);
	double fx = 0, fy = 0;
	for (int64_t gi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; gi < ngroups; gi += (int64_t)gridDim.x * blockDim.x) {
		const int64_t c = gi >> lg;
		const int64_t loc = group_base(gi & gmask, w);
		const int64_t base = (c << L) + loc;
		V x[4], y[4];
#pragma unroll
		for (int m = 0; m < 4; m++) x[m] = FIRST ? basis_amp<T>(loc + off[m], b0 + c) : psi[base + off[m]];
		gate_apply(g, x, y);
		if (LAST) {
#pragma unroll
			for (int m = 0; m < 4; m++) {
				const V p = phi[base + off[m]];
				fx += (double)p.x * y[m].x - (double)p.y * y[m].y;
				fy += (double)p.x * y[m].y + (double)p.y * y[m].x;
			}
		} else {
			V dy[4];
			gate_apply(z, x, dy);
			if (!FIRST) {
				V dx[4];
#pragma unroll
				for (int m = 0; m < 4; m++) dx[m] = dpsi[base + off[m]];
				gate_apply_acc(g, dx, dy);
			}
#pragma unroll
			for (int m = 0; m < 4; m++) {
				psi_o[base + off[m]] = y[m];
				dpsi_o[base + off[m]] = dy[m];
			}
		}
	}
	if (LAST) block_add_f(fx, fy, fpart);
}

// Reverse pass of one gate.  Two threads share an amplitude group; thread half h
// owns gate rows {2h, 2h+1} of the outer-product sums and output components
// {2h, 2h+1} of G^T phi.
//   TAN:   also the tangent terms (HVP)
//   FIRST: k = n-1, dphi = 0
//   LAST:  k = 0, psi is the basis column, dpsi = 0, no outputs
// Partial sums go to part[blockIdx.x][64] (+=): doubles [0, 32) gradient and
// [32, 64) HVP, row-major complex entries.
template <typename T, bool TAN, bool FIRST, bool LAST>
__global__ void __launch_bounds__(TPB) k_reverse(const cplx<T>* __restrict__ phi, const cplx<T>* __restrict__ dphi,
                                                 const cplx<T>* __restrict__ psi, const cplx<T>* __restrict__ dpsi,
                                                 cplx<T>* __restrict__ phi_o, cplx<T>* __restrict__ dphi_o,
                                                 Gate4<T> g, Gate4<T> z, WirePair w, int L, int64_t ngroups,
                                                 int64_t b0, double* __restrict__ part)
{
	using V = cplx<T>;
	constexpr int NA = TAN ? 16 : 8;          // complex accumulators per thread
	constexpr bool FLUSH = sizeof(T) == 4;    // complex64: FP32 runs added into FP64
	constexpr int RUN = 16;
	const int lg = L - 2;
	const int64_t gmask = ((int64_t)1 << lg) - 1;
	int64_t off[4];
	group_offsets(w, off);
	const int h = threadIdx.x & 1;

	T acc[2 * NA];
	double accd[FLUSH ? 2 * NA : 1];
#pragma unroll
	for (int k = 0; k < 2 * NA; k++) acc[k] = 0;
	if (FLUSH) {
#pragma unroll
		for (int k = 0; k < 2 * NA; k++) accd[k] = 0;
	}
	int run = 0;

	const int64_t ntasks = ngroups * 2;
	for (int64_t ti = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; ti < ntasks; ti += (int64_t)gridDim.x * blockDim.x) {
		const int64_t gi = ti >> 1;
		const int64_t c = gi >> lg;
		const int64_t loc = group_base(gi & gmask, w);
		const int64_t base = (c << L) + loc;
		V p[4], x[4], dp[4], dx[4];
#pragma unroll
		for (int m = 0; m < 4; m++) {
			p[m] = phi[base + off[m]];
			x[m] = LAST ? basis_amp<T>(loc + off[m], b0 + c) : psi[base + off[m]];
			if (TAN) {
				dp[m] = FIRST ? czero<V>() : dphi[base + off[m]];
				dx[m] = LAST ? czero<V>() : dpsi[base + off[m]];
			}
		}
		// rows owned by this thread (selects, not dynamic indexing, keep the arrays in registers)
		V pr[2], dpr[2];
#pragma unroll
		for (int rr = 0; rr < 2; rr++) {
			pr[rr] = h ? p[2 + rr] : p[rr];
			if (TAN) dpr[rr] = h ? dp[2 + rr] : dp[rr];
		}
#pragma unroll
		for (int rr = 0; rr < 2; rr++) {
#pragma unroll
			for (int cc = 0; cc < 4; cc++) {
				const int e = 2 * (4 * rr + cc);
				acc[e]     = fma(pr[rr].x, x[cc].x, fma(-pr[rr].y, x[cc].y, acc[e]));
				acc[e + 1] = fma(pr[rr].x, x[cc].y, fma(pr[rr].y, x[cc].x, acc[e + 1]));
				if (TAN) {
					T hx = acc[16 + e], hy = acc[16 + e + 1];
					if (!LAST) {
						hx = fma(pr[rr].x, dx[cc].x, fma(-pr[rr].y, dx[cc].y, hx));
						hy = fma(pr[rr].x, dx[cc].y, fma(pr[rr].y, dx[cc].x, hy));
					}
					if (!FIRST) {
						hx = fma(dpr[rr].x, x[cc].x, fma(-dpr[rr].y, x[cc].y, hx));
						hy = fma(dpr[rr].x, x[cc].y, fma(dpr[rr].y, x[cc].x, hy));
					}
					acc[16 + e] = hx;
					acc[16 + e + 1] = hy;
				}
			}
		}
		if (FLUSH && ++run == RUN) {
			run = 0;
#pragma unroll
			for (int k = 0; k < 2 * NA; k++) { accd[k] += acc[k]; acc[k] = 0; }
		}
		if (!LAST) {
#pragma unroll
			for (int cc = 0; cc < 2; cc++) {
				// output component col = 2h + cc: (G^T p)[col] = sum_r G[r][col] p[r]
				const int64_t o = h ? off[2 + cc] : off[cc];
				V s = czero<V>(), ds = czero<V>();
#pragma unroll
				for (int r = 0; r < 4; r++) {
					const V gr = h ? g.m[4 * r + 2 + cc] : g.m[4 * r + cc];
					s = cfma(gr, p[r], s);
					if (TAN) {
						const V zr = h ? z.m[4 * r + 2 + cc] : z.m[4 * r + cc];
						ds = cfma(zr, p[r], ds);
						if (!FIRST) ds = cfma(gr, dp[r], ds);
					}
				}
				phi_o[base + o] = s;
				if (TAN) dphi_o[base + o] = ds;
			}
		}
	}

	// reduce over the lanes of equal parity, then over warps
	__shared__ double red[TPB / 32][2][32];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
	for (int k = 0; k < 2 * NA; k++) {
		double v = FLUSH ? accd[k] + (double)acc[k] : (double)acc[k];
#pragma unroll
		for (int o = 16; o > 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
		if (lane < 2) red[warp][lane][k] = v;
	}
	__syncthreads();
	if (threadIdx.x < 64) {
		const int half = threadIdx.x >> 5, k = threadIdx.x & 31;
		if (k < 2 * NA) {
			double s = 0;
			for (int wi = 0; wi < (int)(blockDim.x >> 5); wi++) s += red[wi][half][k];
			const int dst = k < 16 ? 16 * half + k : 32 + 16 * half + (k - 16);
			part[(size_t)blockIdx.x * NPART + dst] += s;
		}
	}
}

// out = -conj(in), converting from complex128 host columns to the pass precision
template <typename T>
__global__ void k_conj_neg(const double2* __restrict__ in, cplx<T>* __restrict__ out, int64_t n)
{
	for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
		const double2 v = in[i];
		out[i] = mk<T>((T)(-v.x), (T)v.y);
	}
}

// Sum partials over blocks (compensated).  Block s < nslots reduces gate s, block
// nslots reduces f.  out: [0] f, [1 + 16 s + e] grad, [1 + 16 nslots + 16 s + e] HVP.
__global__ void k_reduce(const double* __restrict__ part, const double2* __restrict__ fpart, int nslots, int nblk,
                         int with_hvp, double2* __restrict__ out)
{
	double* o = reinterpret_cast<double*>(out);
	const int s = blockIdx.x, t = threadIdx.x;
	if (s < nslots) {
		if (t >= NPART || (!with_hvp && t >= 32)) return;
		double sum = 0, comp = 0;
		for (int b = 0; b < nblk; b++) {
			const double y = part[((size_t)s * nblk + b) * NPART + t] - comp;
			const double u = sum + y;
			comp = (u - sum) - y;
			sum = u;
		}
		if (t < 32) o[2 * (1 + 16 * (size_t)s) + t] = sum;
		else o[2 * (1 + 16 * (size_t)nslots + 16 * (size_t)s) + (t - 32)] = sum;
	} else if (t < 2) {
		double sum = 0, comp = 0;
		for (int b = 0; b < nblk; b++) {
			const double v = t == 0 ? fpart[b].x : fpart[b].y;
			const double y = v - comp;
			const double u = sum + y;
			comp = (u - sum) - y;
			sum = u;
		}
		o[t] = sum;
	}
}

__global__ void k_add(const double2* __restrict__ a, const double2* __restrict__ b, double2* __restrict__ c, int64_t n)
{
	for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
		c[i] = make_double2(a[i].x + b[i].x, a[i].y + b[i].y);
}

// ---------------------------------------------------------------------------------- launch helpers

template <typename KernelT>
static int blocks_per_sm(KernelT kernel)
{
	int n = 0;
	if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, TPB, 0) != cudaSuccess || n < 1) {
		cudaGetLastError();
		n = 1;
	}
	return n;
}

static int grid_for(const Runtime& rt, int64_t work_items, int max_per_sm)
{
	const int64_t want = (work_items + TPB - 1) / TPB;
	const int64_t cap = (int64_t)rt.num_sms * max_per_sm;
	return (int)std::max<int64_t>(1, std::min(want, cap));
}

#define RQC_LAUNCH(RT, CLS, KERNEL, GRID, ...)                                   \
	do {                                                                         \
		cudaEvent_t ev__;                                                        \
		launch_begin((RT), (CLS), &ev__);                                        \
		KERNEL<<<(GRID), TPB, 0, (RT).stream>>>(__VA_ARGS__);                    \
		launch_end((RT), (CLS), ev__);                                           \
		if (int e__ = RQC_CUDA(cudaGetLastError())) return e__;                  \
	} while (0)

template <typename T>
static Gate4<T> to_gate(const double2* g)
{
	Gate4<T> r;
	for (int k = 0; k < 16; k++) r.m[k] = mk<T>((T)g[k].x, (T)g[k].y);
	return r;
}

template <typename T>
static int launch_apply(Runtime& rt, int in_mode, int out_mode, const cplx<T>* in, cplx<T>* out, const cplx<T>* phi,
                        const Gate4<T>& g, const WirePair& w, int L, int64_t ngroups, int64_t b0, double2* fpart, int fgrid)
{
	const int grid = out_mode == 2 ? fgrid : grid_for(rt, ngroups, 8);
#define RQC_APPLY_CASE(I, O)                                                                             \
	if (in_mode == I && out_mode == O) {                                                                 \
		RQC_LAUNCH(rt, KC_APPLY, (k_apply<T, I, O>), grid, in, out, phi, g, w, L, ngroups, b0, fpart); \
		return OK;                                                                                       \
	}
	RQC_APPLY_CASE(0, 0) RQC_APPLY_CASE(0, 1) RQC_APPLY_CASE(0, 2)
	RQC_APPLY_CASE(1, 0) RQC_APPLY_CASE(1, 1) RQC_APPLY_CASE(1, 2)
#undef RQC_APPLY_CASE
	return E_ARG;
}

template <typename T>
static int launch_forward(Runtime& rt, bool first, bool last, const cplx<T>* psi, const cplx<T>* dpsi, cplx<T>* psi_o,
                          cplx<T>* dpsi_o, const cplx<T>* phi, const Gate4<T>& g, const Gate4<T>& z, const WirePair& w,
                          int L, int64_t ngroups, int64_t b0, double2* fpart, int fgrid)
{
	const int grid = last ? fgrid : grid_for(rt, ngroups, 8);
#define RQC_FWD_CASE(F, LA)                                                                                         \
	if (first == F && last == LA) {                                                                                 \
		RQC_LAUNCH(rt, KC_FORWARD, (k_forward<T, F, LA>), grid, psi, dpsi, psi_o, dpsi_o, phi, g, z, w, L, ngroups, \
		           b0, fpart);                                                                                      \
		return OK;                                                                                                  \
	}
	RQC_FWD_CASE(false, false) RQC_FWD_CASE(true, false) RQC_FWD_CASE(false, true) RQC_FWD_CASE(true, true)
#undef RQC_FWD_CASE
	return E_ARG;
}

template <typename T>
static int launch_reverse(Runtime& rt, bool tan, bool first, bool last, const cplx<T>* phi, const cplx<T>* dphi,
                          const cplx<T>* psi, const cplx<T>* dpsi, cplx<T>* phi_o, cplx<T>* dphi_o, const Gate4<T>& g,
                          const Gate4<T>& z, const WirePair& w, int L, int64_t ngroups, int64_t b0, double* part,
                          int grid)
{
#define RQC_REV_CASE(TA, F, LA)                                                                                        \
	if (tan == TA && first == F && last == LA) {                                                                       \
		RQC_LAUNCH(rt, KC_REVERSE, (k_reverse<T, TA, F, LA>), grid, phi, dphi, psi, dpsi, phi_o, dphi_o, g, z, w, L,   \
		           ngroups, b0, part);                                                                                 \
		return OK;                                                                                                     \
	}
	RQC_REV_CASE(false, false, false) RQC_REV_CASE(false, true, false)
	RQC_REV_CASE(false, false, true) RQC_REV_CASE(false, true, true)
	RQC_REV_CASE(true, false, false) RQC_REV_CASE(true, true, false)
	RQC_REV_CASE(true, false, true) RQC_REV_CASE(true, true, true)
#undef RQC_REV_CASE
	return E_ARG;
}

// grid of the partial-sum kernels: one full wave of the reverse kernel
template <typename T>
static int partial_grid(const Runtime& rt)
{
	static int per_sm = 0;
	if (per_sm == 0) per_sm = std::max(1, std::min(blocks_per_sm(k_reverse<T, true, false, false>),
	                                                blocks_per_sm(k_forward<T, false, true>)));
	return rt.num_sms * per_sm;
}

static size_t workspace_limit(Runtime& rt)
{
	if (rt.workspace_limit) return rt.workspace_limit;
	size_t free_b = 0, total_b = 0;
	if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
		cudaGetLastError();
		return (size_t)1 << 30;
	}
	return (size_t)((free_b + rt.work.bytes) * 0.75);
}

// ---------------------------------------------------------------------------------- evaluation

template <typename T>
static int evaluate_t(Runtime& rt, const CircuitSpec& c, const TargetSpec& t, int mode, double2* d_out)
{
	using V = cplx<T>;
	const int L = c.L, G = c.ngates;
	const int64_t N = (int64_t)1 << L;
	const int64_t ncols = rt.real_pairs ? N / 2 : N;   // (paired) basis columns
	const bool tan = mode == EVAL_HVP;
	const bool host_target = t.ufunc != nullptr;

	std::vector<Gate4<T>> gg(G), zz(tan ? G : 0), tg(t.ngates);
	std::vector<WirePair> gw(G), tw(t.ngates);
	for (int k = 0; k < G; k++) {
		gg[k] = to_gate<T>(c.gates + 16 * k);
		if (tan) zz[k] = to_gate<T>(c.dirs + 16 * k);
		gw[k] = make_pair_(L, c.wires[2 * k], c.wires[2 * k + 1]);
	}
	for (int k = 0; k < t.ngates; k++) {
		tg[k] = to_gate<T>(t.gates + 16 * k);
		tw[k] = make_pair_(L, t.wires[2 * k], t.wires[2 * k + 1]);
	}

	// states per column: PHI, P0, P1 (+ D0, D1) and the cached forward states
	const int64_t nstates = mode == EVAL_F ? 3 : (mode == EVAL_GRAD ? 3 + (G - 1) : 5 + 2 * (int64_t)(G - 1));
	const size_t col_bytes = (size_t)nstates * N * sizeof(V);
	const int64_t cbeg = std::min<int64_t>(rt.col_begin, ncols);
	const int64_t cend = rt.col_end > 0 ? std::min<int64_t>(rt.col_end, ncols) : ncols;
	int64_t C = (int64_t)(workspace_limit(rt) / col_bytes);
	if (rt.column_chunk > 0) C = std::min<int64_t>(C, rt.column_chunk);
	if (host_target) C = std::min<int64_t>(C, std::max<int64_t>(1, ((int64_t)256 << 20) / (N * 16)));
	C = std::min(C, std::max<int64_t>(1, cend - cbeg));
	if (C < 1) {
		fprintf(stderr, "rqcopt_gpu: one basis column needs %zu bytes of workspace, more than the limit\n", col_bytes);
		return E_ALLOC;
	}
	int ret = ensure_device(rt.work, (size_t)nstates * C * N * sizeof(V));
	if (ret) return ret;
	V* PHI = reinterpret_cast<V*>(rt.work.ptr);
	V* P[2] = { PHI + C * N, PHI + 2 * C * N };
	V* D[2] = { tan ? PHI + 3 * C * N : nullptr, tan ? PHI + 4 * C * N : nullptr };
	V* cache = PHI + (tan ? 5 : 3) * C * N;                       // psi_1 .. psi_{G-1}
	V* dcache = tan ? cache + (int64_t)(G - 1) * C * N : nullptr; // dpsi_1 .. dpsi_{G-1}
	auto cache_at = [&](int k) { return cache + (int64_t)(k - 1) * C * N; };
	auto dcache_at = [&](int k) { return dcache + (int64_t)(k - 1) * C * N; };

	const int nblk = partial_grid<T>(rt);
	const size_t part_doubles = (size_t)G * nblk * NPART + 2 * (size_t)nblk;
	if ((ret = ensure_device(rt.partials, part_doubles * sizeof(double)))) return ret;
	double* part = reinterpret_cast<double*>(rt.partials.ptr);
	double2* fpart = reinterpret_cast<double2*>(part + (size_t)G * nblk * NPART);
	if ((ret = RQC_CUDA(cudaMemsetAsync(part, 0, part_doubles * sizeof(double), rt.stream)))) return ret;

	// host callback target: pinned column buffer and one basis vector
	double2* hcols = nullptr;
	double2* hbasis = nullptr;
	if (host_target) {
		if ((ret = ensure_host_pinned(rt.hpin, (size_t)(C + 1) * N * sizeof(double2)))) return ret;
		hcols = reinterpret_cast<double2*>(rt.hpin.ptr);
		hbasis = hcols + C * N;
	}

	for (int64_t b0 = cbeg; b0 < cend; b0 += C) {
		const int64_t Cc = std::min(C, cend - b0);
		const int64_t ngroups = Cc * (N / 4);

		// target columns phi = -conj(U e_b)
		if (host_target) {
			const linear_func uf = reinterpret_cast<linear_func>(t.ufunc);
			for (int64_t cidx = 0; cidx < Cc; cidx++) {
				memset(hbasis, 0, N * sizeof(double2));
				hbasis[b0 + cidx].x = 1;
				if (rt.real_pairs) hbasis[b0 + cidx + N / 2].y = 1;
				statevector e = { reinterpret_cast<numeric*>(hbasis), L };
				statevector u = { reinterpret_cast<numeric*>(hcols + cidx * N), L };
				const int r = uf(&e, t.udata, &u);
				if (r < 0) {
					fprintf(stderr, "rqcopt_gpu: call of 'ufunc' failed, return value: %i\n", r);
					return E_UFUNC;
				}
			}
			double2* staged = reinterpret_cast<double2*>(P[0]);   // P0 (and P1) are free here
			if ((ret = RQC_CUDA(cudaMemcpyAsync(staged, hcols, Cc * N * sizeof(double2), cudaMemcpyHostToDevice, rt.stream))))
				return ret;
			k_conj_neg<T><<<grid_for(rt, Cc * N, 8), TPB, 0, rt.stream>>>(staged, PHI, Cc * N);
			rt.launches++;
			if ((ret = RQC_CUDA(cudaGetLastError()))) return ret;
			// the pinned buffer is reused by the next chunk
			if ((ret = RQC_CUDA(cudaStreamSynchronize(rt.stream)))) return ret;
		} else {
			const int Gt = t.ngates;
			for (int k = 0; k < Gt; k++) {
				const bool first = k == 0, last = k == Gt - 1;
				const V* in = first ? nullptr : P[(k - 1) & 1];
				V* out = last ? PHI : P[k & 1];
				if ((ret = launch_apply<T>(rt, first ? 1 : 0, last ? 1 : 0, in, out, nullptr, tg[k], tw[k], L, ngroups,
				                           b0, nullptr, nblk)))
					return ret;
			}
		}

		if (mode == EVAL_F) {
			for (int k = 0; k < G; k++) {
				const bool first = k == 0, last = k == G - 1;
				const V* in = first ? nullptr : P[(k - 1) & 1];
				if ((ret = launch_apply<T>(rt, first ? 1 : 0, last ? 2 : 0, in, last ? nullptr : P[k & 1], PHI, gg[k], gw[k],
				                           L, ngroups, b0, fpart, nblk)))
					return ret;
			}
			continue;
		}

		// forward pass, caching psi_k (and dpsi_k)
		for (int k = 0; k < G; k++) {
			const bool first = k == 0, last = k == G - 1;
			if (tan) {
				if ((ret = launch_forward<T>(rt, first, last, first ? nullptr : cache_at(k), first ? nullptr : dcache_at(k),
				                             last ? nullptr : cache_at(k + 1), last ? nullptr : dcache_at(k + 1), PHI, gg[k],
				                             zz[k], gw[k], L, ngroups, b0, fpart, nblk)))
					return ret;
			} else {
				if ((ret = launch_apply<T>(rt, first ? 1 : 0, last ? 2 : 0, first ? nullptr : cache_at(k),
				                           last ? nullptr : cache_at(k + 1), PHI, gg[k], gw[k], L, ngroups, b0, fpart, nblk)))
					return ret;
			}
		}

		// reverse pass
		const Gate4<T> zero_gate{};
		for (int k = G - 1; k >= 0; k--) {
			const bool first = k == G - 1, last = k == 0;
			const int cur = (G - 1 - k) & 1, nxt = cur ^ 1;
			const V* ph = first ? PHI : P[cur];
			const V* dph = (first || !tan) ? nullptr : D[cur];
			if ((ret = launch_reverse<T>(rt, tan, first, last, ph, dph, last ? nullptr : cache_at(k),
			                             (last || !tan) ? nullptr : dcache_at(k), last ? nullptr : P[nxt],
			                             (last || !tan) ? nullptr : D[nxt], gg[k], tan ? zz[k] : zero_gate, gw[k], L,
			                             ngroups, b0, part + (size_t)k * nblk * NPART, nblk)))
				return ret;
		}
	}

	k_reduce<<<G + 1, 64, 0, rt.stream>>>(part, fpart, G, nblk, tan ? 1 : 0, d_out);
	rt.launches++;
	return RQC_CUDA(cudaGetLastError());
}

int set_pair_half_fused(Runtime& rt, int64_t half);

namespace {

__global__ void k_real_part(double2* __restrict__ d, int64_t n)
{
	for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
		d[i].y = 0;
}

int set_pair_half(Runtime& rt, int64_t half)
{
	int ret = RQC_CUDA(cudaMemcpyToSymbolAsync(c_pair_half, &half, sizeof(half), 0, cudaMemcpyHostToDevice, rt.stream));
	return ret ? ret : set_pair_half_fused(rt, half);
}

}  // namespace

static int evaluate_columns(Runtime& rt, const CircuitSpec& c, const TargetSpec& t, int mode, int precision,
                            double2* d_out);

// the configured evaluation (gates per pass, column chunk, reverse variant as set in rt)
int evaluate_configured(Runtime& rt, const CircuitSpec& c, const TargetSpec& t, int mode, int precision, double2* d_out)
{
	return evaluate_columns(rt, c, t, mode, precision, d_out);
}

// With rt.real_pairs (real gates, real target): the 2^(L-1) paired columns
// e_b + i e_{b + N/2}.  Every sum the engine forms pairs an adjoint-type state (from
// -conj(U psi)) with a forward-type state, both propagated by real matrices, so its
// real part is the sum of the two real columns' terms; the imaginary parts (cross
// terms) are cleared.
int evaluate(Runtime& rt, const CircuitSpec& c, const TargetSpec& t, int mode, int precision, double2* d_out)
{
	if (!rt.real_pairs) return evaluate_autotuned(rt, c, t, mode, precision, d_out);
	if (c.L < 2) return E_ARG;
	int ret = set_pair_half(rt, (int64_t)1 << (c.L - 1));
	if (!ret) ret = evaluate_autotuned(rt, c, t, mode, precision, d_out);
	const int reset = set_pair_half(rt, 0);
	if (!ret) ret = reset;
	if (ret) return ret;
	k_real_part<<<1, 256, 0, rt.stream>>>(d_out, (int64_t)result_count(c.ngates));
	rt.launches++;
	return RQC_CUDA(cudaGetLastError());
}

static int evaluate_columns(Runtime& rt, const CircuitSpec& c, const TargetSpec& t, int mode, int precision,
                            double2* d_out)
{
	if (c.L < 2 || c.ngates < 1) return E_ARG;
	for (int k = 0; k < 2 * c.ngates; k++)
		if (c.wires[k] < 0 || c.wires[k] >= c.L) return E_ARG;
	for (int k = 0; k < c.ngates; k++)
		if (c.wires[2 * k] == c.wires[2 * k + 1]) return E_ARG;
	for (int k = 0; k < t.ngates; k++)
		if (t.wires[2 * k] < 0 || t.wires[2 * k] >= c.L || t.wires[2 * k + 1] < 0 || t.wires[2 * k + 1] >= c.L ||
		    t.wires[2 * k] == t.wires[2 * k + 1])
			return E_ARG;
	if (!t.ufunc && t.ngates < 1) return E_ARG;
	if (mode != EVAL_GRAD && mode != EVAL_HVP) {
		// f only: the reduction still writes the (zero) gradient slots
		mode = EVAL_F;
	}
	int ret;
	if ((ret = RQC_CUDA(cudaMemsetAsync(d_out, 0, result_count(c.ngates) * sizeof(double2), rt.stream)))) return ret;
	if (rt.gates_per_pass > 1 && c.L >= 4) return evaluate_fused(rt, c, t, mode, precision, rt.gates_per_pass, d_out);
	if (precision == PREC_C128) return evaluate_t<double>(rt, c, t, mode, d_out);
	return evaluate_t<float>(rt, c, t, mode, d_out);
}

// ---------------------------------------------------------------------------------- single passes

int gate_apply_device(Runtime& rt, int L, const double2* gate, int i, int j, const double2* d_in, double2* d_out, long ncols)
{
	const int64_t ngroups = (int64_t)ncols << (L - 2);
	return launch_apply<double>(rt, 0, 0, d_in, d_out, nullptr, to_gate<double>(gate), make_pair_(L, i, j), L, ngroups, 0,
	                            nullptr, 0);
}

int apply_circuit_device(Runtime& rt, int L, int ngates, const double2* gates, const int* wires, const double2* d_in,
                         double2* d_out, long ncols)
{
	if (ncols == 1 && rt.gates_per_pass > 1 && L >= 10 && L <= 31)
		return apply_circuit_fused_device(rt, L, ngates, gates, wires, d_in, d_out, rt.gates_per_pass);
	// ping-pong between d_out and one scratch buffer so that the last gate writes d_out
	const size_t bytes = (size_t)ncols * ((size_t)1 << L) * sizeof(double2);
	int ret;
	if (ngates > 1 && (ret = ensure_device(rt.stage[3], bytes))) return ret;
	double2* tmp = reinterpret_cast<double2*>(rt.stage[3].ptr);
	const double2* src = d_in;
	for (int k = 0; k < ngates; k++) {
		double2* dst = ((ngates - 1 - k) % 2 == 0) ? d_out : tmp;
		if ((ret = gate_apply_device(rt, L, gates + 16 * k, wires[2 * k], wires[2 * k + 1], src, dst, ncols))) return ret;
		src = dst;
	}
	return OK;
}

int apply_circuit_device_c64(Runtime& rt, int L, int ngates, const double2* gates, const int* wires, const float2* d_in,
                             float2* d_out)
{
	if (rt.gates_per_pass > 1 && L >= 10 && L <= 31)
		return apply_circuit_fused_device_c64(rt, L, ngates, gates, wires, d_in, d_out, rt.gates_per_pass);
	const size_t bytes = ((size_t)1 << L) * sizeof(float2);
	int ret;
	if (ngates > 1 && (ret = ensure_device(rt.stage[3], bytes))) return ret;
	float2* tmp = reinterpret_cast<float2*>(rt.stage[3].ptr);
	const float2* src = d_in;
	const int64_t ngroups = (int64_t)1 << (L - 2);
	for (int k = 0; k < ngates; k++) {
		float2* dst = ((ngates - 1 - k) % 2 == 0) ? d_out : tmp;
		if ((ret = launch_apply<float>(rt, 0, 0, src, dst, nullptr, to_gate<float>(gates + 16 * k),
		                               make_pair_(L, wires[2 * k], wires[2 * k + 1]), L, ngroups, 0, nullptr, 0)))
			return ret;
		src = dst;
	}
	return OK;
}

int gate_backward_device(Runtime& rt, int L, const double2* gate, int i, int j, const double2* d_psi,
                         const double2* d_dout, double2* d_dpsi, double2* d_dgate)
{
	const int64_t ngroups = (int64_t)1 << (L - 2);
	const int nblk = std::min(partial_grid<double>(rt), grid_for(rt, 2 * ngroups, 64));
	int ret;
	const size_t part_doubles = (size_t)nblk * NPART + 2 * (size_t)nblk;
	if ((ret = ensure_device(rt.partials, part_doubles * sizeof(double)))) return ret;
	double* part = reinterpret_cast<double*>(rt.partials.ptr);
	double2* fpart = reinterpret_cast<double2*>(part + (size_t)nblk * NPART);
	if ((ret = RQC_CUDA(cudaMemsetAsync(part, 0, part_doubles * sizeof(double), rt.stream)))) return ret;
	const Gate4<double> zero_gate{};
	if ((ret = launch_reverse<double>(rt, false, true, false, d_dout, nullptr, d_psi, nullptr, d_dpsi, nullptr,
	                                  to_gate<double>(gate), zero_gate, make_pair_(L, i, j), L, ngroups, 0, part, nblk)))
		return ret;
	if ((ret = ensure_device(rt.result, result_count(1) * sizeof(double2)))) return ret;
	double2* res = reinterpret_cast<double2*>(rt.result.ptr);
	k_reduce<<<2, 64, 0, rt.stream>>>(part, fpart, 1, nblk, 0, res);
	rt.launches++;
	if ((ret = RQC_CUDA(cudaGetLastError()))) return ret;
	return RQC_CUDA(cudaMemcpyAsync(d_dgate, res + 1, 16 * sizeof(double2), cudaMemcpyDeviceToDevice, rt.stream));
}

int target_columns_device(Runtime& rt, const TargetSpec& t, int L, int64_t b0, int64_t ncols, double2* phi,
                          double2* p0, double2* p1)
{
	const int64_t N = (int64_t)1 << L;
	const int64_t ngroups = ncols * (N / 4);
	int ret;
	if (t.ufunc) {
		if ((ret = ensure_host_pinned(rt.hpin, (size_t)(ncols + 1) * N * sizeof(double2)))) return ret;
		double2* hcols = reinterpret_cast<double2*>(rt.hpin.ptr);
		double2* hbasis = hcols + ncols * N;
		const linear_func uf = reinterpret_cast<linear_func>(t.ufunc);
		for (int64_t c = 0; c < ncols; c++) {
			memset(hbasis, 0, N * sizeof(double2));
			hbasis[b0 + c].x = 1;
			statevector e = { reinterpret_cast<numeric*>(hbasis), L };
			statevector u = { reinterpret_cast<numeric*>(hcols + c * N), L };
			const int r = uf(&e, t.udata, &u);
			if (r < 0) {
				fprintf(stderr, "rqcopt_gpu: call of 'ufunc' failed, return value: %i\n", r);
				return E_UFUNC;
			}
		}
		if ((ret = RQC_CUDA(cudaMemcpyAsync(p0, hcols, ncols * N * sizeof(double2), cudaMemcpyHostToDevice, rt.stream))))
			return ret;
		k_conj_neg<double><<<grid_for(rt, ncols * N, 8), TPB, 0, rt.stream>>>(p0, phi, ncols * N);
		rt.launches++;
		if ((ret = RQC_CUDA(cudaGetLastError()))) return ret;
		// the pinned buffer is reused by the next chunk
		return RQC_CUDA(cudaStreamSynchronize(rt.stream));
	}
	double2* P[2] = { p0, p1 };
	for (int k = 0; k < t.ngates; k++) {
		const bool first = k == 0, last = k == t.ngates - 1;
		if ((ret = launch_apply<double>(rt, first ? 1 : 0, last ? 1 : 0, first ? nullptr : P[(k - 1) & 1],
		                                last ? phi : P[k & 1], nullptr, to_gate<double>(t.gates + 16 * k),
		                                make_pair_(L, t.wires[2 * k], t.wires[2 * k + 1]), L, ngroups, b0, nullptr, 0)))
			return ret;
	}
	return OK;
}

int target_states_device(Runtime& rt, const TargetSpec& t, int L, const double2* states, int64_t ncols, double2* phi,
                         double2* p0, double2* p1)
{
	const int64_t N = (int64_t)1 << L;
	const int64_t ngroups = ncols * (N / 4);
	int ret;
	if (t.ufunc) {
		if ((ret = ensure_host_pinned(rt.hpin, (size_t)(2 * ncols) * N * sizeof(double2)))) return ret;
		double2* hin = reinterpret_cast<double2*>(rt.hpin.ptr);
		double2* hout = hin + ncols * N;
		if ((ret = RQC_CUDA(cudaMemcpyAsync(hin, states, ncols * N * sizeof(double2), cudaMemcpyDeviceToHost, rt.stream))))
			return ret;
		if ((ret = RQC_CUDA(cudaStreamSynchronize(rt.stream)))) return ret;
		const linear_func uf = reinterpret_cast<linear_func>(t.ufunc);
		for (int64_t c = 0; c < ncols; c++) {
			statevector e = { reinterpret_cast<numeric*>(hin + c * N), L };
			statevector u = { reinterpret_cast<numeric*>(hout + c * N), L };
			const int r = uf(&e, t.udata, &u);
			if (r < 0) {
				fprintf(stderr, "rqcopt_gpu: call of 'ufunc' failed, return value: %i\n", r);
				return E_UFUNC;
			}
		}
		if ((ret = RQC_CUDA(cudaMemcpyAsync(p0, hout, ncols * N * sizeof(double2), cudaMemcpyHostToDevice, rt.stream))))
			return ret;
		k_conj_neg<double><<<grid_for(rt, ncols * N, 8), TPB, 0, rt.stream>>>(p0, phi, ncols * N);
		rt.launches++;
		if ((ret = RQC_CUDA(cudaGetLastError()))) return ret;
		return RQC_CUDA(cudaStreamSynchronize(rt.stream));
	}
	double2* P[2] = { p0, p1 };
	for (int k = 0; k < t.ngates; k++) {
		const bool first = k == 0, last = k == t.ngates - 1;
		if ((ret = launch_apply<double>(rt, 0, last ? 1 : 0, first ? states : P[(k - 1) & 1], last ? phi : P[k & 1],
		                                nullptr, to_gate<double>(t.gates + 16 * k),
		                                make_pair_(L, t.wires[2 * k], t.wires[2 * k + 1]), L, ngroups, 0, nullptr, 0)))
			return ret;
	}
	return OK;
}

int add_device(Runtime& rt, const double2* a, const double2* b, double2* c, long n)
{
	RQC_LAUNCH(rt, KC_APPLY, k_add, grid_for(rt, n, 8), a, b, c, (int64_t)n);
	return OK;
}

}  // namespace rqc

namespace rqc {

int column_passes_device(Runtime& rt, int L, int ngates, const double2* gates, const double2* dirs, const int* wires,
                         const double2* d_psi, const double2* d_phi, double2* d_psi_out, double2* d_dgates,
                         double2* d_hess)
{
	using V = double2;
	const int G = ngates;
	const bool tan = dirs != nullptr;
	const int64_t N = (int64_t)1 << L;
	const int64_t ngroups = N / 4;
	// work: cache psi_1..psi_{G-1} (+ dpsi_0..dpsi_{G-1}), P0, P1 (+ D0, D1), scratch pair
	const int64_t nstates = (G - 1) + 4 + (tan ? G + 2 : 0);
	int ret;
	if ((ret = ensure_device(rt.work, (size_t)nstates * N * sizeof(V)))) return ret;
	V* w0 = reinterpret_cast<V*>(rt.work.ptr);
	V* cache = w0;                              // psi_k at cache + (k-1) N, k >= 1
	V* P[2] = { w0 + (G - 1) * N, w0 + G * N };
	V* sink = w0 + (G + 1) * N;                 // outputs nobody reads (2 states)
	V* dcache = tan ? w0 + (G + 3) * N : nullptr;   // dpsi_k at dcache + k N, k >= 0 (dpsi_0 = 0)
	V* D[2] = { tan ? dcache + G * N : nullptr, tan ? dcache + (G + 1) * N : nullptr };
	auto psi_at = [&](int k) -> const V* { return k == 0 ? d_psi : cache + (int64_t)(k - 1) * N; };
	if (tan && (ret = RQC_CUDA(cudaMemsetAsync(dcache, 0, N * sizeof(V), rt.stream)))) return ret;

	const int nblk = std::min(partial_grid<double>(rt), grid_for(rt, 2 * ngroups, 64));
	const size_t part_doubles = (size_t)G * nblk * NPART + 2 * (size_t)nblk;
	if ((ret = ensure_device(rt.partials, part_doubles * sizeof(double)))) return ret;
	double* part = reinterpret_cast<double*>(rt.partials.ptr);
	double2* fpart = reinterpret_cast<double2*>(part + (size_t)G * nblk * NPART);
	if ((ret = RQC_CUDA(cudaMemsetAsync(part, 0, part_doubles * sizeof(double), rt.stream)))) return ret;

	std::vector<Gate4<double>> gg(G), zz(G);
	std::vector<WirePair> gw(G);
	for (int k = 0; k < G; k++) {
		gg[k] = to_gate<double>(gates + 16 * k);
		zz[k] = tan ? to_gate<double>(dirs + 16 * k) : Gate4<double>{};
		gw[k] = make_pair_(L, wires[2 * k], wires[2 * k + 1]);
	}
	// forward
	for (int k = 0; k < G; k++) {
		V* out = k + 1 < G ? cache + (int64_t)k * N : d_psi_out;
		if (tan) {
			V* dout = k + 1 < G ? dcache + (int64_t)(k + 1) * N : sink;
			if ((ret = launch_forward<double>(rt, false, false, psi_at(k), dcache + (int64_t)k * N, out, dout, nullptr,
			                                  gg[k], zz[k], gw[k], L, ngroups, 0, nullptr, 0)))
				return ret;
		} else {
			if ((ret = launch_apply<double>(rt, 0, 0, psi_at(k), out, nullptr, gg[k], gw[k], L, ngroups, 0, nullptr, 0)))
				return ret;
		}
	}
	// reverse
	for (int k = G - 1; k >= 0; k--) {
		const bool first = k == G - 1;
		const int cur = (G - 1 - k) & 1, nxt = cur ^ 1;
		const V* ph = first ? d_phi : P[cur];
		V* po = k > 0 ? P[nxt] : sink;
		V* dpo = tan ? (k > 0 ? D[nxt] : sink + N) : nullptr;
		if ((ret = launch_reverse<double>(rt, tan, first, false, ph, (first || !tan) ? nullptr : D[cur], psi_at(k),
		                                  tan ? dcache + (int64_t)k * N : nullptr, po, dpo, gg[k], zz[k], gw[k], L, ngroups, 0,
		                                  part + (size_t)k * nblk * NPART, nblk)))
			return ret;
	}
	if ((ret = ensure_device(rt.result, result_count(G) * sizeof(double2)))) return ret;
	double2* res = reinterpret_cast<double2*>(rt.result.ptr);
	k_reduce<<<G + 1, 64, 0, rt.stream>>>(part, fpart, G, nblk, tan ? 1 : 0, res);
	rt.launches++;
	if ((ret = RQC_CUDA(cudaGetLastError()))) return ret;
	if ((ret = RQC_CUDA(cudaMemcpyAsync(d_dgates, res + 1, 16 * (size_t)G * sizeof(double2), cudaMemcpyDeviceToDevice,
	                                    rt.stream))))
		return ret;
	if (tan)
		ret = RQC_CUDA(cudaMemcpyAsync(d_hess, res + 1 + 16 * (size_t)G, 16 * (size_t)G * sizeof(double2),
		                               cudaMemcpyDeviceToDevice, rt.stream));
	return ret;
}

}  // namespace rqc
