// Batched evaluation and Riemannian trust-region optimisation of many
// independent brickwall instances (additions beside the reference interface).
// Per instance the arithmetic is the one of the reference's basis-column sums
// (src/target.c:289-436 via src/quantum_circuit.c:147-236), of truncated CG
// (src/trust_region.c:159-217) and of the trust-region loop
// (src/trust_region.c:306-368, src/brickwall_opt.c:107-149).
//
// Evaluation.  One persistent kernel per precision walks a device work queue of
// (instance, column range) items.  A CTA keeps whole basis columns of one
// instance on chip: psi, dpsi, phi and dphi of 2^L x CW amplitudes live in shared
// memory (or, beyond its budget, in a per-CTA global scratch that stays in L2).
// The forward pass applies the gates in place; the reverse pass rebuilds the
// state entering each gate with the adjoint gate (psi_k = G_k^+ psi_{k+1}) instead
// of storing checkpoints, so an evaluation touches HBM only for its gates and
// its partial sums.  Outer-product sums of a brickwall layer build up in
// registers, are reduced across the CTA once per layer and added into FP64
// Kahan accumulators; every item writes its own partial sums, which the post
// kernel adds up in item order (deterministic).  complex64 arithmetic runs on
// packed FP32 FMAs (fma.rn.f32x2), complex128 on FP64 FMAs.
//
// Optimisation.  Every instance carries a trust-region state machine on the
// device; one round evaluates every active instance once (gradient, HVP or f,
// whichever its state needs next), projects, and advances each state machine.
// A round is six launches, captured once as a CUDA graph and replayed.  With
// sharing on, an instance joins only every period-th round, the period growing
// with its cost per evaluation, so that every instance gets a similar share of
// the GPU and small instances finish without waiting on large ones.
#include <math.h>
#include <stdio.h>
#include <string.h>
#include <algorithm>
#include <vector>

#include "engine.h"
#include "manifold.cuh"
#include "rqc_common.cuh"
#include "rqc_runtime.h"
#include "rqcopt_batch.h"
#include "rqcopt_gpu.h"
#include "trust_region.cuh"

namespace rqc {
namespace {

constexpr int BT = 256;          // threads of the evaluation kernel
constexpr int MAXU = 16;         // circuit layers per instance
constexpr int MAXTU = 16;        // target layers per instance
constexpr int MAXL = 14;         // qubits per instance
constexpr int MAXN = 16 * MAXU;  // real parameters per instance
constexpr int NACC = 2 + 64 * MAXU;   // FP64 accumulators per item: f (re, im), dG and HZ per layer
// Work items of an instance: at least ITEM_WORK amplitude x gate updates each (to amortise
// their set-up) and at most MAX_ITEMS per instance; more items let a single instance
// spread over the SMs, which shortens its rounds when few instances are in flight.
constexpr double ITEM_WORK = 262144.0;
constexpr int MAX_ITEMS = 128;
constexpr int TSTR = 20;               // shared-memory stride of a 4x4 gate table (rows padded to 5)
constexpr int NTABS = (MAXU * 3 + MAXTU) * TSTR;
constexpr int SWIRES = (MAXU + MAXTU) * MAXL + 4;   // wire ints in shared memory (16-byte multiple)

enum Phase { PH_GRAD = 0, PH_TCG = 1, PH_HETA = 2, PH_FNEXT = 3, PH_FINAL = 4, PH_DONE = 5, PH_EVAL = 6 };

template <typename T> struct BTr;
template <> struct BTr<float>
{
	using V = float2;
	using E = float4;                // gate entry {re, re, -im, im}
	static constexpr int AMP = 4096; // amplitudes per state tile
};
template <> struct BTr<double>
{
	using V = double2;
	using E = double2;               // gate entry {re, im}
	static constexpr int AMP = 2048;
};

// shared-memory budget of the four state tiles
constexpr size_t STATE_SMEM = 4 * 4096 * sizeof(float2);   // 128 KiB

struct BInst
{
	int L, nl, tnl, per;       // qubits, layers, target layers, gates per layer
	int mode, prec, active;    // current round: EVAL_* mode, PREC_C64 / PREC_C128, participates
	int item0, item1;          // this instance's work items
	int niter, maxiter;        // RTR iterations, tCG iteration limit
	double radius_init, maxradius, rho_trust, abstol, reltol;
	double gtol;               // stop once the gradient norm is at most gtol (0: run niter iterations)
	int period;                // evaluated in rounds r with (r + slot) % period == 0 (cost-weighted sharing)
};

struct BOpt
{
	int phase, iter, tcg_it, boundary, hvp_prec, fprec, refine;
	double fval, fval_im;      // f of the last round
	TcgState tcg;
	RtrState rtr;
};

// per-slot device arrays (capacity slots)
struct Slots
{
	BInst* inst;
	BOpt* opt;
	int* wires;                // [cap][(MAXU + MAXTU) * MAXL] (pairs of each layer)
	double2* x;                // [cap][MAXU][16]
	double2* xn;
	double2* dirs;
	double2* tgt;              // [cap][MAXTU][16] target layer gates (FP64)
	float4* tab32;             // [cap][MAXU * 3 + MAXTU][16]: G, conj G, Z per layer, then target
	double2* tab64;
	double* vec;               // [cap][7][MAXN]: r, d, hd, z, grad, heta, scratch
	double* fiter;             // [cap][maxiter_cap + 1]
	double* evout;             // [cap][2 + 2 MAXN]: f, grad, hvp of an EVAL round
};

__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c)
{
	unsigned long long d;
	const unsigned long long A = *reinterpret_cast<unsigned long long*>(&a);
	const unsigned long long B = *reinterpret_cast<unsigned long long*>(&b);
	const unsigned long long Cc = *reinterpret_cast<unsigned long long*>(&c);
	asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(A), "l"(B), "l"(Cc));
	return *reinterpret_cast<float2*>(&d);
}

// y += e * x (complex)
__device__ __forceinline__ float2 cmac(float2 y, float4 e, float2 x)
{
	y = ffma2(make_float2(e.x, e.y), x, y);
	return ffma2(make_float2(e.z, e.w), make_float2(x.y, x.x), y);
}
__device__ __forceinline__ double2 cmac(double2 y, double2 e, double2 x)
{
	y.x = fma(e.x, x.x, y.x);
	y.x = fma(-e.y, x.y, y.x);
	y.y = fma(e.x, x.y, y.y);
	y.y = fma(e.y, x.x, y.y);
	return y;
}
__device__ __forceinline__ float4 entry_of(float2 v) { return make_float4(v.x, v.x, -v.y, v.y); }
__device__ __forceinline__ double2 entry_of(double2 v) { return v; }
template <typename V> __device__ __forceinline__ V vzero();
template <> __device__ __forceinline__ float2 vzero<float2>() { return make_float2(0.f, 0.f); }
template <> __device__ __forceinline__ double2 vzero<double2>() { return make_double2(0., 0.); }
__device__ __forceinline__ float2 make_v(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double2 make_v(double a, double b) { return make_double2(a, b); }
__device__ __forceinline__ float2 vsub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 vsub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }

__device__ __forceinline__ int ins2(int v, int lo, int hi)
{
	v = ((v >> lo) << (lo + 1)) | (v & ((1 << lo) - 1));
	return ((v >> hi) << (hi + 1)) | (v & ((1 << hi) - 1));
}

__device__ __forceinline__ void kahan_add(double* s, double* c, double v)
{
	const double y = v - *c;
	const double t = *s + y;
	*c = (t - *s) - y;
	*s = t;
}

// ------------------------------------------------------------------ evaluation kernel

// One work item: columns item.y .. item.z - 1 of instance item.x, with the four
// state tiles in shared memory (SMEM) or in this CTA's global scratch.
template <typename T, bool SMEM>
__device__ __forceinline__ void beval_item(const BInst& in, const int4& item, int it, const int* __restrict__ wires,
                                           const typename BTr<T>::E* __restrict__ tabs, double* __restrict__ partial,
                                           typename BTr<T>::V* __restrict__ gscratch, unsigned char* smem)
{
	using V = typename BTr<T>::V;
	using E = typename BTr<T>::E;
	constexpr int NTAB = (MAXU * 3 + MAXTU) * 16;
	E* stab = reinterpret_cast<E*>(smem);
	double* acc = reinterpret_cast<double*>(stab + NTABS);          // [NACC] sums
	double* cmp = acc + NACC;                                        // [NACC] Kahan compensations
	V* red = reinterpret_cast<V*>(cmp + NACC);                       // [BT/32][32]
	double* fred = reinterpret_cast<double*>(red + BT);              // [2][BT/32]
	int* sw = reinterpret_cast<int*>(fred + 2 * (BT / 32));          // [(MAXU + MAXTU) * MAXL] wires
	V* sstates = reinterpret_cast<V*>(sw + SWIRES);
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const int L = in.L, N = 1 << L, nl = in.nl, tnl = in.tnl, per = in.per;
	const int CW = N >= BTr<T>::AMP ? 1 : BTr<T>::AMP >> L;
	const int lcw = __ffs(CW) - 1;
	const int amps = N * CW, ngc = amps >> 2;
	V* base = SMEM ? sstates : gscratch + (size_t)blockIdx.x * 4 * ((size_t)1 << MAXL);
	V* S = base;
	V* dS = base + amps;
	V* P = base + 2 * amps;
	V* dP = base + 3 * amps;
	const int mode = in.mode;
	const bool tan = mode == EVAL_HVP;
	// gate tables with rows padded to 5 entries (rows 2h and 2h + 1 of a thread pair
	// fall in different banks)
	const E* gt = tabs + (size_t)item.x * NTAB;
	for (int e = tid; e < nl * 3 * 16; e += BT) stab[(e >> 4) * TSTR + 5 * ((e >> 2) & 3) + (e & 3)] = gt[e];
	for (int e = tid; e < tnl * 16; e += BT)
		stab[(MAXU * 3 + (e >> 4)) * TSTR + 5 * ((e >> 2) & 3) + (e & 3)] = gt[MAXU * 3 * 16 + e];
	for (int e = tid; e < (MAXU + MAXTU) * MAXL; e += BT) sw[e] = wires[(size_t)item.x * (MAXU + MAXTU) * MAXL + e];
	const int nacc = 2 + 64 * nl;
	for (int e = tid; e < nacc; e += BT) { acc[e] = 0; cmp[e] = 0; }
	const int* w = sw;
	double fx = 0, fy = 0;
	__syncthreads();

	// Group-columns are split over thread pairs: thread h of a pair computes the
	// output rows 2h, 2h + 1 of every product of its group-column.
	const int h = tid & 1, pr = tid >> 1;
	constexpr int NPAIR = BT / 2;
	auto group = [&](int gc, int wi, int wj, int idx[4]) {
		const int c = gc & (CW - 1), g = gc >> lcw;
		const int pi = L - 1 - wi, pj = L - 1 - wj;
		const int b = ins2(g, min(pi, pj), max(pi, pj));
		idx[0] = (b << lcw) | c;
		idx[1] = ((b | (1 << pj)) << lcw) | c;
		idx[2] = ((b | (1 << pi)) << lcw) | c;
		idx[3] = ((b | (1 << pi) | (1 << pj)) << lcw) | c;
	};
	// rows 2h, 2h + 1 of M x (TR: M^T x)
	auto rows2 = [&](const E* m, const V x[4], V y[2], bool tr, bool accum) {
#pragma unroll
		for (int q = 0; q < 2; q++) {
			const int r = 2 * h + q;
			V a2 = accum ? y[q] : vzero<V>();
#pragma unroll
			for (int c = 0; c < 4; c++) a2 = cmac(a2, m[tr ? 5 * c + r : 5 * r + c], x[c]);
			y[q] = a2;
		}
	};
	// full vector from this thread's two rows and the partner's
	auto share = [&](const V own[2], V full[4]) {
		V o0, o1;
		o0.x = __shfl_xor_sync(0xffffffffu, own[0].x, 1);
		o0.y = __shfl_xor_sync(0xffffffffu, own[0].y, 1);
		o1.x = __shfl_xor_sync(0xffffffffu, own[1].x, 1);
		o1.y = __shfl_xor_sync(0xffffffffu, own[1].y, 1);
		full[0] = h ? o0 : own[0];
		full[1] = h ? o1 : own[1];
		full[2] = h ? own[0] : o0;
		full[3] = h ? own[1] : o1;
	};
	// one gate on X (and the tangent dX += Zm X): in place
	auto apply = [&](V* X, V* dX, const E* m, const E* zm, int wi, int wj) {
		for (int gc = pr; gc < ngc; gc += NPAIR) {
			int idx[4];
			group(gc, wi, wj, idx);
			const V x[4] = { X[idx[0]], X[idx[1]], X[idx[2]], X[idx[3]] };
			V y[2], dy[2];
			rows2(m, x, y, false, false);
			if (dX) {
				const V dx[4] = { dX[idx[0]], dX[idx[1]], dX[idx[2]], dX[idx[3]] };
				rows2(m, dx, dy, false, false);
				rows2(zm, x, dy, false, true);
			}
			const int o0 = h ? idx[2] : idx[0], o1 = h ? idx[3] : idx[1];
			__syncwarp();
			X[o0] = y[0];
			X[o1] = y[1];
			if (dX) {
				dX[o0] = dy[0];
				dX[o1] = dy[1];
			}
		}
		__syncthreads();
	};

	for (int b0 = item.y; b0 < item.z; b0 += CW) {
		// phi = -conj(W e_b) for the columns b0 .. b0 + CW - 1
		for (int e = tid; e < amps; e += BT) {
			const int row = e >> lcw, c = e & (CW - 1);
			P[e] = vzero<V>();
			if (row == b0 + c) P[e].x = 1;
		}
		__syncthreads();
		for (int l = 0; l < tnl; l++)
			for (int p = 0; p < per; p++)
				apply(P, nullptr, stab + (MAXU * 3 + l) * TSTR, nullptr, w[(MAXU + l) * MAXL + 2 * p],
				      w[(MAXU + l) * MAXL + 2 * p + 1]);
		for (int e = tid; e < amps; e += BT) {
			const V v = P[e];
			P[e].x = -v.x;
			P[e].y = v.y;
			const int row = e >> lcw, c = e & (CW - 1);
			S[e] = vzero<V>();
			if (row == b0 + c) S[e].x = 1;
			if (tan) dS[e] = vzero<V>();
		}
		__syncthreads();
		// forward: psi <- G psi, dpsi <- G dpsi + Z psi
		for (int l = 0; l < nl; l++)
			for (int p = 0; p < per; p++)
				apply(S, tan ? dS : nullptr, stab + (3 * l) * TSTR, stab + (3 * l + 2) * TSTR, w[l * MAXL + 2 * p],
				      w[l * MAXL + 2 * p + 1]);
		// f contribution: sum phi . psi (unconjugated)
		for (int e = tid; e < amps; e += BT) {
			const V pp = P[e], ss = S[e];
			fx += (double)pp.x * ss.x - (double)pp.y * ss.y;
			fy += (double)pp.x * ss.y + (double)pp.y * ss.x;
		}
		if (mode == EVAL_F) {
			__syncthreads();
			continue;
		}
		if (tan)
			for (int e = tid; e < amps; e += BT) dP[e] = vzero<V>();
		__syncthreads();
		// reverse
		for (int l = nl - 1; l >= 0; l--) {
			const E* G = stab + (3 * l) * TSTR;
			const E* Gc = stab + (3 * l + 1) * TSTR;
			const E* Z = stab + (3 * l + 2) * TSTR;
			// a[0..15]: dG rows 2h, 2h+1 (re, im), a[16..31]: HZ rows 2h, 2h+1
			T a[32];
#pragma unroll
			for (int e = 0; e < 32; e++) a[e] = 0;
			for (int p = per - 1; p >= 0; p--) {
				const int wi = w[l * MAXL + 2 * p], wj = w[l * MAXL + 2 * p + 1];
				for (int gc = pr; gc < ngc; gc += NPAIR) {
					int idx[4];
					group(gc, wi, wj, idx);
					const V x[4] = { S[idx[0]], S[idx[1]], S[idx[2]], S[idx[3]] };
					const V ph[4] = { P[idx[0]], P[idx[1]], P[idx[2]], P[idx[3]] };
					V xo[2], xk[4], np[2];
					rows2(Gc, x, xo, true, false);     // psi_k = G^+ psi_{k+1}
					share(xo, xk);
					rows2(G, ph, np, true, false);     // phi_k = G^T phi_{k+1}
					const int o0 = h ? idx[2] : idx[0], o1 = h ? idx[3] : idx[1];
					E pe[2];
					pe[0] = entry_of(h ? ph[2] : ph[0]);
					pe[1] = entry_of(h ? ph[3] : ph[1]);
#pragma unroll
					for (int q = 0; q < 2; q++)
#pragma unroll
						for (int c = 0; c < 4; c++) {
							V v = make_v(a[2 * (4 * q + c)], a[2 * (4 * q + c) + 1]);
							v = cmac(v, pe[q], xk[c]);
							a[2 * (4 * q + c)] = v.x;
							a[2 * (4 * q + c) + 1] = v.y;
						}
					V dxo[2], ndp[2];
					if (tan) {
						const V dph[4] = { dP[idx[0]], dP[idx[1]], dP[idx[2]], dP[idx[3]] };
						const V dx2[2] = { dS[o0], dS[o1] };
						V zx[2], to[2], t4[4], dxk[4];
						rows2(Z, xk, zx, false, false);
						to[0] = vsub(dx2[0], zx[0]);
						to[1] = vsub(dx2[1], zx[1]);
						share(to, t4);
						rows2(Gc, t4, dxo, true, false);   // dpsi_k = G^+ (dpsi_{k+1} - Z psi_k)
						share(dxo, dxk);
						rows2(G, dph, ndp, true, false);   // dphi_k = G^T dphi_{k+1} + Z^T phi_{k+1}
						rows2(Z, ph, ndp, true, true);
						E dpe[2];
						dpe[0] = entry_of(h ? dph[2] : dph[0]);
						dpe[1] = entry_of(h ? dph[3] : dph[1]);
#pragma unroll
						for (int q = 0; q < 2; q++)
#pragma unroll
							for (int c = 0; c < 4; c++) {
								V v = make_v(a[16 + 2 * (4 * q + c)], a[16 + 2 * (4 * q + c) + 1]);
								v = cmac(v, pe[q], dxk[c]);
								v = cmac(v, dpe[q], xk[c]);
								a[16 + 2 * (4 * q + c)] = v.x;
								a[16 + 2 * (4 * q + c) + 1] = v.y;
							}
					}
					__syncwarp();
					S[o0] = xo[0];
					S[o1] = xo[1];
					P[o0] = np[0];
					P[o1] = np[1];
					if (tan) {
						dS[o0] = dxo[0];
						dS[o1] = dxo[1];
						dP[o0] = ndp[0];
						dP[o1] = ndp[1];
					}
				}
				__syncthreads();
			}
			// layer sums over the 16 lanes of each parity: lane (h, j = lane >> 1) ends with
			// complex entry j of its parity (j < 8: dG[2h + j/4][j%4], else HZ[2h + (j-8)/4][(j-8)%4])
#pragma unroll
			for (int st = 0; st < 4; st++) {
				const int hh = 16 >> st, m = 16 >> st;
				const bool up = (lane & m) != 0;
#pragma unroll
				for (int i2 = 0; i2 < 16; i2++) {
					if (i2 >= hh) break;
					const T send = up ? a[i2] : a[i2 + hh];
					const T keep = up ? a[i2 + hh] : a[i2];
					a[i2] = keep + __shfl_xor_sync(0xffffffffu, send, m);
				}
			}
			red[warp * 32 + lane] = make_v(a[0], a[1]);
			__syncthreads();
			if (tid < 32) {
				const int hp = tid & 1, j = tid >> 1;
				if (tan || j < 8) {
					double sx = 0, sy = 0;
					for (int ww = 0; ww < BT / 32; ww++) {
						sx += (double)red[ww * 32 + tid].x;
						sy += (double)red[ww * 32 + tid].y;
					}
					const int which = j >> 3, r = 2 * hp + ((j & 7) >> 2), c = j & 3, e = 4 * r + c;
					const int off = which == 0 ? 2 + 32 * l + 2 * e : 2 + 32 * nl + 32 * l + 2 * e;
					kahan_add(acc + off, cmp + off, sx);
					kahan_add(acc + off + 1, cmp + off + 1, sy);
				}
			}
			__syncthreads();
		}
	}
	// f of this item
	fx = warp_sum(fx);
	fy = warp_sum(fy);
	if (lane == 0) {
		fred[warp] = fx;
		fred[BT / 32 + warp] = fy;
	}
	__syncthreads();
	if (tid == 0) {
		double sx = 0, sy = 0;
		for (int ww = 0; ww < BT / 32; ww++) {
			sx += fred[ww];
			sy += fred[BT / 32 + ww];
		}
		acc[0] = sx;
		acc[1] = sy;
		cmp[0] = 0;
		cmp[1] = 0;
	}
	__syncthreads();
	double* out = partial + (size_t)it * NACC;
	for (int e = tid; e < nacc; e += BT) out[e] = acc[e] - cmp[e];
	__syncthreads();

}

template <typename T>
__global__ void __launch_bounds__(BT, 1)
k_beval(const BInst* __restrict__ insts, const int4* __restrict__ items, int nitems, int* __restrict__ queue,
        const int* __restrict__ wires, const typename BTr<T>::E* __restrict__ tabs, double* __restrict__ partial,
        typename BTr<T>::V* __restrict__ gscratch, int prec)
{
	using V = typename BTr<T>::V;
	extern __shared__ __align__(16) unsigned char smem[];
	__shared__ int s_item;
	const int tid = threadIdx.x;
	for (;;) {
		if (tid == 0) s_item = atomicAdd(queue, 1);
		__syncthreads();
		const int it = s_item;
		__syncthreads();
		if (it >= nitems) break;
		const int4 item = items[it];
		const BInst in = insts[item.x];
		if (!in.active || in.prec != prec) continue;
		const int N = 1 << in.L;
		const int amps = N * (N >= BTr<T>::AMP ? 1 : BTr<T>::AMP >> in.L);
		if ((size_t)4 * amps * sizeof(V) <= STATE_SMEM)
			beval_item<T, true>(in, item, it, wires, tabs, partial, gscratch, smem);
		else
			beval_item<T, false>(in, item, it, wires, tabs, partial, gscratch, smem);
	}
}

// ------------------------------------------------------------------ prepare / post / advance

__device__ __forceinline__ float4 fmt32(double2 v) { return make_float4((float)v.x, (float)v.x, (float)-v.y, (float)v.y); }

// Start of a round: reset the work queues and the live count, advance the round number.
__global__ void k_bround(int* counters)
{
	counters[0] = 0;   // work queue of the complex64 kernel
	counters[1] = 0;   // work queue of the complex128 kernel
	counters[2] = 0;   // slots not finished at the start of this round
	counters[8]++;     // round number
}

// Per slot: pick the evaluation of this round from the state machine, build the
// gates (and, for HVPs, the tangent directions) and write the gate tables.
__global__ void k_bprepare(Slots s, int* counters)
{
	const int i = blockIdx.x, t = threadIdx.x;
	BInst& in = s.inst[i];
	const BOpt& op = s.opt[i];
	const int ph = op.phase;
	const bool live = in.L > 0 && ph != PH_DONE;
	const bool turn = live && (in.period <= 1 || (counters[8] + i) % in.period == 0);
	__syncthreads();
	if (t == 0) {
		in.active = turn ? 1 : 0;
		if (live) atomicAdd(&counters[2], 1);
	}
	if (!turn) return;
	const int nl = in.nl;
	double* vec = s.vec + (size_t)i * 7 * MAXN;
	double2* x = s.x + (size_t)i * MAXU * 16;
	double2* xn = s.xn + (size_t)i * MAXU * 16;
	double2* dirs = s.dirs + (size_t)i * MAXU * 16;
	int mode = EVAL_F, prec = op.fprec;
	const double2* gates = x;
	const double* dvec = nullptr;
	switch (ph) {
	case PH_GRAD: mode = EVAL_GRAD; break;
	case PH_TCG: mode = EVAL_HVP; prec = op.hvp_prec; dvec = vec + 1 * MAXN; break;
	case PH_HETA: mode = EVAL_HVP; prec = op.hvp_prec; dvec = vec + 3 * MAXN; break;
	case PH_FNEXT: gates = xn; break;
	case PH_EVAL: mode = in.mode; prec = in.prec; break;
	default: break;
	}
	for (int u = t; u < nl; u += blockDim.x) {
		M4 v, z;
		for (int e = 0; e < 16; e++) v.a[e] = x[16 * u + e];
		if (ph == PH_HETA) {   // candidate point (src/trust_region.c:330-331)
			M4 w;
			m4_retract(v, vec + 3 * MAXN + 16 * u, w);
			for (int e = 0; e < 16; e++) xn[16 * u + e] = w.a[e];
		}
		if (dvec) {
			m4_real_to_tangent(dvec + 16 * u, v, z);
			for (int e = 0; e < 16; e++) dirs[16 * u + e] = z.a[e];
		}
	}
	__syncthreads();
	constexpr int NTAB = (MAXU * 3 + MAXTU) * 16;
	float4* t32 = s.tab32 + (size_t)i * NTAB;
	double2* t64 = s.tab64 + (size_t)i * NTAB;
	const double2* tg = s.tgt + (size_t)i * MAXTU * 16;
	for (int e = t; e < nl * 16; e += blockDim.x) {
		const int u = e >> 4, k = e & 15;
		const double2 g = gates[16 * u + k];
		const double2 z = mode == EVAL_HVP ? dirs[16 * u + k] : make_double2(0, 0);
		if (prec == PREC_C64) {
			t32[(3 * u) * 16 + k] = fmt32(g);
			t32[(3 * u + 1) * 16 + k] = fmt32(make_double2(g.x, -g.y));
			t32[(3 * u + 2) * 16 + k] = fmt32(z);
		} else {
			t64[(3 * u) * 16 + k] = g;
			t64[(3 * u + 1) * 16 + k] = make_double2(g.x, -g.y);
			t64[(3 * u + 2) * 16 + k] = z;
		}
	}
	for (int e = t; e < in.tnl * 16; e += blockDim.x) {
		if (prec == PREC_C64) t32[MAXU * 3 * 16 + e] = fmt32(tg[e]);
		else t64[MAXU * 3 * 16 + e] = tg[e];
	}
	if (t == 0) {
		in.mode = mode;
		in.prec = prec;
	}
}

// Per slot and layer: add the items' partial sums in item order and project
// (src/target.c:256-280, 389-436).
__global__ void k_bpost(Slots s, const double* __restrict__ partial)
{
	const int i = blockIdx.x, u = threadIdx.x;
	const BInst in = s.inst[i];
	if (!in.active) return;
	const int nl = in.nl;
	const BOpt& op = s.opt[i];
	if (u == MAXU) {
		double fr = 0, fi = 0, cr = 0, ci = 0;
		for (int it = in.item0; it < in.item1; it++) {
			kahan_add(&fr, &cr, partial[(size_t)it * NACC]);
			kahan_add(&fi, &ci, partial[(size_t)it * NACC + 1]);
		}
		s.opt[i].fval = fr - cr;
		s.opt[i].fval_im = fi - ci;
		if (op.phase == PH_EVAL) {
			s.evout[(size_t)i * (2 + 2 * MAXN)] = fr - cr;
			s.evout[(size_t)i * (2 + 2 * MAXN) + 1] = fi - ci;
		}
		return;
	}
	if (u >= nl || in.mode == EVAL_F) return;
	const bool tan = in.mode == EVAL_HVP;
	M4 dg, hg, g, z;
	for (int e = 0; e < 16; e++) {
		double sr = 0, si = 0, cr = 0, ci = 0, hr = 0, hi = 0, chr = 0, chi = 0;
		for (int it = in.item0; it < in.item1; it++) {
			const double* p = partial + (size_t)it * NACC;
			kahan_add(&sr, &cr, p[2 + 32 * u + 2 * e]);
			kahan_add(&si, &ci, p[2 + 32 * u + 2 * e + 1]);
			if (tan) {
				kahan_add(&hr, &chr, p[2 + 32 * nl + 32 * u + 2 * e]);
				kahan_add(&hi, &chi, p[2 + 32 * nl + 32 * u + 2 * e + 1]);
			}
		}
		dg.a[e] = make_double2(sr - cr, si - ci);
		hg.a[e] = make_double2(hr - chr, hi - chi);
		g.a[e] = s.x[(size_t)i * MAXU * 16 + 16 * u + e];
		z.a[e] = s.dirs[(size_t)i * MAXU * 16 + 16 * u + e];
	}
	double* vec = s.vec + (size_t)i * 7 * MAXN;
	double *gout = vec + 6 * MAXN, *hout = nullptr;
	switch (op.phase) {
	case PH_GRAD: gout = vec + 4 * MAXN; break;
	case PH_TCG: hout = vec + 2 * MAXN; break;
	case PH_HETA: hout = vec + 5 * MAXN; break;
	case PH_EVAL:
		gout = s.evout + (size_t)i * (2 + 2 * MAXN) + 2;
		hout = tan ? gout + MAXN : nullptr;
		break;
	default: break;
	}
	m4_project_grad_hvp(g, tan ? &z : nullptr, dg, tan ? &hg : nullptr, gout + 16 * u, hout ? hout + 16 * u : nullptr);
}

// Per slot: consume the round's result and move the trust-region state machine on
// (src/trust_region.c:159-217, 306-368; the evaluation order of the device optimiser).
__global__ void k_badvance(Slots s, int cap, int fiter_cap, double refine_threshold, int* counters, int* done_ring,
                           int ring_cap)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= cap) return;
	const BInst in = s.inst[i];
	if (!in.active) return;
	BOpt& op = s.opt[i];
	atomicAdd(reinterpret_cast<unsigned long long*>(counters + 4), 1ull);
	if (in.mode == EVAL_HVP) atomicAdd(reinterpret_cast<unsigned long long*>(counters + 6), 1ull);
	const int n = 16 * in.nl;
	double* vec = s.vec + (size_t)i * 7 * MAXN;
	double *r = vec, *d = vec + MAXN, *hd = vec + 2 * MAXN, *z = vec + 3 * MAXN, *grad = vec + 4 * MAXN,
	       *heta = vec + 5 * MAXN;
	double* fiter = s.fiter + (size_t)i * (fiter_cap + 1);
	switch (op.phase) {
	case PH_GRAD:
		op.rtr.fx = op.fval;
		fiter[op.iter] = op.fval;
		tcg_init_dev(n, grad, r, d, z, &op.tcg, op.rtr.radius, in.abstol, in.reltol);
		if (in.gtol > 0 && sqrt(op.tcg.rsq) <= in.gtol) {   // converged: f_iter[iter] is f at the final point
			op.phase = PH_DONE;
			break;
		}
		if (op.refine && op.hvp_prec != PREC_C128 && sqrt(op.tcg.rsq) < refine_threshold) op.hvp_prec = PREC_C128;
		op.tcg_it = 0;
		op.boundary = 0;
		op.phase = in.maxiter > 0 ? PH_TCG : PH_HETA;
		break;
	case PH_TCG:
		tcg_step_dev(n, d, hd, z, r, &op.tcg);
		op.tcg_it++;
		if (op.tcg.status == TCG_BOUNDARY) op.boundary = 1;
		if (op.tcg.status != TCG_CONTINUE || op.tcg_it >= in.maxiter) op.phase = PH_HETA;
		break;
	case PH_HETA: op.phase = PH_FNEXT; break;
	case PH_FNEXT:
		op.rtr.fnext = op.fval;
		rtr_rho_dev(n, grad, z, heta, &op.rtr, op.boundary);
		if (op.rtr.accept) {
			double2* x = s.x + (size_t)i * MAXU * 16;
			const double2* xn = s.xn + (size_t)i * MAXU * 16;
			for (int e = 0; e < 16 * in.nl; e++) x[e] = xn[e];
		}
		op.iter++;
		op.phase = op.iter >= in.niter ? PH_FINAL : PH_GRAD;
		break;
	case PH_FINAL:
		fiter[in.niter] = op.fval;
		op.phase = PH_DONE;
		break;
	case PH_EVAL: op.phase = PH_DONE; break;
	default: break;
	}
	if (op.phase == PH_DONE) {
		const int k = atomicAdd(&counters[3], 1);
		done_ring[k % ring_cap] = i;
	}
}

}  // namespace

// ------------------------------------------------------------------ host side

struct Batch
{
	int cap = 0, fiter_cap = 0;
	Slots d{};
	void* mem = nullptr;
	std::vector<int> used;                 // slot -> 0 free, 1 in use
	std::vector<BInst> hinst;
	std::vector<int4> hitems;
	std::vector<int> hranges;              // (item0, item1) per slot, staged for the device table
	int4* ditems = nullptr;
	size_t items_cap = 0;
	double* partial = nullptr;
	size_t partial_cap = 0;
	float2* gs32 = nullptr;
	double2* gs64 = nullptr;
	int* counters = nullptr;               // [0] queue c64, [1] queue c128, [2] live slots, [3] done count,
	                                       // [4..5] evaluations, [6..7] HVP evaluations (64-bit), [8] round
	int* ring = nullptr;
	int ring_cap = 0;
	int done_read = 0;
	int grid = 0;
	double refine_threshold = 1e-5;
	bool sharing = false;
	cudaGraphExec_t graph = nullptr;
	bool dirty = true;
	size_t smem32 = 0, smem64 = 0;
	long rounds = 0;
};

namespace {

size_t eval_smem(size_t elem)
{
	return NTABS * elem + 2 * NACC * sizeof(double) + BT * 16 + 2 * (BT / 32) * sizeof(double) + SWIRES * sizeof(int) +
	       STATE_SMEM;
}

int batch_init(Runtime& rt, Batch& b, int cap, int fiter_cap)
{
	b.cap = cap;
	b.fiter_cap = fiter_cap;
	constexpr int NTAB = (MAXU * 3 + MAXTU) * 16;
	size_t off = 0;
	auto take = [&](size_t bytes) { const size_t o = off; off += (bytes + 255) & ~(size_t)255; return o; };
	const size_t o_inst = take(sizeof(BInst) * cap), o_opt = take(sizeof(BOpt) * cap),
	             o_w = take(sizeof(int) * cap * (MAXU + MAXTU) * MAXL), o_x = take(sizeof(double2) * cap * MAXU * 16),
	             o_xn = take(sizeof(double2) * cap * MAXU * 16), o_d = take(sizeof(double2) * cap * MAXU * 16),
	             o_t = take(sizeof(double2) * cap * MAXTU * 16), o_t32 = take(sizeof(float4) * cap * NTAB),
	             o_t64 = take(sizeof(double2) * cap * NTAB), o_v = take(sizeof(double) * cap * 7 * MAXN),
	             o_f = take(sizeof(double) * cap * (fiter_cap + 1)), o_e = take(sizeof(double) * cap * (2 + 2 * MAXN)),
	             o_c = take(sizeof(int) * 16), o_r = take(sizeof(int) * cap);
	if (cudaMalloc(&b.mem, off) != cudaSuccess) { cudaGetLastError(); return E_ALLOC; }
	char* m = static_cast<char*>(b.mem);
	b.d.inst = reinterpret_cast<BInst*>(m + o_inst);
	b.d.opt = reinterpret_cast<BOpt*>(m + o_opt);
	b.d.wires = reinterpret_cast<int*>(m + o_w);
	b.d.x = reinterpret_cast<double2*>(m + o_x);
	b.d.xn = reinterpret_cast<double2*>(m + o_xn);
	b.d.dirs = reinterpret_cast<double2*>(m + o_d);
	b.d.tgt = reinterpret_cast<double2*>(m + o_t);
	b.d.tab32 = reinterpret_cast<float4*>(m + o_t32);
	b.d.tab64 = reinterpret_cast<double2*>(m + o_t64);
	b.d.vec = reinterpret_cast<double*>(m + o_v);
	b.d.fiter = reinterpret_cast<double*>(m + o_f);
	b.d.evout = reinterpret_cast<double*>(m + o_e);
	b.counters = reinterpret_cast<int*>(m + o_c);
	b.ring = reinterpret_cast<int*>(m + o_r);
	b.ring_cap = cap;
	int ret = RQC_CUDA(cudaMemsetAsync(b.mem, 0, off, rt.stream));
	if (ret) return ret;
	b.used.assign(cap, 0);
	b.hinst.assign(cap, BInst{});
	b.smem32 = eval_smem(sizeof(float4));
	b.smem64 = eval_smem(sizeof(double2));
	if ((ret = RQC_CUDA(cudaFuncSetAttribute(k_beval<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b.smem32)))) return ret;
	if ((ret = RQC_CUDA(cudaFuncSetAttribute(k_beval<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b.smem64)))) return ret;
	b.grid = rt.num_sms;
	return sync(rt);
}

// columns per on-chip tile of an instance (the complex64 tile; complex128 tiles divide it)
int tile_cols(int L) { return L >= 12 ? 1 : 4096 >> L; }

// Split every live slot's columns into items of similar work, largest first.
int rebuild_items(Runtime& rt, Batch& b)
{
	struct W { double cost; int slot; };
	std::vector<W> live;
	double total = 0;
	for (int i = 0; i < b.cap; i++)
		if (b.used[i]) {
			const BInst& in = b.hinst[i];
			const double per_col = (double)(1 << in.L) * (in.nl + in.tnl) * in.per;
			live.push_back({per_col, i});
			total += per_col * (1 << in.L);
		}
	std::sort(live.begin(), live.end(), [](const W& a, const W& c) { return a.cost > c.cost || (a.cost == c.cost && a.slot < c.slot); });
	// item size from the instance alone, so that its partial sums (and results) do not
	// depend on what else is in the batch
	const double target = ITEM_WORK;
	(void)total;
	b.hitems.clear();
	bool big = false;
	for (const W& wv : live) {
		BInst& in = b.hinst[wv.slot];
		const int N = 1 << in.L, cw = tile_cols(in.L);
		int cols = cw;
		while (cols < N && (N / cols > MAX_ITEMS || (double)cols * wv.cost < target)) cols *= 2;
		in.item0 = (int)b.hitems.size();
		for (int c0 = 0; c0 < N; c0 += cols) b.hitems.push_back(make_int4(wv.slot, c0, std::min(N, c0 + cols), 0));
		in.item1 = (int)b.hitems.size();
		if (in.L >= 12) big = true;
	}
	// item ranges live in the device instance table: one strided copy of (item0, item1)
	// into every slot (free slots get empty ranges)
	b.hranges.assign(2 * (size_t)b.cap, 0);
	for (const W& wv : live) {
		b.hranges[2 * (size_t)wv.slot] = b.hinst[wv.slot].item0;
		b.hranges[2 * (size_t)wv.slot + 1] = b.hinst[wv.slot].item1;
	}
	{
		int ret = RQC_CUDA(cudaMemcpy2DAsync(&b.d.inst[0].item0, sizeof(BInst), b.hranges.data(), 2 * sizeof(int),
		                                     2 * sizeof(int), b.cap, cudaMemcpyHostToDevice, rt.stream));
		if (ret) return ret;
	}
	const size_t ni = std::max<size_t>(b.hitems.size(), 1);
	if (ni > b.items_cap) {
		if (b.ditems) cudaFree(b.ditems);
		if (b.partial) cudaFree(b.partial);
		b.items_cap = ni * 2;
		if (cudaMalloc(&b.ditems, b.items_cap * sizeof(int4)) != cudaSuccess ||
		    cudaMalloc(&b.partial, b.items_cap * NACC * sizeof(double)) != cudaSuccess) {
			cudaGetLastError();
			return E_ALLOC;
		}
	}
	if (!b.hitems.empty()) {
		int ret = RQC_CUDA(cudaMemcpyAsync(b.ditems, b.hitems.data(), b.hitems.size() * sizeof(int4), cudaMemcpyHostToDevice, rt.stream));
		if (ret) return ret;
	}
	if (big && !b.gs32) {
		// per-CTA state tiles beyond the shared-memory budget
		if (cudaMalloc(&b.gs32, (size_t)b.grid * 4 * ((size_t)1 << MAXL) * sizeof(float2)) != cudaSuccess ||
		    cudaMalloc(&b.gs64, (size_t)b.grid * 4 * ((size_t)1 << MAXL) * sizeof(double2)) != cudaSuccess) {
			cudaGetLastError();
			return E_ALLOC;
		}
	}
	b.dirty = true;
	return OK;
}

int launch_round(Runtime& rt, Batch& b)
{
	const int ni = (int)b.hitems.size();
	k_bround<<<1, 1, 0, rt.stream>>>(b.counters);
	k_bprepare<<<b.cap, 64, 0, rt.stream>>>(b.d, b.counters);
	k_beval<float><<<b.grid, BT, b.smem32, rt.stream>>>(b.d.inst, b.ditems, ni, b.counters + 0, b.d.wires, b.d.tab32,
	                                                     b.partial, b.gs32, PREC_C64);
	k_beval<double><<<b.grid, BT, b.smem64, rt.stream>>>(b.d.inst, b.ditems, ni, b.counters + 1, b.d.wires, b.d.tab64,
	                                                      b.partial, b.gs64, PREC_C128);
	k_bpost<<<b.cap, MAXU + 1, 0, rt.stream>>>(b.d, b.partial);
	k_badvance<<<(b.cap + 127) / 128, 128, 0, rt.stream>>>(b.d, b.cap, b.fiter_cap, b.refine_threshold, b.counters,
	                                                        b.ring, b.ring_cap);
	return RQC_CUDA(cudaGetLastError());
}

// Run rounds (a captured graph of one round, replayed) until no slot is active or
// max_rounds have run; returns the number of active slots or < 0.
int run_rounds(Runtime& rt, Batch& b, int max_rounds, int check_every)
{
	int ret;
	if (b.dirty) {
		if (b.graph) { cudaGraphExecDestroy(b.graph); b.graph = nullptr; }
		cudaGraph_t g;
		if ((ret = RQC_CUDA(cudaStreamBeginCapture(rt.stream, cudaStreamCaptureModeThreadLocal)))) return ret;
		ret = launch_round(rt, b);
		cudaError_t e = cudaStreamEndCapture(rt.stream, &g);
		if (ret) return ret;
		if ((ret = RQC_CUDA(e))) return ret;
		ret = RQC_CUDA(cudaGraphInstantiate(&b.graph, g, 0));
		cudaGraphDestroy(g);
		if (ret) return ret;
		b.dirty = false;
	}
	int active = 1;
	for (int r = 0; r < max_rounds; r++) {
		if ((ret = RQC_CUDA(cudaGraphLaunch(b.graph, rt.stream)))) return ret;
		b.rounds++;
		rt.launches += 6;
		if ((r + 1) % check_every == 0 || r + 1 == max_rounds) {
			if ((ret = RQC_CUDA(cudaMemcpyAsync(&active, b.counters + 2, sizeof(int), cudaMemcpyDeviceToHost, rt.stream)))) return ret;
			if ((ret = sync(rt))) return ret;
			if (!active) break;
		}
	}
	return active;
}

// Write one problem into a slot (host arrays -> device) with the given phase.
int load_slot(Runtime& rt, Batch& b, int i, const struct rqcopt_batch_problem* p, const struct rtr_params* params,
              int niter, int precision, int phase, double gtol = 0)
{
	const int L = p->nqubits, nl = p->nlayers, tnl = p->target_nlayers;
	BInst in{};
	in.L = L;
	in.nl = nl;
	in.tnl = tnl;
	in.per = L / 2;
	in.niter = niter;
	const int n = 16 * nl;
	struct rtr_params dp;
	set_rtr_default_params(n, &dp);
	const struct rtr_params* pp = params ? params : &dp;
	in.maxiter = pp->tcg_params.maxiter;
	in.abstol = pp->tcg_params.abstol;
	in.reltol = pp->tcg_params.reltol;
	in.radius_init = pp->radius_init;
	in.maxradius = pp->maxradius;
	in.rho_trust = pp->rho_trust;
	in.prec = precision == PREC_C128 ? PREC_C128 : PREC_C64;
	in.gtol = gtol;
	in.period = 1;
	if (b.sharing) {
		// cost of one evaluation relative to a 10-qubit, 5-layer instance
		const double cost = std::ldexp(1.0, 2 * L) * (nl + tnl) * (L / 2);
		const double ref = std::ldexp(1.0, 20) * 8 * 5;
		in.period = (int)std::min(1024.0, std::max(1.0, std::round(cost / ref)));
	}
	BOpt op{};
	op.phase = phase;
	op.fprec = precision == PREC_C64 ? PREC_C64 : PREC_C128;
	op.hvp_prec = precision == PREC_C128 ? PREC_C128 : PREC_C64;
	op.refine = precision == PREC_MIXED;
	op.rtr.radius = in.radius_init;
	op.rtr.maxradius = in.maxradius;
	op.rtr.rho_trust = in.rho_trust;
	std::vector<int> w((MAXU + MAXTU) * MAXL, 0);
	for (int l = 0; l < nl; l++)
		for (int q = 0; q < L; q++) w[l * MAXL + q] = p->perms[l][q];
	for (int l = 0; l < tnl; l++)
		for (int q = 0; q < L; q++) w[(MAXU + l) * MAXL + q] = p->target_perms[l][q];
	b.hinst[i] = in;
	int ret = RQC_CUDA(cudaMemcpyAsync(&b.d.inst[i], &in, sizeof(in), cudaMemcpyHostToDevice, rt.stream));
	if (!ret) ret = RQC_CUDA(cudaMemcpyAsync(&b.d.opt[i], &op, sizeof(op), cudaMemcpyHostToDevice, rt.stream));
	if (!ret) ret = RQC_CUDA(cudaMemcpyAsync(b.d.wires + (size_t)i * (MAXU + MAXTU) * MAXL, w.data(), w.size() * sizeof(int),
	                                         cudaMemcpyHostToDevice, rt.stream));
	if (!ret) ret = RQC_CUDA(cudaMemcpyAsync(b.d.x + (size_t)i * MAXU * 16, p->vlist, nl * 16 * sizeof(double2),
	                                         cudaMemcpyHostToDevice, rt.stream));
	if (!ret) ret = RQC_CUDA(cudaMemcpyAsync(b.d.tgt + (size_t)i * MAXTU * 16, p->target_vlist, tnl * 16 * sizeof(double2),
	                                         cudaMemcpyHostToDevice, rt.stream));
	return ret;
}

bool problem_ok(const struct rqcopt_batch_problem* p)
{
	if (!p || p->nqubits < 2 || p->nqubits % 2 || p->nqubits > MAXL || p->nlayers < 1 || p->nlayers > MAXU ||
	    p->target_nlayers < 1 || p->target_nlayers > MAXTU || !p->vlist || !p->perms || !p->target_vlist || !p->target_perms)
		return false;
	for (int l = 0; l < p->nlayers; l++) {
		if (!p->perms[l]) return false;
		for (int q = 0; q < p->nqubits; q++)
			if (p->perms[l][q] < 0 || p->perms[l][q] >= p->nqubits) return false;
	}
	for (int l = 0; l < p->target_nlayers; l++) {
		if (!p->target_perms[l]) return false;
		for (int q = 0; q < p->nqubits; q++)
			if (p->target_perms[l][q] < 0 || p->target_perms[l][q] >= p->nqubits) return false;
	}
	return true;
}

void batch_free(Batch* b)
{
	if (!b) return;
	if (b->graph) cudaGraphExecDestroy(b->graph);
	if (b->mem) cudaFree(b->mem);
	if (b->ditems) cudaFree(b->ditems);
	if (b->partial) cudaFree(b->partial);
	if (b->gs32) cudaFree(b->gs32);
	if (b->gs64) cudaFree(b->gs64);
	delete b;
}

}  // namespace
}  // namespace rqc

using namespace rqc;

struct rqcopt_batch
{
	Batch b;
};

extern "C" {

struct rqcopt_batch* rqcopt_batch_create(int capacity, int max_iterations)
{
	Runtime* rt = runtime();
	if (!rt || capacity < 1 || max_iterations < 0) {
		set_last_error(rt ? E_ARG : E_CUDA);
		return nullptr;
	}
	rqcopt_batch* h = new rqcopt_batch;
	int ret = batch_init(*rt, h->b, capacity, max_iterations);
	if (ret) {
		set_last_error(ret);
		batch_free(&h->b);
		return nullptr;
	}
	return h;
}

void rqcopt_batch_destroy(struct rqcopt_batch* h)
{
	if (!h) return;
	Runtime* rt = runtime();
	if (rt) sync(*rt);
	if (h->b.graph) cudaGraphExecDestroy(h->b.graph);
	if (h->b.mem) cudaFree(h->b.mem);
	if (h->b.ditems) cudaFree(h->b.ditems);
	if (h->b.partial) cudaFree(h->b.partial);
	if (h->b.gs32) cudaFree(h->b.gs32);
	if (h->b.gs64) cudaFree(h->b.gs64);
	delete h;
}

int rqcopt_batch_add(struct rqcopt_batch* h, const struct rqcopt_batch_problem* p, const struct rtr_params* params,
                     int niter, int precision, double grad_tol)
{
	Runtime* rt = runtime();
	if (!rt) return E_CUDA;
	if (!h || !problem_ok(p) || niter < 0 || niter > h->b.fiter_cap || precision < PREC_C128 || precision > PREC_C64 ||
	    !(grad_tol >= 0))
		return E_ARG;
	Batch& b = h->b;
	int slot = -1;
	for (int i = 0; i < b.cap; i++)
		if (!b.used[i]) { slot = i; break; }
	if (slot < 0) return E_ALLOC;
	int ret = load_slot(*rt, b, slot, p, params, niter, precision, PH_GRAD, grad_tol);
	if (ret) return ret;
	b.used[slot] = 1;
	if ((ret = rebuild_items(*rt, b))) return ret;
	return slot;
}

int rqcopt_batch_run(struct rqcopt_batch* h, int max_rounds)
{
	Runtime* rt = runtime();
	if (!rt) return E_CUDA;
	if (!h || max_rounds < 1) return E_ARG;
	return run_rounds(*rt, h->b, max_rounds, 8);
}

int rqcopt_batch_finished(struct rqcopt_batch* h, int* slots, int max_slots)
{
	Runtime* rt = runtime();
	if (!rt) return E_CUDA;
	if (!h || (max_slots > 0 && !slots)) return E_ARG;
	Batch& b = h->b;
	int total = 0;
	int ret = RQC_CUDA(cudaMemcpyAsync(&total, b.counters + 3, sizeof(int), cudaMemcpyDeviceToHost, rt->stream));
	if (!ret) ret = sync(*rt);
	if (ret) return ret;
	const int avail = std::min(total - b.done_read, max_slots);
	// the ring range [done_read, done_read + avail), in at most two pieces
	const int start = b.done_read % b.ring_cap;
	const int first = std::min(avail, b.ring_cap - start);
	if (first > 0 &&
	    (ret = RQC_CUDA(cudaMemcpyAsync(slots, b.ring + start, first * sizeof(int), cudaMemcpyDeviceToHost, rt->stream))))
		return ret;
	if (avail > first &&
	    (ret = RQC_CUDA(cudaMemcpyAsync(slots + first, b.ring, (avail - first) * sizeof(int), cudaMemcpyDeviceToHost,
	                                    rt->stream))))
		return ret;
	if ((ret = sync(*rt))) return ret;
	b.done_read += avail;
	return avail;
}

int rqcopt_batch_result(struct rqcopt_batch* h, int slot, double* f_iter, struct mat4x4* vlist_opt, int* iterations)
{
	Runtime* rt = runtime();
	if (!rt) return E_CUDA;
	if (!h || slot < 0 || slot >= h->b.cap || !h->b.used[slot]) return E_ARG;
	Batch& b = h->b;
	BOpt op;
	int ret = RQC_CUDA(cudaMemcpyAsync(&op, &b.d.opt[slot], sizeof(op), cudaMemcpyDeviceToHost, rt->stream));
	if (!ret) ret = sync(*rt);
	if (ret) return ret;
	if (op.phase != PH_DONE) return 0;
	const BInst& in = b.hinst[slot];
	if (iterations) *iterations = op.iter;
	if (f_iter)
		ret = RQC_CUDA(cudaMemcpyAsync(f_iter, b.d.fiter + (size_t)slot * (b.fiter_cap + 1), (in.niter + 1) * sizeof(double),
		                               cudaMemcpyDeviceToHost, rt->stream));
	if (!ret && vlist_opt)
		ret = RQC_CUDA(cudaMemcpyAsync(vlist_opt, b.d.x + (size_t)slot * MAXU * 16, in.nl * 16 * sizeof(double2),
		                               cudaMemcpyDeviceToHost, rt->stream));
	if (!ret) ret = sync(*rt);
	return ret ? ret : 1;
}

int rqcopt_batch_release(struct rqcopt_batch* h, int slot)
{
	Runtime* rt = runtime();
	if (!rt) return E_CUDA;
	if (!h || slot < 0 || slot >= h->b.cap || !h->b.used[slot]) return E_ARG;
	Batch& b = h->b;
	BInst z{};
	int ret = RQC_CUDA(cudaMemcpyAsync(&b.d.inst[slot], &z, sizeof(z), cudaMemcpyHostToDevice, rt->stream));
	if (ret) return ret;
	b.used[slot] = 0;
	b.hinst[slot] = z;
	return rebuild_items(*rt, b);
}

long rqcopt_batch_rounds(const struct rqcopt_batch* h) { return h ? h->b.rounds : 0; }

int rqcopt_batch_set_sharing(struct rqcopt_batch* h, int on)
{
	if (!h) return E_ARG;
	h->b.sharing = on != 0;   // applies to problems added from now on
	return 0;
}

long rqcopt_batch_evaluations(const struct rqcopt_batch* h, long* hvp_evaluations)
{
	Runtime* rt = runtime();
	if (!rt || !h) return E_ARG;
	unsigned long long c[2] = {0, 0};
	if (RQC_CUDA(cudaMemcpyAsync(&c[0], h->b.counters + 4, sizeof(c[0]), cudaMemcpyDeviceToHost, rt->stream)) ||
	    RQC_CUDA(cudaMemcpyAsync(&c[1], h->b.counters + 6, sizeof(c[1]), cudaMemcpyDeviceToHost, rt->stream)) || sync(*rt))
		return E_CUDA;
	if (hvp_evaluations) *hvp_evaluations = (long)c[1];
	return (long)c[0];
}

size_t rqcopt_batch_footprint(int nqubits, int nlayers)
{
	if (nqubits < 2 || nqubits > MAXL || nlayers < 1 || nlayers > MAXU) return 0;
	constexpr int NTAB = (MAXU * 3 + MAXTU) * 16;
	const size_t slot = sizeof(BInst) + sizeof(BOpt) + sizeof(int) * (MAXU + MAXTU) * MAXL + sizeof(double2) * (3 * MAXU + MAXTU) * 16 +
	                    (sizeof(float4) + sizeof(double2)) * NTAB + sizeof(double) * (7 * MAXN + 2 + 2 * MAXN);
	// partial sums of its work items (at most MAX_ITEMS, at most one per tile of columns)
	const size_t cols = (size_t)1 << nqubits;
	const size_t items = std::min<size_t>(MAX_ITEMS, (cols + tile_cols(nqubits) - 1) / tile_cols(nqubits));
	return slot + items * (sizeof(int4) + NACC * sizeof(double));
}

int rqcopt_brickwall_batch_evaluate(const struct rqcopt_batch_problem* problems, int count,
                                    const struct mat4x4* const* vdirs, int mode, int precision, double* f,
                                    double* grad_vec, double* hvp_vec)
{
	Runtime* rt = runtime();
	if (!rt) return E_CUDA;
	if (count < 1 || !problems || mode < EVAL_F || mode > EVAL_HVP || precision < PREC_C128 || precision > PREC_C64 ||
	    (mode == EVAL_HVP && !vdirs))
		return E_ARG;
	for (int k = 0; k < count; k++)
		if (!problem_ok(&problems[k]) || (mode == EVAL_HVP && !vdirs[k])) return E_ARG;
	Batch* b = new Batch;
	int ret = batch_init(*rt, *b, count, 0);
	for (int k = 0; k < count && !ret; k++) {
		ret = load_slot(*rt, *b, k, &problems[k], nullptr, 0, precision, PH_EVAL);
		if (ret) break;
		b->used[k] = 1;
		b->hinst[k].mode = mode;
		b->hinst[k].prec = precision == PREC_C128 ? PREC_C128 : PREC_C64;
		ret = RQC_CUDA(cudaMemcpyAsync(&b->d.inst[k], &b->hinst[k], sizeof(BInst), cudaMemcpyHostToDevice, rt->stream));
		if (!ret && mode == EVAL_HVP)
			ret = RQC_CUDA(cudaMemcpyAsync(b->d.dirs + (size_t)k * MAXU * 16, vdirs[k], problems[k].nlayers * 16 * sizeof(double2),
			                               cudaMemcpyHostToDevice, rt->stream));
	}
	if (!ret) ret = rebuild_items(*rt, *b);
	if (!ret) ret = launch_round(*rt, *b);
	rt->launches += 6;
	std::vector<double> ev((size_t)count * (2 + 2 * MAXN));
	if (!ret) ret = RQC_CUDA(cudaMemcpyAsync(ev.data(), b->d.evout, ev.size() * sizeof(double), cudaMemcpyDeviceToHost, rt->stream));
	if (!ret) ret = sync(*rt);
	if (!ret) {
		size_t go = 0;
		for (int k = 0; k < count; k++) {
			const double* e = ev.data() + (size_t)k * (2 + 2 * MAXN);
			const int n = 16 * problems[k].nlayers;
			if (f) { f[2 * k] = e[0]; f[2 * k + 1] = e[1]; }
			if (grad_vec && mode != EVAL_F) memcpy(grad_vec + go, e + 2, n * sizeof(double));
			if (hvp_vec && mode == EVAL_HVP) memcpy(hvp_vec + go, e + 2 + MAXN, n * sizeof(double));
			go += n;
		}
	}
	batch_free(b);
	return ret;
}

int rqcopt_optimize_brickwall_batch(const struct rqcopt_batch_problem* problems, int count,
                                    const struct rtr_params* params, int niter, int precision, double* f_iter,
                                    struct mat4x4* vlist_opt)
{
	Runtime* rt = runtime();
	if (!rt) return E_CUDA;
	if (count < 1 || !problems || niter < 0 || precision < PREC_C128 || precision > PREC_C64) return E_ARG;
	for (int k = 0; k < count; k++)
		if (!problem_ok(&problems[k])) return E_ARG;
	Batch* b = new Batch;
	int ret = batch_init(*rt, *b, count, niter);
	b->refine_threshold = rt->refine_threshold;
	for (int k = 0; k < count && !ret; k++) {
		ret = load_slot(*rt, *b, k, &problems[k], params ? &params[k] : nullptr, niter, precision, PH_GRAD);
		b->used[k] = 1;
	}
	if (!ret) ret = rebuild_items(*rt, *b);
	while (!ret) {
		const int active = run_rounds(*rt, *b, 64, 16);
		if (active < 0) ret = active;
		if (active <= 0) break;
	}
	size_t xo = 0;
	for (int k = 0; k < count && !ret; k++) {
		if (f_iter)
			ret = RQC_CUDA(cudaMemcpyAsync(f_iter + (size_t)k * (niter + 1), b->d.fiter + (size_t)k * (niter + 1),
			                               (niter + 1) * sizeof(double), cudaMemcpyDeviceToHost, rt->stream));
		if (!ret && vlist_opt)
			ret = RQC_CUDA(cudaMemcpyAsync(vlist_opt + xo, b->d.x + (size_t)k * MAXU * 16, problems[k].nlayers * 16 * sizeof(double2),
			                               cudaMemcpyDeviceToHost, rt->stream));
		xo += problems[k].nlayers;
	}
	if (!ret) ret = sync(*rt);
	batch_free(b);
	return ret;
}

}  // extern "C"
