// Full-Hessian engine (see hess.h).
//
// Per basis column b (or for one given state) let psi_q be the input state of
// sequential gate q and phi_q the cotangent at its output: phi_{G-1} is the
// target column -conj(U e_b) (or the given output cotangent) and
// phi_{q-1} = G_q^T phi_q.  f = phi_{G-1} . psi_G is linear in every gate
// occurrence, so its second derivative in entry x of occurrence q and entry y of
// an earlier occurrence p is
//     sum over the gate group of  phi_q[x_r] * (G_{q-1} ... G_{p+1} E_y psi_p)[x_c]
// with E_y the unit 4x4 gate with entry y = 4 r + c at p's wires.
//
// The engine stores phi_q for all gates (one reverse chain of G^T applications)
// and then sweeps forward once.  For every layer l already reached and every
// entry y it carries one tangent state
//     T_{l,y} = sum over occurrences p of layer l (before the current gate) of
//               G_{q-1} ... G_{p+1} E_y psi_p,
// so the L/2 occurrences of a layer share one state per entry.  At gate q of
// layer a, one kernel launch (k_hsweep) takes every active state s -- psi_q
// itself and the 16 (a + 1) tangents -- contracts it with phi_q (the outer
// product of a gate gradient: 16 complex numbers, summed per layer), then
// carries it through G_q; the tangents of layer a also gain the placeholder
// E_y psi_q.  The contraction of psi_q is the gate gradient; the contraction of
// T_{l,y} at layer a is the Hessian block (a, l) for l < a, and for l = a the
// pairs p < q of the same layer, which the reference symmetrises
// (src/brickwall_circuit.c:229-237).  This replaces the reference's propagation
// of 16 placeholder states per occurrence (src/brickwall_circuit.c:186-224):
// each gate moves 16 (a + 1) + 1 states instead of 16 times the number of
// earlier occurrences.
//
// Sums: each block reduces its 16 complex products per state (warp transpose
// reduction, then over warps) and adds them to its own slot of a partial-sum
// array, [layer][state][32 doubles][block]; the launches of a layer and the
// column chunks add into the same slots in stream order, and one final kernel
// sums the slots over blocks in index order, so results are deterministic.
#include "hess.h"

#include <stdio.h>
#include <string.h>
#include <algorithm>
#include <vector>

#include "manifold.cuh"
#include "rqc_common.cuh"
#include "rqcopt_gpu.h"
#include "sampling.h"
#include "trust_region.cuh"

namespace rqc {

namespace {

constexpr int HT = 256;       // threads per block of the sweep and array kernels
constexpr int HMAXBX = 64;    // blocks per state and launch (partial-sum slots)

// Lane l returns the warp sum of v[l] (31 shuffles for 32 values).
__device__ __forceinline__ double transpose_sum32(double (&v)[32], int lane)
{
#pragma unroll
	for (int o = 16; o >= 1; o >>= 1) {
		const bool up = (lane & o) != 0;
#pragma unroll
		for (int k = 0; k < o; k++) {
			const double send = up ? v[k] : v[k + o];
			const double keep = up ? v[k + o] : v[k];
			v[k] = keep + __shfl_xor_sync(0xffffffffu, send, o);
		}
	}
	return v[0];
}

// Block sum of acc[32] added to out[c * stride], c = 0..31 (one thread per c).
__device__ __forceinline__ void block_add32(double (&acc)[32], double* __restrict__ out, size_t stride, bool add)
{
	__shared__ double red[HT / 32][32];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	red[warp][lane] = transpose_sum32(acc, lane);
	__syncthreads();
	if (threadIdx.x < 32) {
		double s = 0;
#pragma unroll
		for (int k = 0; k < HT / 32; k++) s += red[k][threadIdx.x];
		double* o = out + (size_t)threadIdx.x * stride;
		*o = add ? *o + s : s;
	}
}

// acc[2 (4 r + c) + {0, 1}] += p[r] * x[c]
__device__ __forceinline__ void contract(double (&acc)[32], const double2 p[4], const double2 x[4])
{
#pragma unroll
	for (int r = 0; r < 4; r++)
#pragma unroll
		for (int c = 0; c < 4; c++) {
			acc[2 * (4 * r + c)] = fma(p[r].x, x[c].x, fma(-p[r].y, x[c].y, acc[2 * (4 * r + c)]));
			acc[2 * (4 * r + c) + 1] = fma(p[r].x, x[c].y, fma(p[r].y, x[c].x, acc[2 * (4 * r + c) + 1]));
		}
}

// One gate of the forward sweep (see the file comment).  Block (s, bx): state s
// (0: psi, 1 + t: tangent t of layer t / 16, entry t % 16), column range bx.
//   basis_b0 >= 0: psi_in is the basis column basis_b0 + c of chunk column c
//   fresh:  the tangents of `layer` are zero before this gate
//   carry:  carry the tangents through the gate (0 at the last gate)
//   psi_out: G psi_in, or null where the next input state is given (one-state pass)
//   fpart:  non-null at the last gate of a target sum: f += phi . (G psi)
__global__ void __launch_bounds__(HT, 2)
k_hsweep(const double2* __restrict__ psi_in, int64_t basis_b0, double2* __restrict__ psi_out,
         const double2* __restrict__ phi, double2* __restrict__ tan, Gate4<double> g, WirePair w, int L,
         int64_t ngroups, int64_t sstride, int layer, int fresh, int carry, double* __restrict__ part, int S,
         double2* __restrict__ fpart)
{
	const int s = blockIdx.x, bx = blockIdx.y, nbx = gridDim.y;
	const int t = s - 1;
	const bool own = s > 0 && (t >> 4) == layer;
	const bool zero_in = own && fresh;
	const int er = (t & 15) >> 2, ec = t & 3;   // placeholder entry (row, column)
	double2* __restrict__ T = s > 0 ? tan + (int64_t)t * sstride : nullptr;
	const int lg = L - 2;
	const int64_t gmask = ((int64_t)1 << lg) - 1;
	int64_t off[4];
	group_offsets(w, off);
	double acc[32];
#pragma unroll
	for (int k = 0; k < 32; k++) acc[k] = 0;
	double fx = 0, fy = 0;
	for (int64_t gi = (int64_t)bx * HT + threadIdx.x; gi < ngroups; gi += (int64_t)nbx * HT) {
		const int64_t c = gi >> lg;
		const int64_t loc = group_base(gi & gmask, w);
		const int64_t base = (c << L) + loc;
		double2 p[4], x[4], y[4];
#pragma unroll
		for (int m = 0; m < 4; m++) p[m] = phi[base + off[m]];
		if (s == 0) {
#pragma unroll
			for (int m = 0; m < 4; m++)
				x[m] = basis_b0 >= 0 ? make_double2(loc + off[m] == basis_b0 + c ? 1.0 : 0.0, 0.0) : psi_in[base + off[m]];
		} else if (zero_in) {
#pragma unroll
			for (int m = 0; m < 4; m++) x[m] = make_double2(0, 0);
		} else {
#pragma unroll
			for (int m = 0; m < 4; m++) x[m] = T[base + off[m]];
		}
		if (!zero_in) contract(acc, p, x);
		if (s == 0) {
			// psi_out is null where the input states are given (one-state backward pass)
			if (psi_out || fpart) gate_apply(g, x, y);
			if (psi_out) {
#pragma unroll
				for (int m = 0; m < 4; m++) psi_out[base + off[m]] = y[m];
			}
			if (fpart) {
#pragma unroll
				for (int m = 0; m < 4; m++) {
					fx += p[m].x * y[m].x - p[m].y * y[m].y;
					fy += p[m].x * y[m].y + p[m].y * y[m].x;
				}
			}
		} else if (carry) {
			if (zero_in) {
#pragma unroll
				for (int m = 0; m < 4; m++) y[m] = make_double2(0, 0);
			} else {
				gate_apply(g, x, y);
			}
			if (own) {
				const double2 v = basis_b0 >= 0 ? make_double2(loc + off[ec] == basis_b0 + c ? 1.0 : 0.0, 0.0)
				                                : psi_in[base + off[ec]];
				y[er].x += v.x;
				y[er].y += v.y;
			}
#pragma unroll
			for (int m = 0; m < 4; m++) T[base + off[m]] = y[m];
		}
	}
	const size_t slot = (size_t)layer * S + s;
	block_add32(acc, part + slot * 32 * nbx + bx, nbx, true);
	if (s == 0 && fpart) {
		__shared__ double fr[2][HT / 32];
		fx = warp_sum(fx);
		fy = warp_sum(fy);
		const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
		if (lane == 0) { fr[0][warp] = fx; fr[1][warp] = fy; }
		__syncthreads();
		if (threadIdx.x == 0) {
			double sx = 0, sy = 0;
			for (int k = 0; k < HT / 32; k++) { sx += fr[0][k]; sy += fr[1][k]; }
			fpart[bx].x += sx;
			fpart[bx].y += sy;
		}
	}
}

constexpr int HTILE = 4096;   // amplitudes per shared-memory tile of the layer kernel (64 KB)
constexpr int HMAXPER = 6;    // gates per layer of the layer kernel (L <= 12)

// The wire pairs of one brickwall layer (every position holds the layer gate).
struct LayerGates
{
	WirePair w[HMAXPER];
	int q0, per;
};

// One whole layer of the forward sweep with each tangent's column tiles held in
// shared memory (L <= 12): the gates of a brickwall layer act on disjoint wires,
// so a block loads HTILE amplitudes of a tangent (cb = HTILE / 2^L columns) once,
// runs the layer's L/2 gates on them -- contraction with phi_q, G_q, placeholder --
// and writes them back once; one thread per amplitude group and gate.  Block
// (s, bx): state s as in k_hsweep, column blocks bx, bx + nbx, ...  psi_q comes
// from the forward cache psi + q * sstride, except psi_0 of a basis-column sum
// (basis_b0 >= 0), which is the basis column basis_b0 + c.  The tangents of
// `layer` start at zero (they are created at its first gate).  last: the layer
// holds the circuit's last gate (no G at that gate, no store of the tiles, f
// summed by the psi blocks).
__global__ void __launch_bounds__(HT, 2)
k_hlayer(const double2* __restrict__ psi, int64_t basis_b0, const double2* __restrict__ phi, double2* __restrict__ tan,
         Gate4<double> g, LayerGates lgts, int L, int64_t ncols, int64_t sstride, int layer, int last,
         double* __restrict__ part, int S, double2* __restrict__ fpart)
{
	extern __shared__ double2 tile[];
	__shared__ WirePair sw[HMAXPER];
	if (threadIdx.x < lgts.per) sw[threadIdx.x] = lgts.w[threadIdx.x];
	__syncthreads();
	const int s = blockIdx.x, bx = blockIdx.y, nbx = gridDim.y;
	const int t = s - 1;
	const bool own = s > 0 && (t >> 4) == layer;
	const int er = (t & 15) >> 2, ec = t & 3;
	double2* __restrict__ T = s > 0 ? tan + (int64_t)t * sstride : nullptr;
	const int lg = L - 2;
	const int64_t gmask = ((int64_t)1 << lg) - 1;
	const int cb = HTILE >> L;                               // columns per tile
	const int64_t nblk = (ncols + cb - 1) / cb;
	double acc[32];
#pragma unroll
	for (int k = 0; k < 32; k++) acc[k] = 0;
	double fx = 0, fy = 0;
	for (int64_t blk = bx; blk < nblk; blk += nbx) {
		const int64_t col0 = blk * cb;
		const int cbn = (int)min((int64_t)cb, ncols - col0);
		const int n = cbn << L;                               // amplitudes of this tile
		const int64_t gofs = col0 << L;
		if (s > 0 && !own) {
			for (int e = threadIdx.x; e < n; e += HT) tile[e] = T[gofs + e];
			__syncthreads();
		}
		const int ngr = n >> 2;
		for (int k = 0; k < lgts.per; k++) {
			const int q = lgts.q0 + k;
			const WirePair w = sw[k];
			int64_t off[4];
			group_offsets(w, off);
			const bool final_gate = last && k == lgts.per - 1;
			const double2* __restrict__ ph = phi + (int64_t)q * sstride + gofs;
			const double2* __restrict__ ps = psi + (int64_t)q * sstride + gofs;
			const bool zero_in = own && k == 0;
			const bool basis = q == 0 && basis_b0 >= 0;
			const int64_t offc = ((ec & 2) ? w.si : 0) + ((ec & 1) ? w.sj : 0);
			for (int gi = threadIdx.x; gi < ngr; gi += HT) {
				const int cc = gi >> lg;
				const int64_t loc = group_base(gi & gmask, w);
				const int64_t li = ((int64_t)cc << L) + loc;      // index within the tile
				double2 p[4], x[4];
#pragma unroll
				for (int m = 0; m < 4; m++) p[m] = ph[li + off[m]];
				if (s == 0) {
#pragma unroll
					for (int m = 0; m < 4; m++)
						x[m] = basis ? make_double2(loc + off[m] == basis_b0 + col0 + cc ? 1.0 : 0.0, 0.0) : ps[li + off[m]];
				} else if (zero_in) {
#pragma unroll
					for (int m = 0; m < 4; m++) x[m] = make_double2(0, 0);
				} else {
#pragma unroll
					for (int m = 0; m < 4; m++) x[m] = tile[li + off[m]];
				}
				if (!zero_in) {
#pragma unroll
					for (int r = 0; r < 4; r++)
#pragma unroll
						for (int c = 0; c < 4; c++) {
							acc[2 * (4 * r + c)] = fma(p[r].x, x[c].x, fma(-p[r].y, x[c].y, acc[2 * (4 * r + c)]));
							acc[2 * (4 * r + c) + 1] = fma(p[r].x, x[c].y, fma(p[r].y, x[c].x, acc[2 * (4 * r + c) + 1]));
						}
				}
				if (s == 0) {
					if (final_gate) {
						double2 y[4];
						gate_apply(g, x, y);
#pragma unroll
						for (int m = 0; m < 4; m++) {
							fx += p[m].x * y[m].x - p[m].y * y[m].y;
							fy += p[m].x * y[m].y + p[m].y * y[m].x;
						}
					}
				} else if (!final_gate) {
					double2 y[4];
					if (zero_in) {
#pragma unroll
						for (int m = 0; m < 4; m++) y[m] = make_double2(0, 0);
					} else {
						gate_apply(g, x, y);
					}
					if (own) {
						const double2 v = basis ? make_double2(loc + offc == basis_b0 + col0 + cc ? 1.0 : 0.0, 0.0)
						                        : ps[li + offc];
						y[er].x += v.x;
						y[er].y += v.y;
					}
#pragma unroll
					for (int m = 0; m < 4; m++) tile[li + off[m]] = y[m];
				}
			}
			__syncthreads();
		}
		if (s > 0 && !last) {
			for (int e = threadIdx.x; e < n; e += HT) T[gofs + e] = tile[e];
			__syncthreads();
		}
	}
	const size_t slot = (size_t)layer * S + s;
	block_add32(acc, part + slot * 32 * nbx + bx, nbx, true);
	if (s == 0 && fpart) {
		__shared__ double fr[2][HT / 32];
		fx = warp_sum(fx);
		fy = warp_sum(fy);
		const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
		if (lane == 0) { fr[0][warp] = fx; fr[1][warp] = fy; }
		__syncthreads();
		if (threadIdx.x == 0) {
			double sx = 0, sy = 0;
			for (int k = 0; k < HT / 32; k++) { sx += fr[0][k]; sy += fr[1][k]; }
			fpart[bx].x += sx;
			fpart[bx].y += sy;
		}
	}
}

// ------------------------------------------------------------------ block encoding

// full-register index of half-register basis state b: bit i of b at bit 2 i + 1
// (src/target.c:1148-1157)
__host__ __device__ __forceinline__ int64_t blockenc_index(int64_t b, int half)
{
	int64_t c = 0;
	for (int i = 0; i < half; i++) c |= ((b >> i) & 1) << (2 * i + 1);
	return c;
}

// psi_0 of columns b0 .. b0 + ncols - 1: the basis states P e_b
__global__ void k_benc_init(double2* __restrict__ states, int L, int64_t b0, int64_t ncols)
{
	const int64_t N = (int64_t)1 << L;
	for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ncols * N; i += (int64_t)gridDim.x * blockDim.x) {
		const int64_t c = i >> L, a = i & (N - 1);
		states[i] = make_double2(a == blockenc_index(b0 + c, L / 2) ? 1.0 : 0.0, 0.0);
	}
}

// residual d = P^dag W P e_b - H e_b on the P rows: f += |d|^2 / 2 (per block), chi = P conj(d)
// (zero elsewhere: chi is cleared before).  hneg[b][a] = -conj((H e_b)[a]).
__global__ void k_benc_residual(const double2* __restrict__ wout, const double2* __restrict__ hneg, int L, int64_t b0,
                                int64_t ncols, double2* __restrict__ chi, double2* __restrict__ fpart)
{
	__shared__ double red[HT / 32];
	const int half = L / 2;
	const int64_t s = (int64_t)1 << half;
	double acc = 0;
	for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ncols * s; i += (int64_t)gridDim.x * blockDim.x) {
		const int64_t c = i >> half, a = i & (s - 1);
		const int64_t idx = (c << L) + blockenc_index(a, half);
		const double2 hn = hneg[(b0 + c) * s + a];
		const double2 w = wout[idx];
		const double dx = w.x + hn.x, dy = w.y - hn.y;   // w - H e_b with H e_b = -conj(hn)
		acc += 0.5 * (dx * dx + dy * dy);
		if (chi) chi[idx] = make_double2(dx, -dy);
	}
	acc = warp_sum(acc);
	if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
	__syncthreads();
	if (threadIdx.x == 0) {
		double t = 0;
		for (int k = 0; k < HT / 32; k++) t += red[k];
		fpart[blockIdx.x].x += t;
	}
}

// Jacobian rows on the P rows: jac[t][c * s + a] = tan_t[c][P a]
__global__ void k_benc_gather(const double2* __restrict__ tan, int L, int64_t ncols, int64_t sstride, int m,
                              double2* __restrict__ jac)
{
	const int half = L / 2;
	const int64_t s = (int64_t)1 << half, K = ncols * s;
	for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (int64_t)m * K; i += (int64_t)gridDim.x * blockDim.x) {
		const int64_t t = i / K, r = i % K;
		jac[i] = tan[t * sstride + ((r >> half) << L) + blockenc_index(r & (s - 1), half)];
	}
}

// Gauss-Newton term: part2[(l i), (k j)] += sum_r conj(jac[l i][r]) jac[k j][r] for layer l >= k
// (src/target.c:1570-1580); one block per entry
__global__ void k_benc_gram(const double2* __restrict__ jac, int64_t K, int nl, double2* __restrict__ part2)
{
	__shared__ double red[2][HT / 32];
	const int m = 16 * nl;
	const int e = blockIdx.x;
	const int row = e / m, col = e % m;
	if ((row >> 4) < (col >> 4)) return;
	const double2* __restrict__ x = jac + (int64_t)row * K;
	const double2* __restrict__ y = jac + (int64_t)col * K;
	double sx = 0, sy = 0;
	for (int64_t r = threadIdx.x; r < K; r += HT) {
		const double2 a = x[r], b = y[r];
		sx += a.x * b.x + a.y * b.y;     // conj(a) b
		sy += a.x * b.y - a.y * b.x;
	}
	sx = warp_sum(sx);
	sy = warp_sum(sy);
	if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = sx; red[1][threadIdx.x >> 5] = sy; }
	__syncthreads();
	if (threadIdx.x == 0) {
		double tx = 0, ty = 0;
		for (int k = 0; k < HT / 32; k++) { tx += red[0][k]; ty += red[1][k]; }
		part2[e].x += tx;
		part2[e].y += ty;
	}
}

// hess2 from the lower blocks, upper blocks by conjugate symmetry; f from the residual parts
__global__ void k_benc_finish(const double2* __restrict__ part2, int nl, const double2* __restrict__ fres, int nres,
                              double2* __restrict__ rec, double2* __restrict__ hess2)
{
	const int m = 16 * nl;
	for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (int64_t)m * m; i += (int64_t)gridDim.x * blockDim.x) {
		const int row = (int)(i / m), col = (int)(i % m);
		if (!hess2) break;
		if ((row >> 4) >= (col >> 4)) hess2[i] = part2[i];
		else {
			const double2 v = part2[(int64_t)col * m + row];
			hess2[i] = make_double2(v.x, -v.y);
		}
	}
	if (blockIdx.x == 0 && threadIdx.x == 0) {
		double t = 0;
		for (int k = 0; k < nres; k++) t += fres[k].x;
		rec[0] = make_double2(t, 0.0);
	}
}

// Sum over the blocks of partial slot (slot, entry e)
__device__ __forceinline__ double2 slot_sum(const double* __restrict__ part, int nbx, size_t slot, int e)
{
	const double* re = part + (slot * 32 + 2 * e) * nbx;
	const double* im = re + nbx;
	double sx = 0, sy = 0;
	for (int b = 0; b < nbx; b++) { sx += re[b]; sy += im[b]; }
	return make_double2(sx, sy);
}

// Record: f, per-layer gradients, symmetric complex Hessian (row (a, x), column (b, y)).
__global__ void k_hassemble(const double* __restrict__ part, int nbx, int nl, int S, const double2* __restrict__ fpart,
                            double2* __restrict__ rec)
{
	const int m = 16 * nl;
	const int64_t n = 1 + 16 * (int64_t)nl + (int64_t)m * m;
	for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
		if (i == 0) {
			double sx = 0, sy = 0;
			for (int b = 0; b < nbx; b++) { sx += fpart[b].x; sy += fpart[b].y; }
			rec[0] = make_double2(sx, sy);
		} else if (i <= 16 * nl) {
			const int l = (int)(i - 1) >> 4, e = (int)(i - 1) & 15;
			rec[i] = slot_sum(part, nbx, (size_t)l * S, e);
		} else {
			const int64_t h = i - 1 - 16 * (int64_t)nl;
			const int row = (int)(h / m), col = (int)(h % m);
			const int a = row >> 4, x = row & 15, b = col >> 4, y = col & 15;
			double2 v;
			if (a < b) {
				v = slot_sum(part, nbx, (size_t)b * S + 1 + 16 * a + x, y);
			} else if (a > b) {
				v = slot_sum(part, nbx, (size_t)a * S + 1 + 16 * b + y, x);
			} else {
				const double2 u = slot_sum(part, nbx, (size_t)a * S + 1 + 16 * a + x, y);
				const double2 u2 = slot_sum(part, nbx, (size_t)a * S + 1 + 16 * a + y, x);
				v = make_double2(u.x + u2.x, u.y + u2.y);
			}
			rec[i] = v;
		}
	}
}

// out = G in over `ngroups` groups of consecutive 2^L-amplitude states
//   basis_b0 >= 0: `in` is the basis column basis_b0 + c of column c
__global__ void __launch_bounds__(HT) k_happly(const double2* __restrict__ in, double2* __restrict__ out, Gate4<double> g,
                                               WirePair w, int L, int64_t ngroups, int64_t basis_b0 = -1)
{
	const int lg = L - 2;
	const int64_t gmask = ((int64_t)1 << lg) - 1;
	int64_t off[4];
	group_offsets(w, off);
	for (int64_t gi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; gi < ngroups; gi += (int64_t)gridDim.x * blockDim.x) {
		const int64_t c = gi >> lg, loc = group_base(gi & gmask, w);
		const int64_t base = (c << L) + loc;
		double2 x[4], y[4];
#pragma unroll
		for (int m = 0; m < 4; m++)
			x[m] = basis_b0 >= 0 ? make_double2(loc + off[m] == basis_b0 + c ? 1.0 : 0.0, 0.0) : in[base + off[m]];
		gate_apply(g, x, y);
#pragma unroll
		for (int m = 0; m < 4; m++) out[base + off[m]] = y[m];
	}
}

// Column (b, k) entries of the real Hessian for layers a <= b (src/target.c:937-987), and
// the gradient vector (src/target.c:1025-1030).  rec as written by k_hassemble.
__global__ void k_hproject(int nl, const double2* __restrict__ ug, const double2* __restrict__ rec,
                           const double2* __restrict__ hess2, double* __restrict__ grad, double* __restrict__ H)
{
	const int m = 16 * nl;
	const int npairs = nl * (nl + 1) / 2;
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	const double2* dv = rec + 1;
	const double2* hess = rec + 1 + 16 * nl;
	if (i < nl) {
		M4 v, d;
		for (int e = 0; e < 16; e++) { v.a[e] = ug[16 * i + e]; d.a[e] = c_conj(dv[16 * i + e]); }
		m4_tangent_to_real(v, d, grad + 16 * i);
	}
	if (i >= npairs * 16) return;
	const int k = i & 15;
	int pr = i >> 4, a = 0;
	while (pr >= nl - a) { pr -= nl - a; a++; }
	const int b = a + pr;
	M4 va, vb, z, g;
	for (int e = 0; e < 16; e++) { va.a[e] = ug[16 * a + e]; vb.a[e] = ug[16 * b + e]; }
	double r[16];
	for (int e = 0; e < 16; e++) r[e] = 0;
	r[k] = 1;
	m4_real_to_tangent(r, vb, z);
	for (int x = 0; x < 16; x++) {
		const double2* row = hess + (size_t)(16 * a + x) * m + 16 * b;
		double2 s = c_(0, 0);
		for (int y = 0; y < 16; y++) s = c_add(s, c_mul(row[y], z.a[y]));
		g.a[x] = c_conj(s);
		if (hess2) {   // block encoding: conj(hess1 Z) + hess2 Z (src/target.c:1673-1683)
			const double2* row2 = hess2 + (size_t)(16 * a + x) * m + 16 * b;
			double2 s2 = c_(0, 0);
			for (int y = 0; y < 16; y++) s2 = c_add(s2, c_mul(row2[y], z.a[y]));
			g.a[x] = c_add(g.a[x], s2);
		}
	}
	if (a == b) {
		M4 p, dc, gh, t;
		m4_project_tangent(va, g, p);
		for (int e = 0; e < 16; e++) dc.a[e] = c_conj(dv[16 * a + e]);
		m4_adjoint(dc, gh);
		m4_symmetric_triple(z, gh, va, t);
		for (int e = 0; e < 16; e++) g.a[e] = c_sub(p.a[e], t.a[e]);
	}
	m4_tangent_to_real(va, g, r);
	for (int x = 0; x < 16; x++) H[(size_t)(16 * a + x) * m + 16 * b + k] = r[x];
}

// rec *= scale (the 2^L / nsamples normalisation of the sampling estimator,
// src/target.c:904-915)
__global__ void k_scale_rec(double2* __restrict__ rec, int64_t n, double scale)
{
	for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
		rec[i] = make_double2(rec[i].x * scale, rec[i].y * scale);
}

// lower triangle from the upper one (src/target.c:981-986)
__global__ void k_hmirror(int m, double* __restrict__ H)
{
	const int64_t n = (int64_t)m * m;
	for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
		const int row = (int)(i / m), col = (int)(i % m);
		if (row > col) H[i] = H[(size_t)col * m + row];
	}
}

// Truncated CG with a dense Hessian (src/trust_region.c:83-141): the matrix-vector
// product by rows in parallel, every other step by thread 0 with sequential FP64
// arithmetic (trust_region.cuh).
__global__ void __launch_bounds__(HT) k_tcg_hmat(int n, const double* __restrict__ grad, const double* __restrict__ hess,
                                                 double radius, int maxiter, double abstol, double reltol, double* r,
                                                 double* d, double* hd, double* z, int* status)
{
	__shared__ TcgState st;
	if (threadIdx.x == 0) tcg_init_dev(n, grad, r, d, z, &st, radius, abstol, reltol);
	__syncthreads();
	for (int it = 0; it < maxiter; it++) {
		for (int row = threadIdx.x; row < n; row += blockDim.x) hd[row] = dot_seq(n, hess + (size_t)row * n, d);
		__syncthreads();
		if (threadIdx.x == 0) tcg_step_dev(n, d, hd, z, r, &st);
		__syncthreads();
		if (st.status != TCG_CONTINUE) break;
	}
	if (threadIdx.x == 0) status[0] = st.status == TCG_BOUNDARY ? 1 : 0;
}

__global__ void k_gemv(int n, const double* __restrict__ a, const double* __restrict__ x, double* __restrict__ y)
{
	const int row = blockIdx.x * blockDim.x + threadIdx.x;
	if (row < n) y[row] = dot_seq(n, a + (size_t)row * n, x);
}

// ------------------------------------------------------------------ interleaved arrays

__global__ void __launch_bounds__(HT) k_gate_array(const double2* __restrict__ in, double2* __restrict__ out,
                                                   Gate4<double> g, WirePair w, int ns, int64_t n)
{
	int64_t off[4];
	group_offsets(w, off);
	for (int64_t gi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; gi < n; gi += (int64_t)gridDim.x * blockDim.x) {
		const int64_t s = gi % ns, base = group_base(gi / ns, w);
		double2 x[4], y[4];
#pragma unroll
		for (int m = 0; m < 4; m++) x[m] = in[(base + off[m]) * ns + s];
		gate_apply(g, x, y);
#pragma unroll
		for (int m = 0; m < 4; m++) out[(base + off[m]) * ns + s] = y[m];
	}
}

// block (s, bx): partial sums of dout (x) psi_s over the groups of column range bx
__global__ void __launch_bounds__(HT) k_gate_backward_array(const double2* __restrict__ psi, const double2* __restrict__ dout,
                                                            WirePair w, int ns, int64_t ngroups, double* __restrict__ part)
{
	const int s = blockIdx.x, bx = blockIdx.y, nbx = gridDim.y;
	int64_t off[4];
	group_offsets(w, off);
	double acc[32];
#pragma unroll
	for (int k = 0; k < 32; k++) acc[k] = 0;
	for (int64_t gi = (int64_t)bx * HT + threadIdx.x; gi < ngroups; gi += (int64_t)nbx * HT) {
		const int64_t base = group_base(gi, w);
		double2 p[4], x[4];
#pragma unroll
		for (int m = 0; m < 4; m++) { p[m] = dout[base + off[m]]; x[m] = psi[(base + off[m]) * ns + s]; }
		contract(acc, p, x);
	}
	block_add32(acc, part + (size_t)s * 32 * nbx + bx, nbx, false);
}

__global__ void k_array_sum(const double* __restrict__ part, int ns, int nbx, double2* __restrict__ dgates)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < 16 * ns) dgates[i] = slot_sum(part, nbx, (size_t)(i >> 4), i & 15);
}

__global__ void __launch_bounds__(HT) k_placeholder(const double2* __restrict__ psi, double2* __restrict__ out, WirePair w,
                                                    int64_t ngroups)
{
	int64_t off[4];
	group_offsets(w, off);
	for (int64_t gi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; gi < ngroups; gi += (int64_t)gridDim.x * blockDim.x) {
		const int64_t base = group_base(gi, w);
		double2 x[4];
#pragma unroll
		for (int m = 0; m < 4; m++) x[m] = psi[base + off[m]];
#pragma unroll
		for (int m = 0; m < 4; m++) {
			double2* o = out + (base + off[m]) * 16;
#pragma unroll
			for (int e = 0; e < 16; e++) o[e] = (e >> 2) == m ? x[e & 3] : make_double2(0, 0);
		}
	}
}

// ------------------------------------------------------------------ host helpers

Gate4<double> gate_of(const double2* g, bool transposed)
{
	Gate4<double> r;
	for (int a = 0; a < 4; a++)
		for (int b = 0; b < 4; b++) r.m[4 * a + b] = transposed ? g[4 * b + a] : g[4 * a + b];
	return r;
}

int grid_of(const Runtime& rt, int64_t items, int per_sm)
{
	const int64_t want = (items + HT - 1) / HT;
	return (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)rt.num_sms * per_sm));
}

int checked(Runtime& rt)
{
	rt.launches++;
	return RQC_CUDA(cudaGetLastError());
}

size_t hess_workspace_limit(Runtime& rt)
{
	if (rt.workspace_limit) return rt.workspace_limit;
	size_t free_b = 0, total_b = 0;
	if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
		cudaGetLastError();
		return (size_t)1 << 30;
	}
	return (size_t)((free_b + rt.work.bytes) * 0.75);
}

// blocks per state: enough for four groups per thread, at most HMAXBX
int blocks_per_state(int64_t ngroups)
{
	return (int)std::max<int64_t>(1, std::min<int64_t>(HMAXBX, ngroups / (4 * HT)));
}

struct Sweep
{
	Runtime& rt;
	const HessCircuit& c;
	int L, nl, per, G, S, nbx;
	double* part = nullptr;
	double2* fpart = nullptr;
	std::vector<Gate4<double>> gg, gt;
	std::vector<WirePair> gw;

	bool keep_final = false;   // carry the tangents through the last gate and store them (block encoding)
	bool psi_only = false;     // gradient only: the psi blocks of the sweep

	Sweep(Runtime& r, const HessCircuit& hc) : rt(r), c(hc), L(hc.L), nl(hc.nlayers), per(hc.L / 2),
	                                           G(hc.nlayers * (hc.L / 2)), S(1 + 16 * hc.nlayers), nbx(1) {}

	// blocks per state: by groups for the per-gate kernel, by column tiles for the layer kernel
	int init(int64_t ngroups_per_state, int64_t layer_tiles = 0)
	{
		nbx = layer_tiles > 0 ? (int)std::min<int64_t>(HMAXBX, layer_tiles) : blocks_per_state(ngroups_per_state);
		gg.resize(nl);
		gt.resize(nl);
		for (int l = 0; l < nl; l++) {
			gg[l] = gate_of(c.ugates + 16 * l, false);
			gt[l] = gate_of(c.ugates + 16 * l, true);
		}
		gw.resize(G);
		for (int q = 0; q < G; q++) gw[q] = make_pair_(L, c.wires[2 * q], c.wires[2 * q + 1]);
		const size_t doubles = (size_t)nl * S * 32 * nbx + 2 * (size_t)nbx;
		int ret = ensure_device(rt.partials, doubles * sizeof(double));
		if (ret) return ret;
		part = reinterpret_cast<double*>(rt.partials.ptr);
		fpart = reinterpret_cast<double2*>(part + (size_t)nl * S * 32 * nbx);
		return RQC_CUDA(cudaMemsetAsync(part, 0, doubles * sizeof(double), rt.stream));
	}

	// phi_{q-1} = G_q^T phi_q for q = G-1 .. 1 (phi_at(G-1) given), and optionally the
	// cotangent of the circuit input
	template <typename PhiAt>
	int reverse_chain(PhiAt phi_at, int64_t ngroups, double2* dpsi_in)
	{
		const int grid = grid_of(rt, ngroups, 8);
		for (int q = G - 1; q >= 1; q--) {
			cudaEvent_t ev;
			launch_begin(rt, KC_APPLY, &ev);
			k_happly<<<grid, HT, 0, rt.stream>>>(phi_at(q), phi_at(q - 1), gt[q / per], gw[q], L, ngroups);
			launch_end(rt, KC_APPLY, ev);   // launch_begin counted the launch
			if (int e = RQC_CUDA(cudaGetLastError())) return e;
		}
		if (dpsi_in) {
			k_happly<<<grid, HT, 0, rt.stream>>>(phi_at(0), dpsi_in, gt[0], gw[0], L, ngroups);
			if (int e = checked(rt)) return e;
		}
		return OK;
	}

	// one gate of the forward sweep
	int gate(int q, const double2* psi_in, int64_t basis_b0, double2* psi_out, const double2* phi, double2* tan,
	         int64_t ngroups, int64_t sstride, bool with_f)
	{
		const int a = q / per;
		const bool last = q == G - 1;
		const dim3 grid(psi_only ? 1 : 1 + 16 * (a + 1), nbx);
		cudaEvent_t ev;
		launch_begin(rt, KC_HESS, &ev);
		k_hsweep<<<grid, HT, 0, rt.stream>>>(psi_in, basis_b0, last ? nullptr : psi_out, phi, tan, gg[a], gw[q], L,
		                                     ngroups, sstride, a, q % per == 0 ? 1 : 0, (last && !keep_final) ? 0 : 1, part,
		                                     S, (with_f && last) ? fpart : nullptr);
		launch_end(rt, KC_HESS, ev);
		return RQC_CUDA(cudaGetLastError());
	}

	// psi_q = G_{q-1} psi_{q-1} for q = 1 .. G-1 into psi_at(q); psi_0 the basis columns from basis_b0
	template <typename PsiAt>
	int forward_chain(PsiAt psi_at, int64_t ngroups, int64_t basis_b0)
	{
		const int grid = grid_of(rt, ngroups, 8);
		for (int q = 1; q < G; q++) {
			cudaEvent_t ev;
			launch_begin(rt, KC_APPLY, &ev);
			k_happly<<<grid, HT, 0, rt.stream>>>(psi_at(q - 1), psi_at(q), gg[(q - 1) / per], gw[q - 1], L, ngroups,
			                                     q == 1 ? basis_b0 : -1);
			launch_end(rt, KC_APPLY, ev);
			if (int e = RQC_CUDA(cudaGetLastError())) return e;
		}
		return OK;
	}

	// one layer with shared-memory tiles (L <= 12)
	int layer(int a, const double2* psi, int64_t basis_b0, const double2* phi, double2* tan, int64_t ncols,
	          int64_t sstride, bool with_f)
	{
		static bool smem_set = false;
		if (!smem_set) {
			if (int e = RQC_CUDA(cudaFuncSetAttribute(k_hlayer, cudaFuncAttributeMaxDynamicSharedMemorySize,
			                                          (int)(HTILE * sizeof(double2)))))
				return e;
			smem_set = true;
		}
		LayerGates lgts;
		lgts.q0 = a * per;
		lgts.per = per;
		for (int k = 0; k < per; k++) lgts.w[k] = gw[a * per + k];
		const bool last = a == nl - 1 && !keep_final;
		const dim3 grid(psi_only ? 1 : 1 + 16 * (a + 1), nbx);
		cudaEvent_t ev;
		launch_begin(rt, KC_HESS, &ev);
		k_hlayer<<<grid, HT, HTILE * sizeof(double2), rt.stream>>>(psi, basis_b0, phi, tan, gg[a], lgts, L, ncols, sstride, a,
		                                                             last ? 1 : 0, part, S,
		                                                             (with_f && last) ? fpart : nullptr);
		launch_end(rt, KC_HESS, ev);
		return RQC_CUDA(cudaGetLastError());
	}

	int assemble(double2* d_rec)
	{
		const int m = 16 * nl;
		const int64_t n = 1 + 16 * (int64_t)nl + (int64_t)m * m;
		k_hassemble<<<grid_of(rt, n, 4), HT, 0, rt.stream>>>(part, nbx, nl, S, fpart, d_rec);
		return checked(rt);
	}
};

}  // namespace

// ------------------------------------------------------------------ engine entry points

int hessian_target_device(Runtime& rt, const HessCircuit& c, const TargetSpec& t, double2* d_rec, const SampleSpec* samp)
{
	const int L = c.L, nl = c.nlayers;
	if (L < 2 || L % 2 || nl < 1) return E_ARG;
	if (samp && samp->nsamples < 1) return E_ARG;
	const int per = L / 2, G = nl * per;
	const int64_t N = (int64_t)1 << L;
	const int64_t ncols = samp ? samp->nsamples : N;   // basis columns, or sample states
	// layer kernel (shared-memory tiles) up to L = 12, one kernel per gate beyond
	const bool layered = L <= 12 && per <= HMAXPER;
	// states per column: phi_q of every gate, psi_q of every gate (layered) or two psi
	// buffers, 16 tangents per layer; sampled: the sample states and two target scratch
	// states besides
	const int64_t nstates = G + (layered ? G : 2) + 16 * (int64_t)nl + (samp ? (layered ? 2 : 3) : 0);
	const size_t col_bytes = (size_t)nstates * N * sizeof(double2);
	int64_t C = (int64_t)(hess_workspace_limit(rt) / col_bytes);
	if (rt.column_chunk > 0) C = std::min<int64_t>(C, rt.column_chunk);
	if (t.ufunc) C = std::min<int64_t>(C, std::max<int64_t>(1, ((int64_t)256 << 20) / (N * 16)));
	C = std::min(C, ncols);
	if (C < 1) {
		fprintf(stderr, "rqcopt_gpu: one basis column of the Hessian sweep needs %zu bytes of workspace, more than the limit\n",
		        col_bytes);
		return E_ALLOC;
	}
	int ret = ensure_device(rt.work, (size_t)nstates * C * N * sizeof(double2));
	if (ret) return ret;
	double2* phi = reinterpret_cast<double2*>(rt.work.ptr);
	const int64_t cs = C * N;   // elements per chunk state
	double2* P[2] = { phi + (int64_t)G * cs, phi + (int64_t)(G + 1) * cs };
	double2* psi = phi + (int64_t)G * cs;                              // layered: psi_q at psi + q cs
	double2* tan = phi + (int64_t)(G + (layered ? G : 2)) * cs;
	double2* extra = tan + 16 * (int64_t)nl * cs;                       // sampled: scratch (and states)
	double2* states = samp ? (layered ? psi : extra + 2 * cs) : nullptr;
	double2* tq[2] = { samp ? extra : P[0], samp ? extra + cs : P[1] };   // target scratch
	auto phi_at = [&](int q) { return phi + (int64_t)q * cs; };
	auto psi_at = [&](int q) { return psi + (int64_t)q * cs; };

	Sweep sw(rt, c);
	if ((ret = sw.init(cs / 4, layered ? (C + (HTILE >> L) - 1) / (HTILE >> L) : 0))) return ret;
	for (int64_t b0 = 0; b0 < ncols; b0 += C) {
		const int64_t Cc = std::min(C, ncols - b0);
		const int64_t ngroups = Cc * (N / 4);
		const int64_t basis = samp ? -1 : b0;
		if (samp) {
			if ((ret = haar_states_device(rt, *samp, L, b0, Cc, states))) return ret;
			if ((ret = target_states_device(rt, t, L, states, Cc, phi_at(G - 1), tq[0], tq[1]))) return ret;
		} else if ((ret = target_columns_device(rt, t, L, b0, Cc, phi_at(G - 1), tq[0], tq[1]))) {
			return ret;
		}
		if ((ret = sw.reverse_chain(phi_at, ngroups, nullptr))) return ret;
		if (layered) {
			if ((ret = sw.forward_chain(psi_at, ngroups, basis))) return ret;
			for (int a = 0; a < nl; a++)
				if ((ret = sw.layer(a, psi, basis, phi, tan, Cc, cs, true))) return ret;
			continue;
		}
		for (int q = 0; q < G; q++) {
			const double2* in = q == 0 ? states : P[(q - 1) & 1];
			if ((ret = sw.gate(q, in, q == 0 ? basis : -1, P[q & 1], phi_at(q), tan, ngroups, cs, true))) return ret;
		}
	}
	if ((ret = sw.assemble(d_rec))) return ret;
	if (samp) {
		const int64_t n = (int64_t)hess_record_count(nl);
		k_scale_rec<<<grid_of(rt, n, 4), HT, 0, rt.stream>>>(d_rec, n, (double)N / (double)samp->nsamples);
		ret = checked(rt);
	}
	return ret;
}

int hessian_single_device(Runtime& rt, const HessCircuit& c, const double2* d_cache, const double2* d_dout,
                          double2* d_dpsi, double2* d_rec)
{
	const int L = c.L, nl = c.nlayers;
	if (L < 2 || L % 2 || nl < 1) return E_ARG;
	const int per = L / 2, G = nl * per;
	const int64_t N = (int64_t)1 << L;
	const bool layered = L <= 12 && per <= HMAXPER;
	// phi_0 .. phi_{G-1} (the last a copy of d_dout) and 16 tangents per layer
	const int64_t nstates = G + 16 * (int64_t)nl;
	int ret = ensure_device(rt.work, (size_t)nstates * N * sizeof(double2));
	if (ret) return ret;
	double2* phi = reinterpret_cast<double2*>(rt.work.ptr);
	double2* tan = phi + (int64_t)G * N;
	auto phi_at = [&](int q) { return phi + (int64_t)q * N; };
	if ((ret = RQC_CUDA(cudaMemcpyAsync(phi_at(G - 1), d_dout, N * sizeof(double2), cudaMemcpyDeviceToDevice, rt.stream))))
		return ret;
	Sweep sw(rt, c);
	if ((ret = sw.init(N / 4, layered ? 1 : 0))) return ret;
	if ((ret = sw.reverse_chain(phi_at, N / 4, d_dpsi))) return ret;
	if (layered) {
		for (int a = 0; a < nl; a++)
			if ((ret = sw.layer(a, d_cache, -1, phi, tan, 1, N, false))) return ret;
	} else {
		for (int q = 0; q < G; q++)
			if ((ret = sw.gate(q, d_cache + (int64_t)q * N, -1, nullptr, phi_at(q), tan, N / 4, N, false))) return ret;
	}
	return sw.assemble(d_rec);
}

int blockenc_device(Runtime& rt, const HessCircuit& c, const TargetSpec& t, int mode, double2* d_rec, double2* d_hess2)
{
	const int L = c.L, nl = c.nlayers;
	if (L < 2 || L % 2 || nl < 1 || mode < 0 || mode > 2) return E_ARG;
	const int per = L / 2, G = nl * per, half = L / 2, m = 16 * nl;
	const int64_t N = (int64_t)1 << L, s = (int64_t)1 << half;
	const bool hess = mode == 2;
	const bool layered = L <= 12 && per <= HMAXPER;
	// states per column: phi_q of every gate; psi_q of every gate (layered) or two psi
	// buffers and the input states; W P e_b; the tangents (Hessian only)
	const int64_t nstates = G + (layered ? G : 3) + 1 + (hess ? 16 * (int64_t)nl : 0);
	const size_t col_bytes = (size_t)nstates * N * sizeof(double2);
	int64_t C = (int64_t)(hess_workspace_limit(rt) / col_bytes);
	if (rt.column_chunk > 0) C = std::min<int64_t>(C, rt.column_chunk);
	C = std::min(C, s);
	if (C < 1) return E_ALLOC;
	int ret = ensure_device(rt.work, (size_t)nstates * C * N * sizeof(double2));
	if (ret) return ret;
	double2* phi = reinterpret_cast<double2*>(rt.work.ptr);
	const int64_t cs = C * N;
	double2* P[2] = { phi + (int64_t)G * cs, phi + (int64_t)(G + 1) * cs };
	double2* psi = phi + (int64_t)G * cs;
	double2* states = layered ? psi : phi + (int64_t)(G + 2) * cs;
	double2* wout = phi + (int64_t)(G + (layered ? G : 3)) * cs;
	double2* tan = wout + cs;
	auto phi_at = [&](int q) { return phi + (int64_t)q * cs; };
	auto psi_at = [&](int q) { return psi + (int64_t)q * cs; };
	// per evaluation: -conj(H e_b) for all b, target scratch, Jacobian rows, Gauss-Newton parts, f parts
	const int nres = rt.num_sms * 2;
	const size_t abytes = (3 * (size_t)s * s + (hess ? (size_t)m * C * s + (size_t)m * m : 0) + nres) * sizeof(double2);
	if ((ret = ensure_device(rt.arrays, abytes))) return ret;
	double2* hneg = static_cast<double2*>(rt.arrays.ptr);
	double2* sc0 = hneg + s * s;
	double2* sc1 = sc0 + s * s;
	double2* jac = sc1 + s * s;
	double2* part2 = hess ? jac + (size_t)m * C * s : jac;
	double2* fres = hess ? part2 + (size_t)m * m : jac;
	if ((ret = RQC_CUDA(cudaMemsetAsync(fres, 0, nres * sizeof(double2), rt.stream)))) return ret;
	if (hess && (ret = RQC_CUDA(cudaMemsetAsync(part2, 0, (size_t)m * m * sizeof(double2), rt.stream)))) return ret;
	if ((ret = target_columns_device(rt, t, half, 0, s, hneg, sc0, sc1))) return ret;

	Sweep sw(rt, c);
	sw.keep_final = hess;
	sw.psi_only = mode == 1;
	if (mode >= 1 && (ret = sw.init(cs / 4, layered ? (C + (HTILE >> L) - 1) / (HTILE >> L) : 0))) return ret;
	if (mode == 0) {   // the gates and wires of the forward passes
		sw.gg.resize(nl);
		for (int l = 0; l < nl; l++) sw.gg[l] = gate_of(c.ugates + 16 * l, false);
		sw.gw.resize(G);
		for (int q = 0; q < G; q++) sw.gw[q] = make_pair_(L, c.wires[2 * q], c.wires[2 * q + 1]);
	}
	for (int64_t b0 = 0; b0 < s; b0 += C) {
		const int64_t Cc = std::min(C, s - b0);
		const int64_t ngroups = Cc * (N / 4);
		const int agrid = grid_of(rt, ngroups, 8);
		k_benc_init<<<grid_of(rt, Cc * N, 8), HT, 0, rt.stream>>>(states, L, b0, Cc);
		if ((ret = checked(rt))) return ret;
		// forward pass to W P e_b
		if (layered && mode >= 1) {
			if ((ret = sw.forward_chain(psi_at, ngroups, -1))) return ret;
			k_happly<<<agrid, HT, 0, rt.stream>>>(psi_at(G - 1), wout, sw.gg[(G - 1) / per], sw.gw[G - 1], L, ngroups);
			if ((ret = checked(rt))) return ret;
		} else {
			const double2* in = states;
			for (int q = 0; q < G; q++) {
				double2* o = q == G - 1 ? wout : P[q & 1];
				k_happly<<<agrid, HT, 0, rt.stream>>>(in, o, sw.gg[q / per], sw.gw[q], L, ngroups);
				if ((ret = checked(rt))) return ret;
				in = o;
			}
		}
		double2* chi = mode >= 1 ? phi_at(G - 1) : nullptr;
		if (chi && (ret = RQC_CUDA(cudaMemsetAsync(chi, 0, (size_t)Cc * N * sizeof(double2), rt.stream)))) return ret;
		k_benc_residual<<<nres, HT, 0, rt.stream>>>(wout, hneg, L, b0, Cc, chi, fres);
		if ((ret = checked(rt))) return ret;
		if (mode == 0) continue;
		if ((ret = sw.reverse_chain(phi_at, ngroups, nullptr))) return ret;
		if (layered) {
			for (int a = 0; a < nl; a++)
				if ((ret = sw.layer(a, psi, -1, phi, tan, Cc, cs, false))) return ret;
		} else {
			for (int q = 0; q < G; q++) {
				const double2* in = q == 0 ? states : P[(q - 1) & 1];
				if ((ret = sw.gate(q, in, -1, P[q & 1], phi_at(q), tan, ngroups, cs, false))) return ret;
			}
		}
		if (hess) {
			k_benc_gather<<<grid_of(rt, (int64_t)m * Cc * s, 8), HT, 0, rt.stream>>>(tan, L, Cc, cs, m, jac);
			if ((ret = checked(rt))) return ret;
			k_benc_gram<<<m * m, HT, 0, rt.stream>>>(jac, Cc * s, nl, part2);
			if ((ret = checked(rt))) return ret;
		}
	}
	if (mode >= 1 && (ret = sw.assemble(d_rec))) return ret;
	k_benc_finish<<<grid_of(rt, (int64_t)m * m, 4), HT, 0, rt.stream>>>(part2, nl, fres, nres, d_rec,
	                                                                     hess ? d_hess2 : nullptr);
	return checked(rt);
}

int project_hessian_device(Runtime& rt, int nlayers, const double2* d_ugates, const double2* d_rec, double* d_grad,
                           double* d_H, const double2* d_hess2)
{
	const int m = 16 * nlayers;
	const int n = std::max(nlayers, 16 * nlayers * (nlayers + 1) / 2);
	k_hproject<<<(n + 63) / 64, 64, 0, rt.stream>>>(nlayers, d_ugates, d_rec, d_hess2, d_grad, d_H);
	int ret = checked(rt);
	if (ret) return ret;
	k_hmirror<<<grid_of(rt, (int64_t)m * m, 4), HT, 0, rt.stream>>>(m, d_H);
	return checked(rt);
}

int tcg_hmat_device(Runtime& rt, int n, const double* d_grad, const double* d_hess, double radius, int maxiter,
                    double abstol, double reltol, double* d_work, double* d_z, int* d_status)
{
	k_tcg_hmat<<<1, HT, 0, rt.stream>>>(n, d_grad, d_hess, radius, maxiter, abstol, reltol, d_work, d_work + n,
	                                    d_work + 2 * n, d_z, d_status);
	return checked(rt);
}

int gemv_device(Runtime& rt, int n, const double* d_a, const double* d_x, double* d_y)
{
	k_gemv<<<(n + 127) / 128, 128, 0, rt.stream>>>(n, d_a, d_x, d_y);
	return checked(rt);
}

int gate_to_array_device(Runtime& rt, int L, int ns, const double2* gate, int i, int j, const double2* d_in,
                         double2* d_out)
{
	const int64_t n = ((int64_t)1 << (L - 2)) * ns;
	k_gate_array<<<grid_of(rt, n, 8), HT, 0, rt.stream>>>(d_in, d_out, gate_of(gate, false), make_pair_(L, i, j), ns, n);
	return checked(rt);
}

int gate_backward_array_device(Runtime& rt, int L, int ns, int i, int j, const double2* d_psi, const double2* d_dout,
                               double2* d_dgates)
{
	const int64_t ngroups = (int64_t)1 << (L - 2);
	const int nbx = blocks_per_state(ngroups);
	int ret = ensure_device(rt.partials, (size_t)ns * 32 * nbx * sizeof(double));
	if (ret) return ret;
	double* part = reinterpret_cast<double*>(rt.partials.ptr);
	k_gate_backward_array<<<dim3(ns, nbx), HT, 0, rt.stream>>>(d_psi, d_dout, make_pair_(L, i, j), ns, ngroups, part);
	if ((ret = checked(rt))) return ret;
	k_array_sum<<<(16 * ns + 127) / 128, 128, 0, rt.stream>>>(part, ns, nbx, d_dgates);
	return checked(rt);
}

int gate_placeholder_device(Runtime& rt, int L, int i, int j, const double2* d_psi, double2* d_out)
{
	const int64_t ngroups = (int64_t)1 << (L - 2);
	k_placeholder<<<grid_of(rt, ngroups, 8), HT, 0, rt.stream>>>(d_psi, d_out, make_pair_(L, i, j), ngroups);
	return checked(rt);
}

}  // namespace rqc
