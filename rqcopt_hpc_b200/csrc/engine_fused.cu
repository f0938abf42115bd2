// Fused basis-column evaluation engine: the gates of a circuit are grouped into
// passes of up to four consecutive gates acting on at most eight qubits (for
// the periodic brickwall a pass is one half of a layer), and each pass is one
// HBM round trip over a column chunk.
//
// Layout: a chunk of C basis columns is stored column-interleaved, [2^L][C]
// (amplitude row a, column j at a*C + j), so that a tile over ANY eight qubits
// -- 256 rows -- reads and writes contiguous runs of CW columns (CW*sizeof =
// 64 B) per row, whatever the qubits' positions.
//
// Per pass (gates g_0..g_{K-1} of the pass, directions z_k):
//   forward  : psi, dpsi (pass input) -> pass output, in shared memory,
//              dpsi <- g dpsi + z psi, psi <- g psi for each gate;
//              only the pass-boundary states are stored (checkpoints);
//   reverse  : from the checkpoint (psi, dpsi at the pass input) the K-1
//              intermediate states are recomputed in shared memory, then for
//              k = K-1..0, with phi, dphi the adjoint at the output of gate k:
//                dG_k += phi (x) psi_k,   HZ_k += phi (x) dpsi_k + dphi (x) psi_k,
//                dphi <- g_k^T dphi + z_k^T phi,  phi <- g_k^T phi;
//              only phi, dphi at the pass input are stored.
// Inside a gate step four threads share an amplitude group (4 amplitudes);
// thread q owns gate row q of the outer products and output component q, so
// each thread keeps 8 complex accumulators per gate of the pass in registers.
//
// These are the same per-column recurrences as the per-gate engine (the
// scheme of src/quantum_circuit.c:147-236), evaluated in a different order of
// memory traffic; results agree to rounding.
#include <stdio.h>
#include <string.h>
#include <algorithm>
#include <type_traits>
#include <vector>

#include "engine.h"
#include "engine_fused.h"
#include "rqc_common.cuh"
#include "rqcopt_gpu.h"

namespace rqc {

namespace {

constexpr int TPB2 = 256;
constexpr int MAXK = 4;
constexpr int MAXNB = 8;
constexpr int NPART2 = 64;
constexpr int EPT = (1 << MAXNB) * 4 / TPB2;   // complex128 tile elements per thread (4 columns per row)

template <typename T> struct ColsPer;
template <> struct ColsPer<double> { static constexpr int v = 4; };   // 4 x 16 B = 64 B runs
template <> struct ColsPer<float>  { static constexpr int v = 8; };   // 8 x 8 B  = 64 B runs

// Geometry of one pass over one chunk (kernel argument).
struct PassGeom
{
	int K;                 // gates in the pass
	int NB;                // tile bits (rows per tile = 2^NB)
	int L;
	int tbit[MAXNB];       // state row bit of tile bit b
	int gi[MAXK], gj[MAXK];// tile-local bits of wire i / wire j of each gate
	int64_t C;             // allocated columns of the chunk (row pitch)
	int64_t ncg;           // column groups of CW columns covering the valid columns
	int64_t ntiles;        // row tiles (2^(L-NB)) x column groups
	int64_t b0;            // basis index of the chunk's first column
	uint32_t rest_mask;    // state row bits that are not tile bits
};

// Paired basis columns (real-orthogonal problems): with c_pair_half = N/2 the column
// with basis index b (< N/2) is e_b + i e_{b + N/2}; 0 selects plain basis columns.
__constant__ int64_t c_pair_half = 0;
// End of the column range of the current evaluation: the columns of a chunk's last
// column group at or beyond it are zero (they add nothing to any sum).
__constant__ int64_t c_col_end = INT64_MAX;

__device__ __forceinline__ float basis_re(int64_t row, int64_t b) { return (row == b && b < c_col_end) ? 1.f : 0.f; }
__device__ __forceinline__ float basis_im(int64_t row, int64_t b)
{
	return (c_pair_half != 0 && b < c_col_end && row == b + c_pair_half) ? 1.f : 0.f;
}

template <typename T> struct PassGates { Gate4<T> g[MAXK]; Gate4<T> z[MAXK]; };
// W_k = G_k^+ Z_k G_k^+ of each gate of a pass (adjoint reconstruction of the tangent state)
template <typename T> struct PassW { Gate4<T> w[MAXK]; };

// deposit the bits of v into the positions set in mask (ascending)
__device__ __forceinline__ int64_t deposit(int64_t v, uint32_t mask)
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
__device__ __forceinline__ void gates_to_smem(const PassGates<T>& pg, int K, bool tan, cplx<T>* sg)
{
	for (int e = threadIdx.x; e < 32 * MAXK; e += blockDim.x) {
		const int k = e / 32, w = e % 32;
		if (k >= K) continue;
		sg[e] = w < 16 ? pg.g[k].m[w] : (tan ? pg.z[k].m[w - 16] : czero<cplx<T>>());
	}
}

__device__ __forceinline__ void row_offsets(const PassGeom& pg, int* rowoff)
{
	const int R = 1 << pg.NB;
	for (int r = threadIdx.x; r < R; r += blockDim.x) {
		int o = 0;
		for (int b = 0; b < pg.NB; b++)
			if ((r >> b) & 1) o |= 1 << pg.tbit[b];
		rowoff[r] = o;
	}
}

// rows of the 4 group members for gate bits (bi, bj) and group base b6
__device__ __forceinline__ void group_rows(int b6, int bi, int bj, int rows[4])
{
	const int lo = bi < bj ? bi : bj, hi = bi < bj ? bj : bi;
	int r = b6;
	r = ((r >> lo) << (lo + 1)) | (r & ((1 << lo) - 1));
	r = ((r >> hi) << (hi + 1)) | (r & ((1 << hi) - 1));
	rows[0] = r;
	rows[1] = r | (1 << bj);
	rows[2] = r | (1 << bi);
	rows[3] = r | (1 << bi) | (1 << bj);
}

template <typename T>
__device__ __forceinline__ cplx<T> sel4(const cplx<T> v[4], int q)
{
	return q == 0 ? v[0] : q == 1 ? v[1] : q == 2 ? v[2] : v[3];
}

__device__ __forceinline__ int sel4_int(const int v[4], int q)
{
	return q == 0 ? v[0] : q == 1 ? v[1] : q == 2 ? v[2] : v[3];
}

// ------------------------------------------------------------------------------ forward kernel

// One pass forward over tiles.  IN: 0 read psi/dpsi, 1 basis columns (dpsi = 0).
// OUT: 0 store psi/dpsi, 1 store -conj(psi) (no tangent), 2 f += <phi, psi> (no store).
template <typename T, bool TAN, int IN, int OUT>
__global__ void __launch_bounds__(TPB2) k2_fwd(const cplx<T>* __restrict__ psi, const cplx<T>* __restrict__ dpsi,
                                               cplx<T>* __restrict__ psi_o, cplx<T>* __restrict__ dpsi_o,
                                               const cplx<T>* __restrict__ phi, PassGeom pg, PassGates<T> gates,
                                               double2* __restrict__ fpart)
{
	using V = cplx<T>;
	constexpr int CW = ColsPer<T>::v;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int R = 1 << pg.NB, A = R * CW;
	V* sg = reinterpret_cast<V*>(smem_raw);                       // 32 * MAXK gate entries
	int* rowoff = reinterpret_cast<int*>(sg + 32 * MAXK);          // R
	V* S = reinterpret_cast<V*>(rowoff + (1 << MAXNB));            // psi tile [R][CW]
	V* dS = S + A;                                                 // dpsi tile
	gates_to_smem<T>(gates, pg.K, TAN, sg);
	row_offsets(pg, rowoff);
	const int64_t rtiles = (int64_t)1 << (pg.L - pg.NB);
	double fx = 0, fy = 0;
	__syncthreads();

	for (int64_t tile = blockIdx.x; tile < pg.ntiles; tile += gridDim.x) {
		const int64_t rt = tile / pg.ncg, cg = tile - rt * pg.ncg;
		(void)rtiles;
		const int64_t rowbase = deposit(rt, pg.rest_mask);
		const int64_t colbase = cg * CW;
		// load
		for (int e = threadIdx.x; e < A; e += blockDim.x) {
			const int r = e / CW, cc = e - r * CW;
			const int64_t row = rowbase + rowoff[r];
			const int64_t col = colbase + cc;
			if (IN == 0) {
				const int64_t a = row * pg.C + col;
				S[e] = psi[a];
				if (TAN) dS[e] = dpsi[a];
			} else {
				S[e] = mk<T>(T(basis_re(row, pg.b0 + col)), T(basis_im(row, pg.b0 + col)));
				if (TAN) dS[e] = czero<V>();
			}
		}
		__syncthreads();
		// gate steps
		for (int k = 0; k < pg.K; k++) {
			const V* gk = sg + 32 * k;
			const int bi = pg.gi[k], bj = pg.gj[k];
			for (int base = 0; base < A; base += blockDim.x) {
				const int task = base + threadIdx.x;
				const bool active = task < A;
				const int g = task >> 2, q = task & 3;
				const int cc = g % CW, b6 = g / CW;
				int rows[4];
				group_rows(b6, bi, bj, rows);
				V x[4], dx[4], y = czero<V>(), dy = czero<V>();
				if (active) {
#pragma unroll
					for (int m = 0; m < 4; m++) {
						x[m] = S[rows[m] * CW + cc];
						if (TAN) dx[m] = dS[rows[m] * CW + cc];
					}
#pragma unroll
					for (int m = 0; m < 4; m++) {
						y = cfma(gk[4 * q + m], x[m], y);
						if (TAN) {
							dy = cfma(gk[4 * q + m], dx[m], dy);
							dy = cfma(gk[16 + 4 * q + m], x[m], dy);
						}
					}
				}
				__syncwarp();
				if (active) {
					const int r = sel4_int(rows, q);
					S[r * CW + cc] = y;
					if (TAN) dS[r * CW + cc] = dy;
				}
			}
			__syncthreads();
		}
		// store / reduce
		for (int e = threadIdx.x; e < A; e += blockDim.x) {
			const int r = e / CW, cc = e - r * CW;
			const int64_t a = (rowbase + rowoff[r]) * pg.C + colbase + cc;
			if (OUT == 2) {
				const V p = phi[a];
				const V s = S[e];
				fx += (double)p.x * s.x - (double)p.y * s.y;
				fy += (double)p.x * s.y + (double)p.y * s.x;
			} else if (OUT == 1) {
				psi_o[a] = cneg_conj(S[e]);
			} else {
				psi_o[a] = S[e];
				if (TAN) dpsi_o[a] = dS[e];
			}
		}
		__syncthreads();
	}
	if (OUT == 2) {
		__shared__ double red[2][TPB2 / 32];
		fx = warp_sum(fx);
		fy = warp_sum(fy);
		const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
		if (lane == 0) { red[0][warp] = fx; red[1][warp] = fy; }
		__syncthreads();
		if (threadIdx.x == 0) {
			double sx = 0, sy = 0;
			for (int w = 0; w < TPB2 / 32; w++) { sx += red[0][w]; sy += red[1][w]; }
			fpart[blockIdx.x].x += sx;
			fpart[blockIdx.x].y += sy;
		}
	}
}

// ------------------------------------------------------------------------------ reverse kernel

// One pass in reverse over tiles.  FIRST: the pass ends the circuit (dphi = 0).
// LAST: the pass starts the circuit (psi is the basis column, dpsi = 0, no outputs).
// part: per-gate partial sums of the pass, gate k at part + k * nblk * 64, block b at + b * 64.
template <typename T, bool TAN, bool FIRST, bool LAST>
__global__ void __launch_bounds__(TPB2, 1) k2_rev(const cplx<T>* __restrict__ psi, const cplx<T>* __restrict__ dpsi,
                                                  const cplx<T>* __restrict__ phi, const cplx<T>* __restrict__ dphi,
                                                  cplx<T>* __restrict__ phi_o, cplx<T>* __restrict__ dphi_o,
                                                  PassGeom pg, PassGates<T> gates, double* __restrict__ part, int nblk)
{
	using V = cplx<T>;
	constexpr int CW = ColsPer<T>::v;
	constexpr bool FLUSH = sizeof(T) == 4;
	constexpr int RUN = 4;
	constexpr int NV = TAN ? 16 : 8;   // accumulator reals per gate: row q of dG (and of HZ)
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int R = 1 << pg.NB, A = R * CW, K = pg.K;
	V* sg = reinterpret_cast<V*>(smem_raw);
	int* rowoff = reinterpret_cast<int*>(sg + 32 * MAXK);
	V* tiles = reinterpret_cast<V*>(rowoff + (1 << MAXNB));
	V* Psi = tiles;                               // K tiles: state entering gate k
	V* dPsi = TAN ? tiles + K * A : nullptr;      // K tiles
	V* Phi = tiles + (TAN ? 2 * K : K) * A;       // adjoint
	V* dPhi = TAN ? Phi + A : nullptr;
	gates_to_smem<T>(gates, K, TAN, sg);
	row_offsets(pg, rowoff);
	const int q = threadIdx.x & 3;

	T acc[MAXK][NV];
	double accd[MAXK][FLUSH ? NV : 1];
#pragma unroll
	for (int k = 0; k < MAXK; k++)
#pragma unroll
		for (int v = 0; v < NV; v++) {
			acc[k][v] = 0;
			if (FLUSH) accd[k][v] = 0;
		}
	int run = 0;
	__syncthreads();

	for (int64_t tile = blockIdx.x; tile < pg.ntiles; tile += gridDim.x) {
		const int64_t rt = tile / pg.ncg, cg = tile - rt * pg.ncg;
		const int64_t rowbase = deposit(rt, pg.rest_mask);
		const int64_t colbase = cg * CW;
		for (int e = threadIdx.x; e < A; e += blockDim.x) {
			const int r = e / CW, cc = e - r * CW;
			const int64_t row = rowbase + rowoff[r], col = colbase + cc;
			const int64_t a = row * pg.C + col;
			if (LAST) {
				Psi[e] = mk<T>(T(basis_re(row, pg.b0 + col)), T(basis_im(row, pg.b0 + col)));
				if (TAN) dPsi[e] = czero<V>();
			} else {
				Psi[e] = psi[a];
				if (TAN) dPsi[e] = dpsi[a];
			}
			Phi[e] = phi[a];
			if (TAN) dPhi[e] = FIRST ? czero<V>() : dphi[a];
		}
		__syncthreads();
		// recompute the states entering gates 1..K-1
#pragma unroll
		for (int k = 0; k < MAXK - 1; k++) {
			if (k + 1 >= K) break;
			const V* gk = sg + 32 * k;
			const V* src = Psi + k * A;
			V* dst = Psi + (k + 1) * A;
			const V* dsrc = TAN ? dPsi + k * A : nullptr;
			V* ddst = TAN ? dPsi + (k + 1) * A : nullptr;
			for (int base = 0; base < A; base += blockDim.x) {
				const int task = base + threadIdx.x;
				if (task >= A) break;
				const int g = task >> 2;
				const int cc = g % CW, b6 = g / CW;
				int rows[4];
				group_rows(b6, pg.gi[k], pg.gj[k], rows);
				V y = czero<V>(), dy = czero<V>();
#pragma unroll
				for (int m = 0; m < 4; m++) {
					const V x = src[rows[m] * CW + cc];
					y = cfma(gk[4 * q + m], x, y);
					if (TAN) {
						dy = cfma(gk[16 + 4 * q + m], x, dy);
						dy = cfma(gk[4 * q + m], dsrc[rows[m] * CW + cc], dy);
					}
				}
				const int r = sel4_int(rows, q);
				dst[r * CW + cc] = y;
				if (TAN) ddst[r * CW + cc] = dy;
			}
			__syncthreads();
		}
		// reverse through the pass
#pragma unroll
		for (int k = MAXK - 1; k >= 0; k--) {
			if (k >= K) continue;
			const V* gk = sg + 32 * k;
			const V* X = Psi + k * A;
			const V* dX = TAN ? dPsi + k * A : nullptr;
			const bool first_gate = FIRST && k == K - 1;   // adjoint tangent still zero
			const bool last_gate = LAST && k == 0;         // entering state is the basis column, dpsi = 0
			for (int base = 0; base < A; base += blockDim.x) {
				const int task = base + threadIdx.x;
				const bool active = task < A;
				const int g = task >> 2;
				const int cc = g % CW, b6 = g / CW;
				int rows[4];
				group_rows(b6, pg.gi[k], pg.gj[k], rows);
				V p[4], dp[4], x[4], dx[4];
				V np = czero<V>(), ndp = czero<V>();
				if (active) {
#pragma unroll
					for (int m = 0; m < 4; m++) {
						const int a = rows[m] * CW + cc;
						p[m] = Phi[a];
						x[m] = X[a];
						if (TAN) {
							dp[m] = dPhi[a];
							dx[m] = dX[a];
						}
					}
					const V pq = sel4<T>(p, q);
					const V dpq = TAN ? sel4<T>(dp, q) : czero<V>();
#pragma unroll
					for (int c = 0; c < 4; c++) {
						acc[k][2 * c]     = fma(pq.x, x[c].x, fma(-pq.y, x[c].y, acc[k][2 * c]));
						acc[k][2 * c + 1] = fma(pq.x, x[c].y, fma(pq.y, x[c].x, acc[k][2 * c + 1]));
						if (TAN) {
							T hx = acc[k][8 + 2 * c], hy = acc[k][8 + 2 * c + 1];
							if (!last_gate) {
								hx = fma(pq.x, dx[c].x, fma(-pq.y, dx[c].y, hx));
								hy = fma(pq.x, dx[c].y, fma(pq.y, dx[c].x, hy));
							}
							if (!first_gate) {
								hx = fma(dpq.x, x[c].x, fma(-dpq.y, x[c].y, hx));
								hy = fma(dpq.x, x[c].y, fma(dpq.y, x[c].x, hy));
							}
							acc[k][8 + 2 * c] = hx;
							acc[k][8 + 2 * c + 1] = hy;
						}
					}
					if (!(LAST && k == 0)) {
#pragma unroll
						for (int r = 0; r < 4; r++) {
							np = cfma(gk[4 * r + q], p[r], np);
							if (TAN) {
								ndp = cfma(gk[16 + 4 * r + q], p[r], ndp);
								if (!first_gate) ndp = cfma(gk[4 * r + q], dp[r], ndp);
							}
						}
					}
				}
				__syncwarp();
				if (active && !(LAST && k == 0)) {
					const int r = sel4_int(rows, q);
					Phi[r * CW + cc] = np;
					if (TAN) dPhi[r * CW + cc] = ndp;
				}
			}
			if (FLUSH && ++run == RUN) {
				run = 0;
#pragma unroll
				for (int kk = 0; kk < MAXK; kk++)
#pragma unroll
					for (int v = 0; v < NV; v++) { accd[kk][v] += acc[kk][v]; acc[kk][v] = 0; }
			}
			__syncthreads();
		}
		if (!LAST) {
			for (int e = threadIdx.x; e < A; e += blockDim.x) {
				const int r = e / CW, cc = e - r * CW;
				const int64_t a = (rowbase + rowoff[r]) * pg.C + colbase + cc;
				phi_o[a] = Phi[e];
				if (TAN) dphi_o[a] = dPhi[e];
			}
		}
		__syncthreads();
	}

	// reduce: lanes with equal q (xor 16, 8, 4), then over warps
	double* red = reinterpret_cast<double*>(tiles);   // [warps][4][MAXK * NV]
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
	for (int k = 0; k < MAXK; k++)
#pragma unroll
		for (int v = 0; v < NV; v++) {
			double x = FLUSH ? accd[k][v] + (double)acc[k][v] : (double)acc[k][v];
			x += __shfl_xor_sync(0xffffffffu, x, 16);
			x += __shfl_xor_sync(0xffffffffu, x, 8);
			x += __shfl_xor_sync(0xffffffffu, x, 4);
			if (lane < 4) red[(warp * 4 + lane) * (MAXK * NV) + k * NV + v] = x;
		}
	__syncthreads();
	const int nwarps = blockDim.x >> 5;
	for (int idx = threadIdx.x; idx < 4 * K * NV; idx += blockDim.x) {
		const int qq = idx / (K * NV), rem = idx % (K * NV), k = rem / NV, v = rem % NV;
		double s = 0;
		for (int w = 0; w < nwarps; w++) s += red[(w * 4 + qq) * (MAXK * NV) + k * NV + v];
		// v < 8: dG row qq (complex c = v/2); v >= 8: HZ row qq
		const int dst = v < 8 ? 8 * qq + v : 32 + 8 * qq + (v - 8);
		part[(size_t)k * nblk * NPART2 + (size_t)blockIdx.x * NPART2 + dst] += s;
	}
}

// ------------------------------------------------------------------------------ complex128 kernels on the FP64 MMA

// Every per-group step is a small product over real 8x8 embeddings of the 4x4
// complex gates, issued as FP64 MMAs (mma.sync m8n8k4):
//   outputs      out = in * M,  M the embedding of G (out[c] = sum_r in[r] G[r][c]) or of G^T,
//                with in/out 8 groups x 8 components (re/im of 4 amplitudes, interleaved);
//   outer sums   C += P^T X with P, X 4 groups x 8 components, C the raw 8x8 sum whose 2x2
//                blocks hold re/im products (folded into complex dG, HZ by the reduction).
// Shared-memory tiles store row r at physical row (r & ~1) | parity(r): the rows of an
// amplitude group differ in one bit, so the 64-bit operand loads of a half warp hit both
// halves of the bank window and are free of bank conflicts for any gate wires.

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b)
{
	asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
	             : "+d"(d0), "+d"(d1)
	             : "d"(a), "d"(b));
}

__device__ __forceinline__ int prow(int r) { return (r & ~1) | (__popc(r) & 1); }

// element [rowk][coln] of the real embedding of m (or of m^T) for row-vector products
__device__ __forceinline__ double embed(const double2* m, int rowk, int coln, bool tr)
{
	const int r = rowk >> 1, a = rowk & 1, c = coln >> 1, b = coln & 1;
	const double2 v = tr ? m[4 * c + r] : m[4 * r + c];
	return a == 0 ? (b == 0 ? v.x : v.y) : (b == 0 ? -v.y : v.x);
}

constexpr int NTF = 128;   // threads of the complex128 forward kernel (three blocks per SM)
constexpr int NTR = 512;   // threads of the complex128 reverse kernel
constexpr int NPART3 = 128;   // raw 8x8 sums per gate and block: dG then HZ

__device__ __forceinline__ int insert2(int v, int lo, int hi)
{
	v = ((v >> lo) << (lo + 1)) | (v & ((1 << lo) - 1));
	return ((v >> hi) << (hi + 1)) | (v & ((1 << hi) - 1));
}

// row bits of group member `amp` (row index 2*b_i + b_j) for wire bits (bi, bj)
__device__ __forceinline__ int mbits(int amp, int bi, int bj) { return ((amp >> 1) << bi) | ((amp & 1) << bj); }

// complex index of (row, column) in a swizzled tile of 4 columns
__device__ __forceinline__ int sidx(int row, int cc) { return prow(row) * 4 + cc; }

// Per-lane addressing of one gate step: member bits of the operands this lane loads.
struct StepLane
{
	int lo, hi;
	int m_outer, m_k0, m_k1, m_st;   // member bits: outer-product operand, output k-steps 0/1, store
	int part_outer, part_out;
	__device__ __forceinline__ StepLane(int bi, int bj, int lane)
	{
		lo = bi < bj ? bi : bj;
		hi = bi < bj ? bj : bi;
		m_outer = mbits(lane >> 3, bi, bj);
		m_k0 = mbits((lane & 3) >> 1, bi, bj);
		m_k1 = mbits(2 + ((lane & 3) >> 1), bi, bj);
		m_st = mbits(lane & 3, bi, bj);
		part_outer = (lane >> 2) & 1;
		part_out = lane & 1;
	}
};

// B fragments (k-steps 0, 1) of the embedding of gate matrix m (16 complex in smem)
__device__ __forceinline__ void bfrag(const double2* m, bool tr, int lane, double b[2])
{
	b[0] = embed(m, lane & 3, lane >> 2, tr);
	b[1] = embed(m, 4 + (lane & 3), lane >> 2, tr);
}

// out (8 groups of unit u) = in * B (+ in2 * B2 + in_extra * B), stored at the group members
template <bool TAN>
__device__ __forceinline__ void apply_unit(const double* in, const double* din, double2* out, double2* dout, int u,
                                          const StepLane& sl, const double bg[2], const double bz[2], bool dzero,
                                          int lane, bool inplace)
{
	const int bsel = insert2(2 * u + (lane >> 4), sl.lo, sl.hi);
	const int cc = (lane >> 2) & 3;
	const int j0 = sidx(bsel | sl.m_k0, cc) * 2 + sl.part_out;
	const int j1 = sidx(bsel | sl.m_k1, cc) * 2 + sl.part_out;
	const double a0 = in[j0], a1 = in[j1];
	double y0 = 0, y1 = 0, z0 = 0, z1 = 0;
	dmma(y0, y1, a0, bg[0]);
	if (TAN) dmma(z0, z1, a0, bz[0]);
	dmma(y0, y1, a1, bg[1]);
	if (TAN) {
		dmma(z0, z1, a1, bz[1]);
		if (!dzero) {
			dmma(z0, z1, din[j0], bg[0]);
			dmma(z0, z1, din[j1], bg[1]);
		}
	}
	if (inplace) __syncwarp();
	const int st = sidx(bsel | sl.m_st, cc);
	out[st] = make_double2(y0, y1);
	if (TAN) dout[st] = make_double2(z0, z1);
}

// Rows owned by one warp across two gates.  When gates a and b of a pass act on
// disjoint tile bits, the 2^NB tile rows split into 2^(NB-4) sets of 16 rows that are
// closed under both gates (the rows that agree outside the four bits), so a warp can
// apply a then b to its sets with warp-level synchronisation only, and the block
// barrier between the two gates goes away.
__device__ __forceinline__ bool gates_disjoint(const PassGeom& pg, int a, int b)
{
	return (((1 << pg.gi[a]) | (1 << pg.gj[a])) & ((1 << pg.gi[b]) | (1 << pg.gj[b]))) == 0;
}

// first row of set s: s with zero bits inserted at the set bits of m (in increasing order)
__device__ __forceinline__ int set_base(int s, int m)
{
#pragma unroll
	for (int i = 0; i < 4; i++) {
		const int p = __ffs(m) - 1;
		s = ((s >> p) << (p + 1)) | (s & ((1 << p) - 1));
		m &= m - 1;
	}
	return s;
}

// The group bases of the two units a warp works on at once: unit 0 holds the groups at
// bases b00 and b01, unit 1 those at b10 and b11 (the group base of a unit is selected by
// lane >> 4, as in apply_unit).
struct UnitBases
{
	int b00, b01, b10, b11;
};

// units u0 and u1 of a gate's own enumeration (unit u: group bases 2u, 2u+1 with zero
// bits inserted at the gate's tile bits)
__device__ __forceinline__ UnitBases unit_pair(int u0, int u1, int lo, int hi)
{
	return {insert2(2 * u0, lo, hi), insert2(2 * u0 + 1, lo, hi), insert2(2 * u1, lo, hi),
	        insert2(2 * u1 + 1, lo, hi)};
}

// the two units of the row set with first row S for a gate whose partner gate has tile
// bits (o1, o2): bases S, S|2^o1 and S|2^o2, S|2^o1|2^o2
__device__ __forceinline__ UnitBases set_units(int S, int o1, int o2)
{
	return {S, S | (1 << o1), S | (1 << o2), S | (1 << o1) | (1 << o2)};
}

// apply_unit for two units of a warp at once; bs0 and bs1 are this lane's group bases of
// the two units (the second is ignored unless has1, which is the same for all lanes).
// Both units' operands are loaded before either is stored, so the two independent MMA
// chains overlap; in place like apply_unit(..., inplace = true).
template <bool TAN>
__device__ __forceinline__ void apply_bases2(const double* in, const double* din, double2* out, double2* dout,
                                            int bs0, int bs1, bool has1, const StepLane& sl, const double bg[2],
                                            const double bz[2], bool dzero, int lane)
{
	const int cc = (lane >> 2) & 3;
	if (!has1) bs1 = bs0;
	const int j00 = sidx(bs0 | sl.m_k0, cc) * 2 + sl.part_out, j01 = sidx(bs0 | sl.m_k1, cc) * 2 + sl.part_out;
	const int j10 = sidx(bs1 | sl.m_k0, cc) * 2 + sl.part_out, j11 = sidx(bs1 | sl.m_k1, cc) * 2 + sl.part_out;
	const double a00 = in[j00], a01 = in[j01], a10 = in[j10], a11 = in[j11];
	double d00 = 0, d01 = 0, d10 = 0, d11 = 0;
	if (TAN && !dzero) {
		d00 = din[j00];
		d01 = din[j01];
		d10 = din[j10];
		d11 = din[j11];
	}
	double y0a = 0, y1a = 0, y0b = 0, y1b = 0, z0a = 0, z1a = 0, z0b = 0, z1b = 0;
	dmma(y0a, y1a, a00, bg[0]);
	dmma(y0b, y1b, a10, bg[0]);
	if (TAN) {
		dmma(z0a, z1a, a00, bz[0]);
		dmma(z0b, z1b, a10, bz[0]);
	}
	dmma(y0a, y1a, a01, bg[1]);
	dmma(y0b, y1b, a11, bg[1]);
	if (TAN) {
		dmma(z0a, z1a, a01, bz[1]);
		dmma(z0b, z1b, a11, bz[1]);
		if (!dzero) {
			dmma(z0a, z1a, d00, bg[0]);
			dmma(z0b, z1b, d10, bg[0]);
			dmma(z0a, z1a, d01, bg[1]);
			dmma(z0b, z1b, d11, bg[1]);
		}
	}
	__syncwarp();
	const int st0 = sidx(bs0 | sl.m_st, cc), st1 = sidx(bs1 | sl.m_st, cc);
	out[st0] = make_double2(y0a, y1a);
	if (TAN) dout[st0] = make_double2(z0a, z1a);
	if (has1) {
		out[st1] = make_double2(y0b, y1b);
		if (TAN) dout[st1] = make_double2(z0b, z1b);
	}
}

// apply_bases2 for units u0 and u1 of a gate (unit u: the group bases 2u, 2u+1 of the
// gate's own enumeration)
template <bool TAN>
__device__ __forceinline__ void apply_unit2(const double* in, const double* din, double2* out, double2* dout, int u0,
                                           int u1, bool has1, const StepLane& sl, const double bg[2], const double bz[2],
                                           bool dzero, int lane)
{
	const int bs0 = insert2(2 * u0 + (lane >> 4), sl.lo, sl.hi);
	const int bs1 = insert2(2 * (has1 ? u1 : u0) + (lane >> 4), sl.lo, sl.hi);
	apply_bases2<TAN>(in, din, out, dout, bs0, bs1, has1, sl, bg, bz, dzero, lane);
}

// 16-byte asynchronous copy global -> shared (cp.async, L2 only), and its group fences
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src)
{
	const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// shared memory of k3_fwd: gates, row offsets and two buffers of (state, tangent) tiles
inline size_t k3_fwd_smem(int NB, bool tan)
{
	return 32 * MAXK * sizeof(double2) + (1 << MAXNB) * sizeof(int) + (tan ? 4 : 2) * ((size_t)1 << NB) * 4 * sizeof(double2);
}

// Forward pass (complex128).  Same contract as k2_fwd; OUT 3 writes the pass output
// and adds f, as the last pass does when the reverse pass rebuilds states from it.
// Tiles are double-buffered in shared memory: the next tile position's state arrives
// by cp.async while the gates run on the current one.
template <bool TAN, int IN, int OUT>
__global__ void __launch_bounds__(NTF, TAN ? 3 : 6) k3_fwd(const double2* __restrict__ psi, const double2* __restrict__ dpsi,
                                              double2* __restrict__ psi_o, double2* __restrict__ dpsi_o,
                                              const double2* __restrict__ phi, PassGeom pg, PassGates<double> gates,
                                              double2* __restrict__ fpart)
{
	constexpr int CW = 4;
	constexpr int EPTF = (1 << MAXNB) * CW / NTF;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int R = 1 << pg.NB, A = R * CW, K = pg.K;
	double2* sg = reinterpret_cast<double2*>(smem_raw);
	int* rowoff = reinterpret_cast<int*>(sg + 32 * MAXK);
	double2* bufs = reinterpret_cast<double2*>(rowoff + (1 << MAXNB));   // [2][state, tangent][A], or [2][state][A] without tangents
	gates_to_smem<double>(gates, K, TAN, sg);
	row_offsets(pg, rowoff);
	__syncthreads();
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
	double fx = 0, fy = 0;
	const int units = R / 8;
	// the pass input of a tile position into buffer b (IN 0: read from psi, dpsi)
	auto fetch = [&](int64_t tile, int b) {
		if (IN != 0 || tile >= pg.ntiles) return;
		const int64_t rt = tile / pg.ncg, cg = tile - rt * pg.ncg;
		const int64_t rowbase = deposit(rt, pg.rest_mask), colbase = cg * CW;
		double2* dst = bufs + (size_t)b * (TAN ? 2 : 1) * A;
#pragma unroll
		for (int i = 0; i < EPTF; i++) {
			const int e = threadIdx.x + i * NTF;
			if (e >= A) continue;
			const int64_t a = (rowbase + rowoff[e >> 2]) * pg.C + colbase + (e & 3);
			const int pe = sidx(e >> 2, e & 3);
			cp_async16(dst + pe, psi + a);
			if (TAN) cp_async16(dst + A + pe, dpsi + a);
		}
	};
	fetch(blockIdx.x, 0);
	cp_async_commit();

	int buf = 0;
	for (int64_t tile = blockIdx.x; tile < pg.ntiles; tile += gridDim.x, buf ^= 1) {
		const int64_t rt = tile / pg.ncg, cg = tile - rt * pg.ncg;
		const int64_t rowbase = deposit(rt, pg.rest_mask);
		const int64_t colbase = cg * CW;
		double2* S = bufs + (size_t)buf * (TAN ? 2 : 1) * A;
		double2* dS = TAN ? S + A : nullptr;
		if (IN == 0) {
			cp_async_wait_all();
		} else {
#pragma unroll
			for (int i = 0; i < EPTF; i++) {
				const int e = threadIdx.x + i * NTF;
				if (e >= A) continue;
				const int r = e >> 2, cc = e & 3;
				const int pe = sidx(r, cc);
				const int64_t row = rowbase + rowoff[r], col = colbase + cc;
				S[pe] = make_double2(basis_re(row, pg.b0 + col), basis_im(row, pg.b0 + col));
				if (TAN) dS[pe] = make_double2(0, 0);
			}
		}
		// every thread's copies (or writes) of this tile have landed, and every thread is
		// done with the other buffer (its previous tile), which the next fetch overwrites
		__syncthreads();
		fetch(tile + gridDim.x, buf ^ 1);
		cp_async_commit();
		const double* fS = reinterpret_cast<const double*>(S);
		const double* fdS = reinterpret_cast<const double*>(dS);
		bool skip = false;   // gate k was applied with gate k-1
#pragma unroll
		for (int k = 0; k < MAXK; k++) {
			if (k >= K) break;
			if (skip) { skip = false; continue; }
			const bool dzero = IN == 1 && k == 0;
			const int k2 = k + 1 < MAXK ? k + 1 : k;
			if (k + 1 < K && pg.NB >= 4 && gates_disjoint(pg, k, k2)) {
				// gates k and k+1 on this warp's row sets, one block barrier for both (each
				// gate's operands are loaded per set, which keeps registers for one gate)
				const int m = (1 << pg.gi[k]) | (1 << pg.gj[k]) | (1 << pg.gi[k2]) | (1 << pg.gj[k2]);
				const int hs = lane >> 4;
				for (int s = warp; s < (R >> 4); s += nwarps) {
					const int S0 = set_base(s, m);
					{
						const StepLane sl(pg.gi[k], pg.gj[k], lane);
						double bg[2], bz[2] = {0, 0};
						bfrag(sg + 32 * k, true, lane, bg);
						if (TAN) bfrag(sg + 32 * k + 16, true, lane, bz);
						const UnitBases ua = set_units(S0, pg.gi[k2], pg.gj[k2]);
						apply_bases2<TAN>(fS, fdS, S, dS, hs ? ua.b01 : ua.b00, hs ? ua.b11 : ua.b10, true, sl, bg,
						                  bz, dzero, lane);
					}
					__syncwarp();
					const StepLane sl2(pg.gi[k2], pg.gj[k2], lane);
					double bg2[2], bz2[2] = {0, 0};
					bfrag(sg + 32 * k2, true, lane, bg2);
					if (TAN) bfrag(sg + 32 * k2 + 16, true, lane, bz2);
					const UnitBases ub = set_units(S0, pg.gi[k], pg.gj[k]);
					apply_bases2<TAN>(fS, fdS, S, dS, hs ? ub.b01 : ub.b00, hs ? ub.b11 : ub.b10, true, sl2, bg2, bz2,
					                  false, lane);
				}
				skip = true;
			} else {
				const StepLane sl(pg.gi[k], pg.gj[k], lane);
				double bg[2], bz[2] = {0, 0};
				bfrag(sg + 32 * k, true, lane, bg);
				if (TAN) bfrag(sg + 32 * k + 16, true, lane, bz);
				for (int u = warp; u < units; u += 2 * nwarps)
					apply_unit2<TAN>(fS, fdS, S, dS, u, u + nwarps, u + nwarps < units, sl, bg, bz, dzero, lane);
			}
			__syncthreads();
		}
		for (int i = 0; i < EPTF; i++) {
			const int e = threadIdx.x + i * NTF;
			if (e >= A) continue;
			const int r = e >> 2, cc = e & 3;
			const int64_t a = (rowbase + rowoff[r]) * pg.C + colbase + cc;
			const int pe = sidx(r, cc);
			if (OUT == 2 || OUT == 3) {
				const double2 p = phi[a], v = S[pe];
				fx += p.x * v.x - p.y * v.y;
				fy += p.x * v.y + p.y * v.x;
			}
			if (OUT == 1) {
				psi_o[a] = cneg_conj(S[pe]);
			} else if (OUT != 2) {
				psi_o[a] = S[pe];
				if (TAN) dpsi_o[a] = dS[pe];
			}
		}
	}
	cp_async_wait_all();
	if (OUT == 2 || OUT == 3) {
		__shared__ double red[2][NTF / 32];
		fx = warp_sum(fx);
		fy = warp_sum(fy);
		if (lane == 0) { red[0][warp] = fx; red[1][warp] = fy; }
		__syncthreads();
		if (threadIdx.x == 0) {
			double sx = 0, sy = 0;
			for (int w = 0; w < nwarps; w++) { sx += red[0][w]; sy += red[1][w]; }
			fpart[blockIdx.x].x += sx;
			fpart[blockIdx.x].y += sy;
		}
	}
}

// Reverse pass (complex128).  Same contract as k2_rev; partials are raw 8x8 sums
// (part + k * nblk * 128 + blockIdx.x * 128: [0, 64) dG, [64, 128) HZ, index m*8 + n).
template <bool TAN, bool FIRST, bool LAST>
__global__ void __launch_bounds__(NTR, 1) k3_rev(const double2* __restrict__ psi, const double2* __restrict__ dpsi,
                                                 const double2* __restrict__ phi, const double2* __restrict__ dphi,
                                                 double2* __restrict__ phi_o, double2* __restrict__ dphi_o,
                                                 PassGeom pg, PassGates<double> gates, double* __restrict__ part, int nblk)
{
	constexpr int CW = 4;
	constexpr int EPTR = (1 << MAXNB) * CW / NTR;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int R = 1 << pg.NB, A = R * CW, K = pg.K;
	double2* sg = reinterpret_cast<double2*>(smem_raw);
	int* rowoff = reinterpret_cast<int*>(sg + 32 * MAXK);
	double2* tiles = reinterpret_cast<double2*>(rowoff + (1 << MAXNB));
	double2* Psi = tiles;
	double2* dPsi = TAN ? tiles + K * A : nullptr;
	double2* Phi = tiles + (TAN ? 2 * K : K) * A;
	double2* dPhi = TAN ? Phi + A : nullptr;
	gates_to_smem<double>(gates, K, TAN, sg);
	row_offsets(pg, rowoff);
	__syncthreads();
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
	double cg0[MAXK], cg1[MAXK], ch0[MAXK], ch1[MAXK];
#pragma unroll
	for (int k = 0; k < MAXK; k++) { cg0[k] = cg1[k] = ch0[k] = ch1[k] = 0; }
	const int units = R / 8;
	double2 ra[EPTR], rb[EPTR], rc[EPTR], rd[EPTR];
	auto fetch = [&](int64_t tile) {
		const int64_t rt = tile / pg.ncg, cg = tile - rt * pg.ncg;
		const int64_t rowbase = deposit(rt, pg.rest_mask), colbase = cg * CW;
#pragma unroll
		for (int i = 0; i < EPTR; i++) {
			const int e = threadIdx.x + i * NTR;
			if (e >= A || tile >= pg.ntiles) continue;
			const int64_t a = (rowbase + rowoff[e >> 2]) * pg.C + colbase + (e & 3);
			if (!LAST) {
				ra[i] = psi[a];
				if (TAN) rb[i] = dpsi[a];
			}
			rc[i] = phi[a];
			if (TAN && !FIRST) rd[i] = dphi[a];
		}
	};
	fetch(blockIdx.x);

	for (int64_t tile = blockIdx.x; tile < pg.ntiles; tile += gridDim.x) {
		const int64_t rt = tile / pg.ncg, cgp = tile - rt * pg.ncg;
		const int64_t rowbase = deposit(rt, pg.rest_mask);
		const int64_t colbase = cgp * CW;
#pragma unroll
		for (int i = 0; i < EPTR; i++) {
			const int e = threadIdx.x + i * NTR;
			if (e >= A) continue;
			const int r = e >> 2, cc = e & 3;
			const int pe = sidx(r, cc);
			if (LAST) {
				const int64_t row = rowbase + rowoff[r], col = colbase + cc;
				Psi[pe] = make_double2(basis_re(row, pg.b0 + col), basis_im(row, pg.b0 + col));
				if (TAN) dPsi[pe] = make_double2(0, 0);
			} else {
				Psi[pe] = ra[i];
				if (TAN) dPsi[pe] = rb[i];
			}
			Phi[pe] = rc[i];
			if (TAN) dPhi[pe] = FIRST ? make_double2(0, 0) : rd[i];
		}
		__syncthreads();
		fetch(tile + gridDim.x);
		// recompute the states entering gates 1..K-1
#pragma unroll
		for (int k = 0; k < MAXK - 1; k++) {
			if (k + 1 >= K) break;
			const StepLane sl(pg.gi[k], pg.gj[k], lane);
			double bg[2], bz[2] = {0, 0};
			bfrag(sg + 32 * k, true, lane, bg);
			if (TAN) bfrag(sg + 32 * k + 16, true, lane, bz);
			const bool dzero = LAST && k == 0;
			for (int u = warp; u < units; u += nwarps)
				apply_unit<TAN>(reinterpret_cast<const double*>(Psi + k * A),
				                TAN ? reinterpret_cast<const double*>(dPsi + k * A) : nullptr, Psi + (k + 1) * A,
				                TAN ? dPsi + (k + 1) * A : nullptr, u, sl, bg, bz, dzero, lane, false);
			__syncthreads();
		}
		// reverse through the pass
		const double* P = reinterpret_cast<const double*>(Phi);
		const double* dP = TAN ? reinterpret_cast<const double*>(dPhi) : nullptr;
#pragma unroll
		for (int k = MAXK - 1; k >= 0; k--) {
			if (k >= K) continue;
			const StepLane sl(pg.gi[k], pg.gj[k], lane);
			double bg[2], bz[2] = {0, 0};
			bfrag(sg + 32 * k, false, lane, bg);
			if (TAN) bfrag(sg + 32 * k + 16, false, lane, bz);
			const bool first_gate = FIRST && k == K - 1;
			const bool last_gate = LAST && k == 0;
			const double* X = reinterpret_cast<const double*>(Psi + k * A);
			const double* dX = TAN ? reinterpret_cast<const double*>(dPsi + k * A) : nullptr;
			for (int u = warp; u < units; u += nwarps) {
				const int base0 = insert2(2 * u, sl.lo, sl.hi), base1 = insert2(2 * u + 1, sl.lo, sl.hi);
				// outer products over the two sets of four groups
				const int i0 = sidx(base0 | sl.m_outer, lane & 3) * 2 + sl.part_outer;
				const int i1 = sidx(base1 | sl.m_outer, lane & 3) * 2 + sl.part_outer;
				const double p0 = P[i0], x0 = X[i0], p1 = P[i1], x1 = X[i1];
				dmma(cg0[k], cg1[k], p0, x0);
				if (TAN && !last_gate) dmma(ch0[k], ch1[k], p0, dX[i0]);
				dmma(cg0[k], cg1[k], p1, x1);
				if (TAN && !last_gate) dmma(ch0[k], ch1[k], p1, dX[i1]);
				if (TAN && !first_gate) {
					dmma(ch0[k], ch1[k], dP[i0], x0);
					dmma(ch0[k], ch1[k], dP[i1], x1);
				}
				if (last_gate) continue;
				// adjoint outputs: phi' = phi G, dphi' = dphi G + phi Z (in place)
				apply_unit<TAN>(P, dP, Phi, dPhi, u, sl, bg, bz, first_gate, lane, true);
			}
			__syncthreads();
		}
		if (!LAST) {
			for (int i = 0; i < EPTR; i++) {
				const int e = threadIdx.x + i * NTR;
				if (e >= A) continue;
				const int r = e >> 2, cc = e & 3;
				const int64_t a = (rowbase + rowoff[r]) * pg.C + colbase + cc;
				const int pe = sidx(r, cc);
				phi_o[a] = Phi[pe];
				if (TAN) dphi_o[a] = dPhi[pe];
			}
		}
		__syncthreads();
	}

	// sum the warps' raw 8x8 accumulators; lane l holds entries 2l, 2l+1
	double* red = reinterpret_cast<double*>(tiles);   // [warps][MAXK][128]
#pragma unroll
	for (int k = 0; k < MAXK; k++) {
		if (k >= K) break;
		double* w = red + ((size_t)warp * MAXK + k) * NPART3;
		w[2 * lane] = cg0[k];
		w[2 * lane + 1] = cg1[k];
		w[64 + 2 * lane] = TAN ? ch0[k] : 0.0;
		w[64 + 2 * lane + 1] = TAN ? ch1[k] : 0.0;
	}
	__syncthreads();
	for (int idx = threadIdx.x; idx < K * NPART3; idx += blockDim.x) {
		const int k = idx / NPART3, v = idx % NPART3;
		double s = 0;
		for (int w = 0; w < nwarps; w++) s += red[((size_t)w * MAXK + k) * NPART3 + v];
		part[(size_t)k * nblk * NPART3 + (size_t)blockIdx.x * NPART3 + v] += s;
	}
}

// Sum raw 8x8 partials over blocks (compensated) and fold them into complex dG, HZ:
// X[r][c] = (R[2r][2c] - R[2r+1][2c+1]) + i (R[2r][2c+1] + R[2r+1][2c]).
__global__ void k3_reduce(const double* __restrict__ part, int nslots, int nblk, const double2* __restrict__ fpart,
                          int nblk_f, int with_hvp, double2* __restrict__ out)
{
	__shared__ double raw[NPART3];
	const int s = blockIdx.x, t = threadIdx.x;
	if (s < nslots) {
		if (t < NPART3) {
			double sum = 0, comp = 0;
			for (int b = 0; b < nblk; b++) {
				const double y = part[((size_t)s * nblk + b) * NPART3 + t] - comp;
				const double u = sum + y;
				comp = (u - sum) - y;
				sum = u;
			}
			raw[t] = sum;
		}
		__syncthreads();
		if (t < 32) {
			const int which = t >> 4, e = t & 15, r = e >> 2, c = e & 3;
			if (which == 1 && !with_hvp) return;
			const double* R = raw + 64 * which;
			const double re = R[(2 * r) * 8 + 2 * c] - R[(2 * r + 1) * 8 + 2 * c + 1];
			const double im = R[(2 * r) * 8 + 2 * c + 1] + R[(2 * r + 1) * 8 + 2 * c];
			out[1 + 16 * (size_t)(which ? nslots + s : s) + e] = make_double2(re, im);
		}
	} else if (t < 2) {
		double sum = 0, comp = 0;
		for (int b = 0; b < nblk_f; b++) {
			const double y = (t == 0 ? fpart[b].x : fpart[b].y) - comp;
			const double u = sum + y;
			comp = (u - sum) - y;
			sum = u;
		}
		reinterpret_cast<double*>(out)[t] = sum;
	}
}

// ------------------------------------------------------------------------------ complex64 kernels on TF32 MMAs

// complex64 passes on the tensor cores: every product of the passes is a
// mma.sync m16n8k8 with TF32 inputs, split three ways (a = big + small, both
// TF32; a*b = big*big + big*small + small*big), which keeps FP32 accuracy.
//   outputs       (16 groups x 8 components) * (8 x 8 embedding of G, G^T, Z or Z^T);
//   outer sums    [P; dP]^T (16 components x 8 groups) * X (8 groups x 8 components)
//                 plus [0; P]^T * dX into the same accumulator: rows 0-7 give dG,
//                 rows 8-15 give HZ (raw real 8x8 blocks).
// Tiles hold 256 rows x 8 complex64 columns (64-byte runs), rows swizzled as in the
// complex128 kernels.  The FP32 MMA accumulators are added every few tiles into FP64
// per-lane sums in global scratch (resident in L2) and reduced in FP64.

constexpr int NT4 = 512;
constexpr int CW4 = 8;
constexpr int NRAW4 = 128;      // raw partial sums per gate and block: lane*4 + v
constexpr int FLUSH4 = 4;       // tiles between FP32 -> FP64 flushes

// x = big + small: big is x rounded to the 10 explicit mantissa bits of TF32
// (round half away from zero on the bit pattern), small = x - big exactly; the
// tensor core reads small truncated, an error below 2^-22 |x|.
__device__ __forceinline__ void tf32_split(float x, uint32_t& big, uint32_t& small)
{
	big = (__float_as_uint(x) + 0x1000u) & 0xffffe000u;
	small = __float_as_uint(x - __uint_as_float(big));
}

__device__ __forceinline__ void split4(const float a[4], uint32_t ab[4], uint32_t as[4])
{
#pragma unroll
	for (int i = 0; i < 4; i++) tf32_split(a[i], ab[i], as[i]);
}

__device__ __forceinline__ void mma_tf32(float c[4], const uint32_t a[4], const uint32_t b[2])
{
	asm("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
	             : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
	             : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// c += a * b with 3xTF32 on split operands (a = ab + as, b = bb + bs)
__device__ __forceinline__ void mma3(float c[4], const uint32_t ab[4], const uint32_t as[4], const uint32_t bb[2],
                                     const uint32_t bs[2])
{
	mma_tf32(c, as, bb);
	mma_tf32(c, ab, bs);
	mma_tf32(c, ab, bb);
}

// B fragment (rows t, t+4; column g) of the embedding of the complex 4x4 matrix m (float2 smem)
__device__ __forceinline__ void bfrag4(const float2* m, bool tr, int lane, uint32_t bb[2], uint32_t bs[2])
{
	const int t = lane & 3, g = lane >> 2;
#pragma unroll
	for (int h = 0; h < 2; h++) {
		const int rowk = t + 4 * h, coln = g;
		const int r = rowk >> 1, a = rowk & 1, c = coln >> 1, b = coln & 1;
		const float2 v = tr ? m[4 * c + r] : m[4 * r + c];
		const float x = a == 0 ? (b == 0 ? v.x : v.y) : (b == 0 ? -v.y : v.x);
		tf32_split(x, bb[h], bs[h]);
	}
}

// B fragment of the embedding of m (tr: m^T; conj: conj(m); neg: -m), split:
// f[0..1] big, f[2..3] small parts (rows t, t+4; column g).
__device__ __forceinline__ void bfrag4x(const float2* m, bool tr, bool conj, bool neg, int lane, uint32_t f[4])
{
	const int t = lane & 3, g = lane >> 2;
#pragma unroll
	for (int h = 0; h < 2; h++) {
		const int rowk = t + 4 * h, coln = g;
		const int r = rowk >> 1, a = rowk & 1, c = coln >> 1, b = coln & 1;
		float2 v = tr ? m[4 * c + r] : m[4 * r + c];
		if (conj) v.y = -v.y;
		if (neg) { v.x = -v.x; v.y = -v.y; }
		const float x = a == 0 ? (b == 0 ? v.x : v.y) : (b == 0 ? -v.y : v.x);
		tf32_split(x, f[h], f[2 + h]);
	}
}

// Float index of (row, column cc, part) in a swizzled complex64 tile of 8 columns is
// 16 prow(row) + 2 cc + part.  prow(r) = r ^ (parity of r >> 1), so for disjoint bit
// sets 16 prow(x | y) = roff(x) ^ roff(y): every operand address of a gate step is the
// unit's base offset XOR a per-lane offset fixed for the gate.
__device__ __forceinline__ int roff(int x) { return (x ^ (__popc(x >> 1) & 1)) << 4; }

struct Lane4
{
	int lo, hi;
	int E0;              // offset of the unit's second set of groups (b6 odd)
	int LA, LB, LS, LO;  // lane offsets: output operand k-steps 0 / 1, output store, outer-product operand
	__device__ __forceinline__ Lane4(int bi, int bj, int lane)
	{
		const int g = lane >> 2, t = lane & 3;
		lo = bi < bj ? bi : bj;
		hi = bi < bj ? bj : bi;
		E0 = roff(insert2(1, lo, hi));
		LA = roff(mbits(t >> 1, bi, bj)) | (2 * g + (t & 1));
		LB = roff(mbits(2 + (t >> 1), bi, bj)) | (2 * g + (t & 1));
		LS = roff(mbits(t, bi, bj)) | (2 * g);
		LO = roff(mbits(g >> 1, bi, bj)) | (2 * t + (g & 1));
	}
	// base offset of unit u (groups b6 = 2u, 2u + 1): roff(insert2(2u)), whose parity is popc(u)
	__device__ __forceinline__ int unit_base(int u) const
	{
		const int b = insert2(2 * u, lo, hi);
		return (b ^ ((__popc(u) ^ b) & 1)) << 4;
	}
};

// out = in * Bg (dout = din * Bg + in * Bz) for the 16 groups of the unit at base offset B0
// (b6 = 2u, 2u+1; cc = 0..7)
template <bool TAN>
__device__ __forceinline__ void apply_unit4(const float* in, const float* din, float* out, float* dout, int B0,
                                           const Lane4& ln, const uint32_t gb[2], const uint32_t gs[2],
                                           const uint32_t zb[2], const uint32_t zs[2], bool dzero, bool inplace)
{
	const int B1 = B0 ^ ln.E0;
	const int i0 = B0 ^ ln.LA, i1 = B1 ^ ln.LA, i2 = B0 ^ ln.LB, i3 = B1 ^ ln.LB;
	const float a[4] = { in[i0], in[i1], in[i2], in[i3] };
	uint32_t ab[4], as[4];
	split4(a, ab, as);
	float y[4] = {0, 0, 0, 0}, z[4] = {0, 0, 0, 0};
	mma3(y, ab, as, gb, gs);
	if (TAN) {
		mma3(z, ab, as, zb, zs);
		if (!dzero) {
			const float da[4] = { din[i0], din[i1], din[i2], din[i3] };
			split4(da, ab, as);
			mma3(z, ab, as, gb, gs);
		}
	}
	if (inplace) __syncwarp();
	const int s0 = B0 ^ ln.LS, s1 = B1 ^ ln.LS;
	*reinterpret_cast<float2*>(out + s0) = make_float2(y[0], y[1]);
	*reinterpret_cast<float2*>(out + s1) = make_float2(y[2], y[3]);
	if (TAN) {
		*reinterpret_cast<float2*>(dout + s0) = make_float2(z[0], z[1]);
		*reinterpret_cast<float2*>(dout + s1) = make_float2(z[2], z[3]);
	}
}

// apply_unit4 with the lane offsets passed explicitly (kept in registers by the caller)
template <bool TAN>
__device__ __forceinline__ void apply_unit4o(const float* in, const float* din, float* out, float* dout, int B0, int E0,
                                            int LA, int LB, int LS, const uint32_t gb[2], const uint32_t gs[2],
                                            const uint32_t zb[2], const uint32_t zs[2], bool dzero, bool inplace)
{
	const int B1 = B0 ^ E0;
	const int i0 = B0 ^ LA, i1 = B1 ^ LA, i2 = B0 ^ LB, i3 = B1 ^ LB;
	const float a[4] = { in[i0], in[i1], in[i2], in[i3] };
	uint32_t ab[4], as[4];
	split4(a, ab, as);
	float y[4] = {0, 0, 0, 0}, z[4] = {0, 0, 0, 0};
	mma3(y, ab, as, gb, gs);
	if (TAN) {
		mma3(z, ab, as, zb, zs);
		if (!dzero) {
			const float da[4] = { din[i0], din[i1], din[i2], din[i3] };
			split4(da, ab, as);
			mma3(z, ab, as, gb, gs);
		}
	}
	if (inplace) __syncwarp();
	const int s0 = B0 ^ LS, s1 = B1 ^ LS;
	*reinterpret_cast<float2*>(out + s0) = make_float2(y[0], y[1]);
	*reinterpret_cast<float2*>(out + s1) = make_float2(y[2], y[3]);
	if (TAN) {
		*reinterpret_cast<float2*>(dout + s0) = make_float2(z[0], z[1]);
		*reinterpret_cast<float2*>(dout + s1) = make_float2(z[2], z[3]);
	}
}


constexpr int NT4F = 256;   // threads of the complex64 forward kernel (up to three blocks per SM)
constexpr int NT4R = 256;   // threads of the complex64 reverse kernel
constexpr int UPW4 = (1 << MAXNB) / 8 / (NT4R / 32); // units per warp and gate step (full tiles)
static_assert(NT4F == NT4R, "the unit tables assume equal block sizes");

constexpr int AMAX4 = (1 << MAXNB) * CW4;   // tile stride (complex64 elements) of the complex64 kernels

// shared memory of k4_fwd: gates and two sets of tiles (state[, tangent][, phi])
inline size_t k4_fwd_smem(int NB, bool tan, bool with_phi)
{
	(void)NB;
	const size_t A = AMAX4;
	const int ns = (tan ? 2 : 1) + (with_phi ? 1 : 0);
	// gates, per-gate lane tables (fragments of G^T and Z^T, lane offsets, unit bases), tiles
	return 32 * MAXK * sizeof(float2) + MAXK * 2 * 32 * sizeof(uint4) + MAXK * 4 * 32 * sizeof(int) +
	       MAXK * 32 * sizeof(int) + 2 * ns * A * sizeof(float2);
}

// Forward pass (complex64).  Same contract as k2_fwd.  The next tile streams into a
// second set of shared-memory buffers with cp.async while the current one is processed.
template <bool TAN, int IN, int OUT>
__global__ void __launch_bounds__(NT4F, 3) k4_fwd(const float2* __restrict__ psi, const float2* __restrict__ dpsi,
                                                 float2* __restrict__ psi_o, float2* __restrict__ dpsi_o,
                                                 const float2* __restrict__ phi, PassGeom pg, PassGates<float> gates,
                                                 double2* __restrict__ fpart)
{
	constexpr bool FSUM = OUT >= 2;            // sum f = phi . psi (OUT 2: only that; OUT 3: also write psi)
	constexpr int NS = (TAN ? 2 : 1) + (FSUM ? 1 : 0);
	constexpr int CPT = (1 << MAXNB) * 4 / NT4F;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int R = 1 << pg.NB, K = pg.K;
	float2* sg = reinterpret_cast<float2*>(smem_raw);
	uint4* sfr = reinterpret_cast<uint4*>(sg + 32 * MAXK);              // [MAXK][2][32] fragments of G^T, Z^T
	int* slc = reinterpret_cast<int*>(sfr + MAXK * 2 * 32);             // [MAXK][4][32] E0, LA, LB, LS
	int* sub = slc + MAXK * 4 * 32;                                      // [MAXK][32] unit bases
	float2* tiles = reinterpret_cast<float2*>(sub + MAXK * 32);
	auto stage = [&](int buf, int st) { return tiles + (buf * NS + st) * AMAX4; };
	gates_to_smem<float>(gates, K, TAN, sg);
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
	const int units = R / 8;
	__syncthreads();
	if (warp < K) {   // one warp per gate builds its lane tables
		const int k = warp;
		const Lane4 ln(pg.gi[k], pg.gj[k], lane);
		uint32_t f[8] = {0, 0, 0, 0, 0, 0, 0, 0};
		bfrag4x(sg + 32 * k, true, false, false, lane, f);
		if (TAN) bfrag4x(sg + 32 * k + 16, true, false, false, lane, f + 4);
		sfr[(k * 2 + 0) * 32 + lane] = make_uint4(f[0], f[1], f[2], f[3]);
		sfr[(k * 2 + 1) * 32 + lane] = make_uint4(f[4], f[5], f[6], f[7]);
		slc[(k * 4 + 0) * 32 + lane] = ln.E0;
		slc[(k * 4 + 1) * 32 + lane] = ln.LA;
		slc[(k * 4 + 2) * 32 + lane] = ln.LB;
		slc[(k * 4 + 3) * 32 + lane] = ln.LS;
		for (int u = lane; u < units; u += 32) sub[k * 32 + u] = ln.unit_base(u);
	}
	int ro[CPT];
#pragma unroll
	for (int i = 0; i < CPT; i++) {
		const int r = (threadIdx.x + i * NT4F) >> 2;
		int o = 0;
		for (int b = 0; b < pg.NB; b++)
			if ((r >> b) & 1) o |= 1 << pg.tbit[b];
		ro[i] = o;
	}
	double fx = 0, fy = 0;
	auto fetch = [&](int64_t tile, int buf) {
		const int64_t rt = tile / pg.ncg, cg = tile - rt * pg.ncg;
		const int64_t rowbase = deposit(rt, pg.rest_mask), colbase = cg * CW4;
#pragma unroll
		for (int i = 0; i < CPT; i++) {
			const int e = threadIdx.x + i * NT4F;
			if (e >= 4 * R) continue;
			const int r = e >> 2, c2i = 2 * (e & 3);
			const int64_t a = (rowbase + ro[i]) * pg.C + colbase + c2i;
			const int pe = prow(r) * CW4 + c2i;
			if (IN == 0) {
				cp_async16(stage(buf, 0) + pe, psi + a);
				if (TAN) cp_async16(stage(buf, 1) + pe, dpsi + a);
			} else {
				const int64_t row = rowbase + ro[i], col = colbase + c2i;
				*reinterpret_cast<float4*>(stage(buf, 0) + pe) =
				    make_float4(basis_re(row, pg.b0 + col), basis_im(row, pg.b0 + col), basis_re(row, pg.b0 + col + 1),
				                basis_im(row, pg.b0 + col + 1));
				if (TAN) *reinterpret_cast<float4*>(stage(buf, 1) + pe) = make_float4(0.f, 0.f, 0.f, 0.f);
			}
			if (FSUM) cp_async16(stage(buf, NS - 1) + pe, phi + a);
		}
		cp_async_commit();
	};
	__syncthreads();
	if (blockIdx.x < pg.ntiles) fetch(blockIdx.x, 0);
	int buf = 0;
	for (int64_t tile = blockIdx.x; tile < pg.ntiles; tile += gridDim.x, buf ^= 1) {
		cp_async_wait_all();
		__syncthreads();
		if (tile + gridDim.x < pg.ntiles) fetch(tile + gridDim.x, buf ^ 1);
		float* S = reinterpret_cast<float*>(stage(buf, 0));
		float* dS = TAN ? reinterpret_cast<float*>(stage(buf, 1)) : nullptr;
#pragma unroll
		for (int k = 0; k < MAXK; k++) {
			if (k >= K) break;
			const uint4 q0 = sfr[(k * 2 + 0) * 32 + lane], q1 = sfr[(k * 2 + 1) * 32 + lane];
			const uint32_t gb[2] = { q0.x, q0.y }, gs[2] = { q0.z, q0.w };
			const uint32_t zb[2] = { q1.x, q1.y }, zs[2] = { q1.z, q1.w };
			const int E0 = slc[(k * 4 + 0) * 32 + lane], LA = slc[(k * 4 + 1) * 32 + lane];
			const int LB = slc[(k * 4 + 2) * 32 + lane], LS = slc[(k * 4 + 3) * 32 + lane];
#pragma unroll 2
			for (int j = 0; j < UPW4; j++) {
				const int u = warp + j * nwarps;
				if (u >= units) break;
				apply_unit4o<TAN>(S, dS, S, dS, sub[k * 32 + u], E0, LA, LB, LS, gb, gs, zb, zs, IN == 1 && k == 0, true);
			}
			__syncthreads();
		}
		const int64_t rt = tile / pg.ncg, cg = tile - rt * pg.ncg;
		const int64_t rowbase = deposit(rt, pg.rest_mask), colbase = cg * CW4;
#pragma unroll
		for (int i = 0; i < CPT; i++) {
			const int e = threadIdx.x + i * NT4F;
			if (e >= 4 * R) continue;
			const int r = e >> 2, c2i = 2 * (e & 3);
			const int64_t a = (rowbase + ro[i]) * pg.C + colbase + c2i;
			const int pe = prow(r) * CW4 + c2i;
			const float4 v = *reinterpret_cast<const float4*>(stage(buf, 0) + pe);
			if (FSUM) {
				const float4 p = *reinterpret_cast<const float4*>(stage(buf, NS - 1) + pe);
				fx += (double)p.x * v.x - (double)p.y * v.y + (double)p.z * v.z - (double)p.w * v.w;
				fy += (double)p.x * v.y + (double)p.y * v.x + (double)p.z * v.w + (double)p.w * v.z;
			}
			if (OUT == 2) {
			} else if (OUT == 1) {
				*reinterpret_cast<float4*>(psi_o + a) = make_float4(-v.x, v.y, -v.z, v.w);
			} else {
				*reinterpret_cast<float4*>(psi_o + a) = v;
				if (TAN) *reinterpret_cast<float4*>(dpsi_o + a) = *reinterpret_cast<const float4*>(stage(buf, 1) + pe);
			}
		}
	}
	if (FSUM) {
		__shared__ double red[2][NT4F / 32];
		fx = warp_sum(fx);
		fy = warp_sum(fy);
		if (lane == 0) { red[0][warp] = fx; red[1][warp] = fy; }
		__syncthreads();
		if (threadIdx.x == 0) {
			double sx = 0, sy = 0;
			for (int w = 0; w < nwarps; w++) { sx += red[0][w]; sy += red[1][w]; }
			fpart[blockIdx.x].x += sx;
			fpart[blockIdx.x].y += sy;
		}
	}
}

// shared memory of k4_rev: gates, two sets of staged input tiles (psi, phi[, dpsi, dphi])
// and the K-1 recomputed intermediate states (and their tangents)
inline size_t k4_rev_smem(int NB, int K, bool tan)
{
	(void)NB;
	(void)K;
	const int ns = tan ? 4 : 2;
	return 32 * MAXK * sizeof(float2) + (2 * ns + (tan ? 2 : 1) * (MAXK - 1)) * (size_t)AMAX4 * sizeof(float2);
}


// Reverse pass (complex64).  Same contract as k2_rev; partials are raw sums
// (part + k * nblk * NRAW4 + blockIdx.x * NRAW4 + lane * 4 + v).
// scratch: per-block FP64 lane sums, blockIdx.x * (NT4R/32 * 32 * MAXK * 4) doubles.
// The next tile's inputs stream into a second set of shared-memory buffers with
// cp.async while the current tile is processed.  Lane offsets, unit bases and the
// split gate fragments of every gate of the pass stay in registers for the whole launch.
template <bool TAN, bool FIRST, bool LAST>
__global__ void __launch_bounds__(NT4R, 1) k4_rev(const float2* __restrict__ psi, const float2* __restrict__ dpsi,
                                                  const float2* __restrict__ phi, const float2* __restrict__ dphi,
                                                  float2* __restrict__ phi_o, float2* __restrict__ dphi_o, PassGeom pg,
                                                  PassGates<float> gates, double* __restrict__ part, int nblk,
                                                  double* __restrict__ scratch)
{
	constexpr int NS = TAN ? 4 : 2;            // staged streams: psi, phi, dpsi, dphi
	constexpr int CPT = (1 << MAXNB) * 4 / NT4R; // 16-byte chunks per thread and stream
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int R = 1 << pg.NB, K = pg.K;
	float2* sg = reinterpret_cast<float2*>(smem_raw);
	float2* tiles = sg + 32 * MAXK;
	auto stage = [&](int buf, int st) { return tiles + (buf * NS + st) * AMAX4; };
	float2* Mid = tiles + 2 * NS * AMAX4;                        // Psi[1..K-1]
	float2* dMid = TAN ? Mid + (MAXK - 1) * AMAX4 : nullptr;     // dPsi[1..K-1]
	gates_to_smem<float>(gates, K, TAN, sg);
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
	const int units = R / 8;
	// chunks of this thread: row r = e >> 2, columns 2(e & 3), 2(e & 3) + 1
	int ro[CPT];
#pragma unroll
	for (int i = 0; i < CPT; i++) {
		const int r = (threadIdx.x + i * NT4R) >> 2;
		int o = 0;
		for (int b = 0; b < pg.NB; b++)
			if ((r >> b) & 1) o |= 1 << pg.tbit[b];
		ro[i] = o;
	}
	__syncthreads();
	// per-gate constants
	int E0[MAXK], LA[MAXK], LB[MAXK], LS[MAXK], LO[MAXK], GL[MAXK], GH[MAXK];
	uint32_t rgb[MAXK][2], rgs[MAXK][2], rzb[MAXK][2], rzs[MAXK][2];   // G, Z (reverse)
#pragma unroll
	for (int k = 0; k < MAXK; k++) {
		const int kk = k < K ? k : 0;
		const Lane4 ln(pg.gi[kk], pg.gj[kk], lane);
		E0[k] = ln.E0;
		LA[k] = ln.LA;
		LB[k] = ln.LB;
		LS[k] = ln.LS;
		LO[k] = ln.LO;
		GL[k] = ln.lo;
		GH[k] = ln.hi;
		rzb[k][0] = rzb[k][1] = rzs[k][0] = rzs[k][1] = 0;
		bfrag4(sg + 32 * kk, false, lane, rgb[k], rgs[k]);
		if (TAN) bfrag4(sg + 32 * kk + 16, false, lane, rzb[k], rzs[k]);
	}
	double* scr = scratch + ((size_t)blockIdx.x * nwarps + warp) * 32 * MAXK * 4 + (size_t)lane * MAXK * 4;
#pragma unroll
	for (int v = 0; v < MAXK * 4; v++) scr[v] = 0;
	// outer sums: cx = [P; dP]^T X (rows 0-7 dG, rows 8-15 dP^T X), cd = [P; dP]^T dX (rows 0-7 P^T dX)
	float cx[MAXK][4], cd[MAXK][4];
#pragma unroll
	for (int k = 0; k < MAXK; k++)
#pragma unroll
		for (int v = 0; v < 4; v++) { cx[k][v] = 0; cd[k][v] = 0; }
	auto flush = [&]() {
#pragma unroll
		for (int k = 0; k < MAXK; k++) {
			scr[k * 4 + 0] += (double)cx[k][0];
			scr[k * 4 + 1] += (double)cx[k][1];
			scr[k * 4 + 2] += (double)cx[k][2] + (double)cd[k][0];
			scr[k * 4 + 3] += (double)cx[k][3] + (double)cd[k][1];
#pragma unroll
			for (int v = 0; v < 4; v++) { cx[k][v] = 0; cd[k][v] = 0; }
		}
	};
	// stage the inputs of tile `tile` into buffer set `buf`
	auto fetch = [&](int64_t tile, int buf) {
		const int64_t rt = tile / pg.ncg, cg = tile - rt * pg.ncg;
		const int64_t rowbase = deposit(rt, pg.rest_mask), colbase = cg * CW4;
#pragma unroll
		for (int i = 0; i < CPT; i++) {
			const int e = threadIdx.x + i * NT4R;
			if (e >= 4 * R) continue;
			const int r = e >> 2, c2i = 2 * (e & 3);
			const int64_t a = (rowbase + ro[i]) * pg.C + colbase + c2i;
			const int pe = prow(r) * CW4 + c2i;
			if (LAST) {
				const int64_t row = rowbase + ro[i], col = colbase + c2i;
				*reinterpret_cast<float4*>(stage(buf, 0) + pe) =
				    make_float4(basis_re(row, pg.b0 + col), basis_im(row, pg.b0 + col), basis_re(row, pg.b0 + col + 1),
				                basis_im(row, pg.b0 + col + 1));
				if (TAN) *reinterpret_cast<float4*>(stage(buf, 2) + pe) = make_float4(0.f, 0.f, 0.f, 0.f);
			} else {
				cp_async16(stage(buf, 0) + pe, psi + a);
				if (TAN) cp_async16(stage(buf, 2) + pe, dpsi + a);
			}
			cp_async16(stage(buf, 1) + pe, phi + a);
			if (TAN) {
				if (FIRST)
					*reinterpret_cast<float4*>(stage(buf, 3) + pe) = make_float4(0.f, 0.f, 0.f, 0.f);
				else
					cp_async16(stage(buf, 3) + pe, dphi + a);
			}
		}
		cp_async_commit();
	};
	if (blockIdx.x < pg.ntiles) fetch(blockIdx.x, 0);
	int ntile = 0, buf = 0;
	for (int64_t tile = blockIdx.x; tile < pg.ntiles; tile += gridDim.x, buf ^= 1) {
		cp_async_wait_all();
		__syncthreads();
		if (tile + gridDim.x < pg.ntiles) fetch(tile + gridDim.x, buf ^ 1);
		float2* Psi0 = stage(buf, 0);
		float2* Phi = stage(buf, 1);
		float2* dPsi0 = TAN ? stage(buf, 2) : nullptr;
		float2* dPhi = TAN ? stage(buf, 3) : nullptr;
		auto psi_at = [&](int k) { return k == 0 ? Psi0 : Mid + (k - 1) * AMAX4; };
		auto dpsi_at = [&](int k) { return k == 0 ? dPsi0 : dMid + (k - 1) * AMAX4; };
		// recompute the states entering gates 1..K-1
#pragma unroll
		for (int k = 0; k < MAXK - 1; k++) {
			if (k + 1 >= K) break;
			const float* in = reinterpret_cast<const float*>(psi_at(k));
			const float* din = TAN ? reinterpret_cast<const float*>(dpsi_at(k)) : nullptr;
			float* out = reinterpret_cast<float*>(psi_at(k + 1));
			float* dout = TAN ? reinterpret_cast<float*>(dpsi_at(k + 1)) : nullptr;
			uint32_t fgb[2], fgs[2], fzb[2] = {0, 0}, fzs[2] = {0, 0};   // G^T, Z^T
			bfrag4(sg + 32 * k, true, lane, fgb, fgs);
			if (TAN) bfrag4(sg + 32 * k + 16, true, lane, fzb, fzs);
#pragma unroll 2
			for (int j = 0; j < UPW4; j++) {
				const int u = warp + j * nwarps;
				if (u >= units) break;
				const int b = insert2(2 * u, GL[k], GH[k]);
				apply_unit4o<TAN>(in, din, out, dout, (b ^ ((__popc(u) ^ b) & 1)) << 4, E0[k], LA[k], LB[k], LS[k], fgb,
				                  fgs, fzb, fzs, LAST && k == 0, false);
			}
			__syncthreads();
		}
		// reverse through the pass
		const float* P = reinterpret_cast<const float*>(Phi);
		const float* dP = TAN ? reinterpret_cast<const float*>(dPhi) : nullptr;
#pragma unroll
		for (int k = MAXK - 1; k >= 0; k--) {
			if (k >= K) continue;
			const bool first_gate = FIRST && k == K - 1;
			const bool last_gate = LAST && k == 0;
			const float* X = reinterpret_cast<const float*>(psi_at(k));
			const float* dX = TAN ? reinterpret_cast<const float*>(dpsi_at(k)) : nullptr;
#pragma unroll 2
			for (int j = 0; j < UPW4; j++) {
				const int u = warp + j * nwarps;
				if (u >= units) break;
				const int b = insert2(2 * u, GL[k], GH[k]);
				const int B0 = (b ^ ((__popc(u) ^ b) & 1)) << 4;
				// outer products over the two sets (b6 = 2u, 2u+1) of eight groups (cc = 0..7);
				// this lane's operands sit in columns t and t + 4
#pragma unroll
				for (int sset = 0; sset < 2; sset++) {
					const int j0 = (sset ? B0 ^ E0[k] : B0) ^ LO[k], j1 = j0 + 8;
					const float a[4] = { P[j0], (TAN && !first_gate) ? dP[j0] : 0.f, P[j1],
					                     (TAN && !first_gate) ? dP[j1] : 0.f };
					uint32_t ab[4], as[4];
					split4(a, ab, as);
					uint32_t xb[2], xs[2];
					tf32_split(X[j0], xb[0], xs[0]);
					tf32_split(X[j1], xb[1], xs[1]);
					mma3(cx[k], ab, as, xb, xs);
					if (TAN && !last_gate) {
						uint32_t db[2], ds[2];
						tf32_split(dX[j0], db[0], ds[0]);
						tf32_split(dX[j1], db[1], ds[1]);
						mma3(cd[k], ab, as, db, ds);   // rows 0-7: P^T dX (rows 8-15 unused)
					}
				}
				if (last_gate) continue;
				// adjoint outputs: phi' = phi G, dphi' = dphi G + phi Z (in place)
				apply_unit4o<TAN>(P, dP, reinterpret_cast<float*>(Phi), TAN ? reinterpret_cast<float*>(dPhi) : nullptr,
				                  B0, E0[k], LA[k], LB[k], LS[k], rgb[k], rgs[k], rzb[k], rzs[k], first_gate, true);
			}
			__syncthreads();
		}
		if (!LAST) {
			const int64_t rt = tile / pg.ncg, cgp = tile - rt * pg.ncg;
			const int64_t rowbase = deposit(rt, pg.rest_mask), colbase = cgp * CW4;
#pragma unroll
			for (int i = 0; i < CPT; i++) {
				const int e = threadIdx.x + i * NT4R;
				if (e >= 4 * R) continue;
				const int r = e >> 2, c2i = 2 * (e & 3);
				const int64_t a = (rowbase + ro[i]) * pg.C + colbase + c2i;
				const int pe = prow(r) * CW4 + c2i;
				*reinterpret_cast<float4*>(phi_o + a) = *reinterpret_cast<const float4*>(Phi + pe);
				if (TAN) *reinterpret_cast<float4*>(dphi_o + a) = *reinterpret_cast<const float4*>(dPhi + pe);
			}
		}
		if (++ntile == FLUSH4) {
			ntile = 0;
			flush();
		}
	}
	flush();
	__syncthreads();
	// sum over warps: (k, lane, v) -> part
	for (int idx = threadIdx.x; idx < K * NRAW4; idx += blockDim.x) {
		const int k = idx / NRAW4, rem = idx % NRAW4, ln = rem / 4, v = rem % 4;
		double s2 = 0;
		for (int w = 0; w < nwarps; w++)
			s2 += scratch[((size_t)blockIdx.x * nwarps + w) * 32 * MAXK * 4 + (size_t)ln * MAXK * 4 + k * 4 + v];
		part[(size_t)k * nblk * NRAW4 + (size_t)blockIdx.x * NRAW4 + rem] += s2;
	}
}

constexpr int NT5 = 256;   // threads of the reconstructing complex64 reverse kernel (two blocks per SM)

// shared memory of k5_rev: gate matrices (G, Z, W), per-lane fragment and offset
// tables of every gate, unit bases, and the four state tiles (two without tangents)
inline size_t k5_rev_smem(bool tan)
{
	return 48 * MAXK * sizeof(float2) + MAXK * 32 * 16 * sizeof(uint32_t) + MAXK * 5 * 32 * sizeof(int) +
	       MAXK * 32 * sizeof(int) + (tan ? 4 : 2) * (size_t)AMAX4 * sizeof(float2);
}

// Reverse pass (complex64) for unitary gates: starts from the state at the OUTPUT of
// the pass (psi, dpsi = the next pass's checkpoint) and walks back through the pass,
// rebuilding the state entering each gate with the adjoint gate,
//   psi_k = G^+ psi_{k+1},  dpsi_k = G^+ dpsi_{k+1} - (G^+ Z G^+) psi_{k+1},
// so no state inside the pass is recomputed or kept: four tiles, updated in place.
// Partial sums, scratch and the other arguments as in k4_rev.
template <bool TAN, bool FIRST, bool LAST>
__global__ void __launch_bounds__(NT5, 2) k5_rev(const float2* __restrict__ psi, const float2* __restrict__ dpsi,
                                                 const float2* __restrict__ phi, const float2* __restrict__ dphi,
                                                 float2* __restrict__ phi_o, float2* __restrict__ dphi_o, PassGeom pg,
                                                 PassGates<float> gates, PassW<float> wg, double* __restrict__ part,
                                                 int nblk, double* __restrict__ scratch)
{
	constexpr int CPT = (1 << MAXNB) * 4 / NT5;   // 16-byte chunks per thread and state
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int R = 1 << pg.NB, K = pg.K, units = R / 8;
	float2* sg = reinterpret_cast<float2*>(smem_raw);                       // [MAXK][48]: G, Z, W
	uint4* sfr = reinterpret_cast<uint4*>(sg + 48 * MAXK);                  // [MAXK][4][32] fragments
	int* slc = reinterpret_cast<int*>(sfr + MAXK * 4 * 32);                 // [MAXK][5][32] lane offsets
	int* sub = slc + MAXK * 5 * 32;                                          // [MAXK][32] unit bases
	float2* Psi = reinterpret_cast<float2*>(sub + MAXK * 32);
	float2* Phi = Psi + AMAX4;
	float2* dPsi = TAN ? Phi + AMAX4 : nullptr;
	float2* dPhi = TAN ? Phi + 2 * AMAX4 : nullptr;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
	for (int e = threadIdx.x; e < 48 * MAXK; e += blockDim.x) {
		const int k = e / 48, w = e % 48;
		if (k >= K) continue;
		float2 v = make_float2(0.f, 0.f);
		if (w < 16) v = gates.g[k].m[w];
		else if (TAN && w < 32) v = gates.z[k].m[w - 16];
		else if (TAN) v = wg.w[k].m[w - 32];
		sg[e] = v;
	}
	__syncthreads();
	if (warp < K) {   // one warp per gate builds its lane tables
		const int k = warp;
		const Lane4 ln(pg.gi[k], pg.gj[k], lane);
		uint32_t f[16];
		bfrag4x(sg + 48 * k, false, true, false, lane, f);            // G^+ (row-vector operand conj(G))
		bfrag4x(sg + 48 * k + 32, true, false, true, lane, f + 4);    // -W
		bfrag4x(sg + 48 * k, false, false, false, lane, f + 8);       // G^T (operand G)
		bfrag4x(sg + 48 * k + 16, false, false, false, lane, f + 12); // Z^T (operand Z)
#pragma unroll
		for (int q = 0; q < 4; q++) sfr[(k * 4 + q) * 32 + lane] = make_uint4(f[4 * q], f[4 * q + 1], f[4 * q + 2], f[4 * q + 3]);
		slc[(k * 5 + 0) * 32 + lane] = ln.E0;
		slc[(k * 5 + 1) * 32 + lane] = ln.LA;
		slc[(k * 5 + 2) * 32 + lane] = ln.LB;
		slc[(k * 5 + 3) * 32 + lane] = ln.LS;
		slc[(k * 5 + 4) * 32 + lane] = ln.LO;
		for (int u = lane; u < units; u += 32) sub[k * 32 + u] = ln.unit_base(u);
	}
	int ro[CPT];
#pragma unroll
	for (int i = 0; i < CPT; i++) {
		const int r = (threadIdx.x + i * NT5) >> 2;
		int o = 0;
		for (int b = 0; b < pg.NB; b++)
			if ((r >> b) & 1) o |= 1 << pg.tbit[b];
		ro[i] = o;
	}
	double* scr = scratch + ((size_t)blockIdx.x * nwarps + warp) * 32 * MAXK * 4 + (size_t)lane * MAXK * 4;
#pragma unroll
	for (int v = 0; v < MAXK * 4; v++) scr[v] = 0;
	// outer sums: cx = [P; dP]^T X (rows 0-7 dG, rows 8-15 dP^T X), cd = [P; dP]^T dX (rows 0-7 P^T dX)
	float cx[MAXK][4], cd[MAXK][4];
#pragma unroll
	for (int k = 0; k < MAXK; k++)
#pragma unroll
		for (int v = 0; v < 4; v++) { cx[k][v] = 0; cd[k][v] = 0; }
	auto flush = [&]() {
#pragma unroll
		for (int k = 0; k < MAXK; k++) {
			scr[k * 4 + 0] += (double)cx[k][0];
			scr[k * 4 + 1] += (double)cx[k][1];
			scr[k * 4 + 2] += (double)cx[k][2] + (double)cd[k][0];
			scr[k * 4 + 3] += (double)cx[k][3] + (double)cd[k][1];
#pragma unroll
			for (int v = 0; v < 4; v++) { cx[k][v] = 0; cd[k][v] = 0; }
		}
	};
	__syncthreads();
	float* fPsi = reinterpret_cast<float*>(Psi);
	float* fdPsi = reinterpret_cast<float*>(dPsi);
	float* fPhi = reinterpret_cast<float*>(Phi);
	float* fdPhi = reinterpret_cast<float*>(dPhi);
	int ntile = 0;
	for (int64_t tile = blockIdx.x; tile < pg.ntiles; tile += gridDim.x) {
		const int64_t rt = tile / pg.ncg, cgp = tile - rt * pg.ncg;
		const int64_t rowbase = deposit(rt, pg.rest_mask), colbase = cgp * CW4;
#pragma unroll
		for (int i = 0; i < CPT; i++) {
			const int e = threadIdx.x + i * NT5;
			if (e >= 4 * R) continue;
			const int r = e >> 2, c2i = 2 * (e & 3);
			const int64_t a = (rowbase + ro[i]) * pg.C + colbase + c2i;
			const int pe = prow(r) * CW4 + c2i;
			cp_async16(Psi + pe, psi + a);
			cp_async16(Phi + pe, phi + a);
			if (TAN) {
				cp_async16(dPsi + pe, dpsi + a);
				if (FIRST) *reinterpret_cast<float4*>(dPhi + pe) = make_float4(0.f, 0.f, 0.f, 0.f);
				else cp_async16(dPhi + pe, dphi + a);
			}
		}
		cp_async_commit();
		cp_async_wait_all();
		__syncthreads();
#pragma unroll
		for (int k = MAXK - 1; k >= 0; k--) {
			if (k >= K) continue;
			const uint4 q0 = sfr[(k * 4 + 0) * 32 + lane], q1 = sfr[(k * 4 + 1) * 32 + lane];
			const uint4 q2 = sfr[(k * 4 + 2) * 32 + lane], q3 = sfr[(k * 4 + 3) * 32 + lane];
			const uint32_t rcb[2] = { q0.x, q0.y }, rcs[2] = { q0.z, q0.w };
			const uint32_t wb[2] = { q1.x, q1.y }, ws[2] = { q1.z, q1.w };
			const uint32_t gb[2] = { q2.x, q2.y }, gs[2] = { q2.z, q2.w };
			const uint32_t zb[2] = { q3.x, q3.y }, zs[2] = { q3.z, q3.w };
			const int E0 = slc[(k * 5 + 0) * 32 + lane], LA = slc[(k * 5 + 1) * 32 + lane];
			const int LB = slc[(k * 5 + 2) * 32 + lane], LS = slc[(k * 5 + 3) * 32 + lane];
			const int LO = slc[(k * 5 + 4) * 32 + lane];
			const bool first_gate = FIRST && k == K - 1;
			const bool last_gate = LAST && k == 0;
#pragma unroll 2
			for (int j = 0; j < UPW4; j++) {
				const int u = warp + j * nwarps;
				if (u >= units) break;
				const int B0 = sub[k * 32 + u], B1 = B0 ^ E0;
				// 1. the state (and tangent) entering gate k, in place
				{
					const int i0 = B0 ^ LA, i1 = B1 ^ LA, i2 = B0 ^ LB, i3 = B1 ^ LB;
					const float a[4] = { fPsi[i0], fPsi[i1], fPsi[i2], fPsi[i3] };
					uint32_t ab[4], as[4];
					split4(a, ab, as);
					float y[4] = {0, 0, 0, 0}, z[4] = {0, 0, 0, 0};
					mma3(y, ab, as, rcb, rcs);
					const bool dt = TAN && !last_gate;
					if (dt) {
						mma3(z, ab, as, wb, ws);
						const float da[4] = { fdPsi[i0], fdPsi[i1], fdPsi[i2], fdPsi[i3] };
						split4(da, ab, as);
						mma3(z, ab, as, rcb, rcs);
					}
					__syncwarp();
					const int s0 = B0 ^ LS, s1 = B1 ^ LS;
					*reinterpret_cast<float2*>(fPsi + s0) = make_float2(y[0], y[1]);
					*reinterpret_cast<float2*>(fPsi + s1) = make_float2(y[2], y[3]);
					if (dt) {
						*reinterpret_cast<float2*>(fdPsi + s0) = make_float2(z[0], z[1]);
						*reinterpret_cast<float2*>(fdPsi + s1) = make_float2(z[2], z[3]);
					}
					__syncwarp();
				}
				// 2. outer products over the two sets (b6 = 2u, 2u+1) of eight groups
#pragma unroll
				for (int sset = 0; sset < 2; sset++) {
					const int j0 = (sset ? B1 : B0) ^ LO, j1 = j0 + 8;
					const float a[4] = { fPhi[j0], (TAN && !first_gate) ? fdPhi[j0] : 0.f, fPhi[j1],
					                     (TAN && !first_gate) ? fdPhi[j1] : 0.f };
					uint32_t ab[4], as[4];
					split4(a, ab, as);
					uint32_t xb[2], xs[2];
					tf32_split(fPsi[j0], xb[0], xs[0]);
					tf32_split(fPsi[j1], xb[1], xs[1]);
					mma3(cx[k], ab, as, xb, xs);
					if (TAN && !last_gate) {
						uint32_t db[2], ds[2];
						tf32_split(fdPsi[j0], db[0], ds[0]);
						tf32_split(fdPsi[j1], db[1], ds[1]);
						mma3(cd[k], ab, as, db, ds);   // rows 0-7: P^T dX (rows 8-15 unused)
					}
				}
				// 3. adjoint outputs: phi' = phi G, dphi' = dphi G + phi Z (in place)
				if (!last_gate)
					apply_unit4o<TAN>(fPhi, fdPhi, fPhi, fdPhi, B0, E0, LA, LB, LS, gb, gs, zb, zs, first_gate, true);
			}
			__syncthreads();
		}
		if (!LAST) {
#pragma unroll
			for (int i = 0; i < CPT; i++) {
				const int e = threadIdx.x + i * NT5;
				if (e >= 4 * R) continue;
				const int r = e >> 2, c2i = 2 * (e & 3);
				const int64_t a = (rowbase + ro[i]) * pg.C + colbase + c2i;
				const int pe = prow(r) * CW4 + c2i;
				*reinterpret_cast<float4*>(phi_o + a) = *reinterpret_cast<const float4*>(Phi + pe);
				if (TAN) *reinterpret_cast<float4*>(dphi_o + a) = *reinterpret_cast<const float4*>(dPhi + pe);
			}
		}
		if (++ntile == FLUSH4) {
			ntile = 0;
			flush();
		}
		__syncthreads();
	}
	flush();
	__syncthreads();
	for (int idx = threadIdx.x; idx < K * NRAW4; idx += blockDim.x) {
		const int k = idx / NRAW4, rem = idx % NRAW4, ln = rem / 4, v = rem % 4;
		double s2 = 0;
		for (int w = 0; w < nwarps; w++)
			s2 += scratch[((size_t)blockIdx.x * nwarps + w) * 32 * MAXK * 4 + (size_t)ln * MAXK * 4 + k * 4 + v];
		part[(size_t)k * nblk * NRAW4 + (size_t)blockIdx.x * NRAW4 + rem] += s2;
	}
}

// ------------------------------------------------------------------------------ complex128 reverse pass, adjoint reconstruction

// Per-gate operands of the reconstructing complex128 reverse pass, formed on the host in
// FP64: gc = conj(G) (as a row-vector operand it applies G^+) and wn = -W, W = G^+ Z G^+.
struct PassAdj { Gate4<double> gc[MAXK]; Gate4<double> wn[MAXK]; };

// Operands of one gate of the reconstructing reverse pass: B fragments of conj(G) (the
// adjoint gate as a row-vector operand), -W, G and Z, from the gate block of shared memory
// ([G, Z, conj(G), -W], 16 complex each).
template <bool TAN>
struct RevGate
{
	StepLane sl;
	double bc[2], bw[2] = {0, 0}, bg[2], bz[2] = {0, 0};
	bool first_gate, last_gate;
	__device__ __forceinline__ RevGate(const double2* sg, int k, int K, bool first, bool last, const PassGeom& pg,
	                                   int lane)
		: sl(pg.gi[k], pg.gj[k], lane), first_gate(first && k == K - 1), last_gate(last && k == 0)
	{
		bfrag(sg + 64 * k + 32, false, lane, bc);
		if (TAN) bfrag(sg + 64 * k + 48, true, lane, bw);
		bfrag(sg + 64 * k, false, lane, bg);
		if (TAN) bfrag(sg + 64 * k + 16, false, lane, bz);
	}
};

// One gate of the reconstructing reverse pass on two units (the second unless has1 is
// false): rebuild the state (and tangent) entering the gate, in place; add the outer
// sums dG += phi (x) psi, HZ += phi (x) dpsi + dphi (x) psi over the units' groups, into
// fresh partials first (short MMA chains); move phi, dphi through the gate in place.
template <bool TAN>
__device__ __forceinline__ void rev_gate6(const RevGate<TAN>& g, const UnitBases& ub, bool has1, double2* Psi,
                                          double2* dPsi, double2* Phi, double2* dPhi, double& g0, double& g1,
                                          double& h0, double& h1, int lane)
{
	const double* fPsi = reinterpret_cast<const double*>(Psi);
	const double* fPhi = reinterpret_cast<const double*>(Phi);
	const double* fdPsi = reinterpret_cast<const double*>(dPsi);
	const double* fdPhi = reinterpret_cast<const double*>(dPhi);
	const int hs = lane >> 4;
	const int bs0 = hs ? ub.b01 : ub.b00, bs1 = hs ? ub.b11 : ub.b10;
	const StepLane& sl = g.sl;
	if (TAN && !g.last_gate)
		apply_bases2<true>(fPsi, fdPsi, Psi, dPsi, bs0, bs1, has1, sl, g.bc, g.bw, false, lane);
	else
		apply_bases2<false>(fPsi, nullptr, Psi, nullptr, bs0, bs1, has1, sl, g.bc, g.bw, false, lane);
	__syncwarp();
	double tg[2][2] = {{0, 0}, {0, 0}}, th[2][2] = {{0, 0}, {0, 0}};
#pragma unroll
	for (int q = 0; q < 2; q++) {
		if (q == 1 && !has1) break;
		const int base0 = q ? ub.b10 : ub.b00, base1 = q ? ub.b11 : ub.b01;
		const int i0 = sidx(base0 | sl.m_outer, lane & 3) * 2 + sl.part_outer;
		const int i1 = sidx(base1 | sl.m_outer, lane & 3) * 2 + sl.part_outer;
		const double p0 = fPhi[i0], x0 = fPsi[i0], p1 = fPhi[i1], x1 = fPsi[i1];
		double dx0 = 0, dx1 = 0, dp0 = 0, dp1 = 0;
		if (TAN && !g.last_gate) { dx0 = fdPsi[i0]; dx1 = fdPsi[i1]; }
		if (TAN && !g.first_gate) { dp0 = fdPhi[i0]; dp1 = fdPhi[i1]; }
		dmma(tg[q][0], tg[q][1], p0, x0);
		if (TAN && !g.last_gate) dmma(th[q][0], th[q][1], p0, dx0);
		dmma(tg[q][0], tg[q][1], p1, x1);
		if (TAN && !g.last_gate) dmma(th[q][0], th[q][1], p1, dx1);
		if (TAN && !g.first_gate) {
			dmma(th[q][0], th[q][1], dp0, x0);
			dmma(th[q][0], th[q][1], dp1, x1);
		}
	}
	g0 += tg[0][0] + tg[1][0];
	g1 += tg[0][1] + tg[1][1];
	if (TAN) {
		h0 += th[0][0] + th[1][0];
		h1 += th[0][1] + th[1][1];
	}
	if (g.last_gate) return;
	apply_bases2<TAN>(fPhi, fdPhi, Phi, dPhi, bs0, bs1, has1, sl, g.bg, g.bz, g.first_gate, lane);
}

constexpr int NT6 = 128;   // threads of the reconstructing complex128 reverse kernel (three blocks per SM)
constexpr int EPT6 = (1 << MAXNB) * 4 / NT6;   // tile elements per thread and state

inline size_t k6_rev_smem(bool tan)
{
	const size_t A = (size_t)(1 << MAXNB) * 4;
	const size_t tiles = (tan ? 4 : 2) * A * sizeof(double2);
	const size_t red = (size_t)(NT6 / 32) * MAXK * NPART3 * sizeof(double);
	return 64 * MAXK * sizeof(double2) + (1 << MAXNB) * sizeof(int) + std::max(tiles, red);
}

// Reverse pass (complex128) for unitary gates.  It starts from the state at the OUTPUT
// of the pass (psi, dpsi: the next pass's checkpoint, or the circuit's final state) and
// walks back through the pass, rebuilding the state entering each gate with the adjoint
// gate on the FP64 tensor pipe,
//   psi_k = G^+ psi_{k+1},  dpsi_k = G^+ dpsi_{k+1} - W psi_{k+1},  W = G^+ Z G^+,
// so that no state inside the pass is recomputed or kept: four tiles (psi, dpsi, phi,
// dphi), updated in place, and two blocks per SM whose load, compute and store phases
// overlap.  For each gate, per unit of eight amplitude groups: rebuild psi_k, dpsi_k;
// add the outer sums dG_k += phi (x) psi_k, HZ_k += phi (x) dpsi_k + dphi (x) psi_k; move
// phi, dphi through gate k.  Partials and contract as in k3_rev.
template <bool TAN, bool FIRST, bool LAST>
__global__ void __launch_bounds__(NT6, 3) k6_rev(const double2* __restrict__ psi, const double2* __restrict__ dpsi,
                                                 const double2* __restrict__ phi, const double2* __restrict__ dphi,
                                                 double2* __restrict__ phi_o, double2* __restrict__ dphi_o, PassGeom pg,
                                                 PassGates<double> gates, PassAdj adj, double* __restrict__ part, int nblk)
{
	constexpr int CW = 4;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int R = 1 << pg.NB, A = R * CW, K = pg.K;
	double2* sg = reinterpret_cast<double2*>(smem_raw);           // [MAXK][64]: G, Z, conj(G), -W
	int* rowoff = reinterpret_cast<int*>(sg + 64 * MAXK);
	double2* tiles = reinterpret_cast<double2*>(rowoff + (1 << MAXNB));
	double2* Psi = tiles;
	double2* Phi = tiles + A;
	double2* dPsi = TAN ? tiles + 2 * A : nullptr;
	double2* dPhi = TAN ? tiles + 3 * A : nullptr;
	for (int e = threadIdx.x; e < 64 * MAXK; e += blockDim.x) {
		const int k = e / 64, w = e % 64;
		if (k >= K) continue;
		double2 v = make_double2(0, 0);
		if (w < 16) v = gates.g[k].m[w];
		else if (w < 32) v = TAN ? gates.z[k].m[w - 16] : make_double2(0, 0);
		else if (w < 48) v = adj.gc[k].m[w - 32];
		else v = TAN ? adj.wn[k].m[w - 48] : make_double2(0, 0);
		sg[e] = v;
	}
	row_offsets(pg, rowoff);
	__syncthreads();
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
	double cg0[MAXK], cg1[MAXK], ch0[MAXK], ch1[MAXK];
#pragma unroll
	for (int k = 0; k < MAXK; k++) { cg0[k] = cg1[k] = ch0[k] = ch1[k] = 0; }
	const int units = R / 8;

	for (int64_t tile = blockIdx.x; tile < pg.ntiles; tile += gridDim.x) {
		const int64_t rt = tile / pg.ncg, cgp = tile - rt * pg.ncg;
		const int64_t rowbase = deposit(rt, pg.rest_mask);
		const int64_t colbase = cgp * CW;
#pragma unroll
		for (int i = 0; i < EPT6; i++) {
			const int e = threadIdx.x + i * NT6;
			if (e >= A) continue;
			const int r = e >> 2, cc = e & 3;
			const int64_t a = (rowbase + rowoff[r]) * pg.C + colbase + cc;
			const int pe = sidx(r, cc);
			cp_async16(Psi + pe, psi + a);
			cp_async16(Phi + pe, phi + a);
			if (TAN) {
				cp_async16(dPsi + pe, dpsi + a);
				if (FIRST) dPhi[pe] = make_double2(0, 0);
				else cp_async16(dPhi + pe, dphi + a);
			}
		}
		cp_async_commit();
		cp_async_wait_all();
		__syncthreads();
		bool skip = false;   // gate k was done with gate k+1
#pragma unroll
		for (int k = MAXK - 1; k >= 0; k--) {
			if (k >= K) continue;
			if (skip) { skip = false; continue; }
			const int k2 = k >= 1 ? k - 1 : 0;
			if (k >= 1 && pg.NB >= 4 && gates_disjoint(pg, k, k2)) {
				// gates k and k-1 on this warp's row sets, one block barrier for both (each
				// gate's operands are loaded per set, which keeps registers for one gate)
				const int m = (1 << pg.gi[k]) | (1 << pg.gj[k]) | (1 << pg.gi[k2]) | (1 << pg.gj[k2]);
				for (int s = warp; s < (R >> 4); s += nwarps) {
					const int S0 = set_base(s, m);
					{
						const RevGate<TAN> ga(sg, k, K, FIRST, LAST, pg, lane);
						rev_gate6<TAN>(ga, set_units(S0, pg.gi[k2], pg.gj[k2]), true, Psi, dPsi, Phi, dPhi, cg0[k],
						               cg1[k], ch0[k], ch1[k], lane);
					}
					__syncwarp();
					const RevGate<TAN> gb(sg, k2, K, FIRST, LAST, pg, lane);
					rev_gate6<TAN>(gb, set_units(S0, pg.gi[k], pg.gj[k]), true, Psi, dPsi, Phi, dPhi, cg0[k2], cg1[k2],
					               ch0[k2], ch1[k2], lane);
				}
				skip = true;
			} else {
				const RevGate<TAN> ga(sg, k, K, FIRST, LAST, pg, lane);
				for (int u = warp; u < units; u += 2 * nwarps) {
					const int u1 = u + nwarps;
					const bool has1 = u1 < units;   // the same for the whole warp
					rev_gate6<TAN>(ga, unit_pair(u, has1 ? u1 : u, ga.sl.lo, ga.sl.hi), has1, Psi, dPsi, Phi, dPhi,
					               cg0[k], cg1[k], ch0[k], ch1[k], lane);
				}
			}
			__syncthreads();
		}
		if (!LAST) {
#pragma unroll
			for (int i = 0; i < EPT6; i++) {
				const int e = threadIdx.x + i * NT6;
				if (e >= A) continue;
				const int r = e >> 2, cc = e & 3;
				const int64_t a = (rowbase + rowoff[r]) * pg.C + colbase + cc;
				const int pe = sidx(r, cc);
				phi_o[a] = Phi[pe];
				if (TAN) dphi_o[a] = dPhi[pe];
			}
		}
		__syncthreads();
	}

	// sum the warps' raw 8x8 accumulators; lane l holds entries 2l, 2l+1
	double* red = reinterpret_cast<double*>(tiles);   // [warps][MAXK][128]
#pragma unroll
	for (int k = 0; k < MAXK; k++) {
		if (k >= K) break;
		double* w = red + ((size_t)warp * MAXK + k) * NPART3;
		w[2 * lane] = cg0[k];
		w[2 * lane + 1] = cg1[k];
		w[64 + 2 * lane] = TAN ? ch0[k] : 0.0;
		w[64 + 2 * lane + 1] = TAN ? ch1[k] : 0.0;
	}
	__syncthreads();
	for (int idx = threadIdx.x; idx < K * NPART3; idx += blockDim.x) {
		const int k = idx / NPART3, v = idx % NPART3;
		double s = 0;
		for (int w = 0; w < nwarps; w++) s += red[((size_t)w * MAXK + k) * NPART3 + v];
		part[(size_t)k * nblk * NPART3 + (size_t)blockIdx.x * NPART3 + v] += s;
	}
}

// ------------------------------------------------------------------------------ complex64 passes on the FP32 pipe

// The complex64 passes in FP32 FMAs.  Four threads share an amplitude group: thread
// q = lane & 3 computes component q of every product and owns row q of the outer sums,
// column cc = (lane >> 2) & 7 of the tile; a warp handles one group base (eight columns)
// per step, so every operand load is one 64-byte row read by four threads at once and
// every gate coefficient a thread needs (row or column q of G, Z, W: 12 complex numbers)
// stays in registers for the whole gate.  No operand splitting, no fragment exchange:
// 4 x 4 complex products at the FP32 FMA rate (about 2x the FP64 rate on B200).
// Tiles are the k5 tiles (256 rows x 8 columns, rows swizzled by prow so the four rows a
// warp stores land in both halves of the bank window).
constexpr int NT7 = 256;
constexpr int CPT7 = (1 << MAXNB) * 4 / NT7;   // 16-byte chunks per thread and state (two columns each)

__device__ __forceinline__ float2 c7fma(float2 a, float2 b, float2 c)   // a * b + c
{
	return make_float2(fmaf(a.x, b.x, fmaf(-a.y, b.y, c.x)), fmaf(a.x, b.y, fmaf(a.y, b.x, c.y)));
}
__device__ __forceinline__ float2 c7fma_conj(float2 a, float2 b, float2 c)   // conj(a) * b + c
{
	return make_float2(fmaf(a.x, b.x, fmaf(a.y, b.y, c.x)), fmaf(a.x, b.y, fmaf(-a.y, b.x, c.y)));
}

inline size_t k7_fwd_smem() { return 32 * MAXK * sizeof(float2) + 2 * (size_t)AMAX4 * sizeof(float2); }
inline size_t k7_rev_smem()
{
	return 48 * MAXK * sizeof(float2) + 4 * (size_t)AMAX4 * sizeof(float2) + (size_t)(NT7 / 32) * MAXK * 4 * 16 * sizeof(double);
}

// Forward pass (complex64, FP32 FMAs).  Same contract as k4_fwd: IN 0 reads psi/dpsi, 1
// starts from basis columns; OUT 0 stores psi/dpsi, 1 stores -conj(psi), 2 adds f = <phi, psi>
// without storing, 3 stores and adds f.
template <bool TAN, int IN, int OUT>
__global__ void __launch_bounds__(NT7, 3) k7_fwd(const float2* __restrict__ psi, const float2* __restrict__ dpsi,
                                                 float2* __restrict__ psi_o, float2* __restrict__ dpsi_o,
                                                 const float2* __restrict__ phi, PassGeom pg, PassGates<float> gates,
                                                 double2* __restrict__ fpart)
{
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int R = 1 << pg.NB, K = pg.K;
	float2* sg = reinterpret_cast<float2*>(smem_raw);   // [MAXK][32]: G, Z
	float2* S = sg + 32 * MAXK;
	float2* dS = S + AMAX4;
	for (int e = threadIdx.x; e < 32 * MAXK; e += blockDim.x) {
		const int k = e / 32, w = e % 32;
		sg[e] = k >= K ? make_float2(0.f, 0.f) : (w < 16 ? gates.g[k].m[w] : (TAN ? gates.z[k].m[w - 16] : make_float2(0.f, 0.f)));
	}
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
	const int q = lane & 3, cc = (lane >> 2) & 7;
	int ro[CPT7];
#pragma unroll
	for (int i = 0; i < CPT7; i++) {
		const int r = (threadIdx.x + i * NT7) >> 2;
		int o = 0;
		for (int b = 0; b < pg.NB; b++)
			if ((r >> b) & 1) o |= 1 << pg.tbit[b];
		ro[i] = o;
	}
	double fx = 0, fy = 0;
	__syncthreads();
	for (int64_t tile = blockIdx.x; tile < pg.ntiles; tile += gridDim.x) {
		const int64_t rt = tile / pg.ncg, cgp = tile - rt * pg.ncg;
		const int64_t rowbase = deposit(rt, pg.rest_mask), colbase = cgp * CW4;
#pragma unroll
		for (int i = 0; i < CPT7; i++) {
			const int e = threadIdx.x + i * NT7;
			if (e >= 4 * R) continue;
			const int r = e >> 2, c2i = 2 * (e & 3);
			const int pe = prow(r) * CW4 + c2i;
			if (IN == 0) {
				const int64_t a = (rowbase + ro[i]) * pg.C + colbase + c2i;
				cp_async16(S + pe, psi + a);
				if (TAN) cp_async16(dS + pe, dpsi + a);
			} else {
				const int64_t row = rowbase + ro[i], col = colbase + c2i;
				*reinterpret_cast<float4*>(S + pe) =
				    make_float4(basis_re(row, pg.b0 + col), basis_im(row, pg.b0 + col), basis_re(row, pg.b0 + col + 1),
				                basis_im(row, pg.b0 + col + 1));
				if (TAN) *reinterpret_cast<float4*>(dS + pe) = make_float4(0.f, 0.f, 0.f, 0.f);
			}
		}
		if (IN == 0) {
			cp_async_commit();
			cp_async_wait_all();
		}
		__syncthreads();
#pragma unroll 1
		for (int k = 0; k < K; k++) {
			float2 g[4], z[4];
#pragma unroll
			for (int m = 0; m < 4; m++) {
				g[m] = sg[32 * k + 4 * q + m];              // row q of G
				z[m] = TAN ? sg[32 * k + 16 + 4 * q + m] : make_float2(0.f, 0.f);   // row q of Z
			}
			const bool dzero = IN == 1 && k == 0;
			const int bi = pg.gi[k], bj = pg.gj[k];
			for (int b6 = warp; b6 < R / 4; b6 += nwarps) {
				int rows[4];
				group_rows(b6, bi, bj, rows);
				float2 x[4], dx[4];
#pragma unroll
				for (int m = 0; m < 4; m++) {
					x[m] = S[prow(rows[m]) * CW4 + cc];
					dx[m] = (TAN && !dzero) ? dS[prow(rows[m]) * CW4 + cc] : make_float2(0.f, 0.f);
				}
				float2 y = make_float2(0.f, 0.f), dy = make_float2(0.f, 0.f);
#pragma unroll
				for (int m = 0; m < 4; m++) {
					y = c7fma(g[m], x[m], y);
					if (TAN) {
						dy = c7fma(z[m], x[m], dy);
						if (!dzero) dy = c7fma(g[m], dx[m], dy);
					}
				}
				__syncwarp();
				const int st = prow(sel4_int(rows, q)) * CW4 + cc;
				S[st] = y;
				if (TAN) dS[st] = dy;
			}
			__syncthreads();
		}
#pragma unroll
		for (int i = 0; i < CPT7; i++) {
			const int e = threadIdx.x + i * NT7;
			if (e >= 4 * R) continue;
			const int r = e >> 2, c2i = 2 * (e & 3);
			const int64_t a = (rowbase + ro[i]) * pg.C + colbase + c2i;
			const int pe = prow(r) * CW4 + c2i;
			const float4 v = *reinterpret_cast<const float4*>(S + pe);
			if (OUT == 2 || OUT == 3) {
				const float4 p = *reinterpret_cast<const float4*>(phi + a);
				fx += (double)p.x * v.x - (double)p.y * v.y + (double)p.z * v.z - (double)p.w * v.w;
				fy += (double)p.x * v.y + (double)p.y * v.x + (double)p.z * v.w + (double)p.w * v.z;
			}
			if (OUT == 1) {
				*reinterpret_cast<float4*>(psi_o + a) = make_float4(-v.x, v.y, -v.z, v.w);
			} else if (OUT != 2) {
				*reinterpret_cast<float4*>(psi_o + a) = v;
				if (TAN) *reinterpret_cast<float4*>(dpsi_o + a) = *reinterpret_cast<const float4*>(dS + pe);
			}
		}
		__syncthreads();
	}
	if (OUT == 2 || OUT == 3) {
		__shared__ double red[2][NT7 / 32];
		fx = warp_sum(fx);
		fy = warp_sum(fy);
		if (lane == 0) { red[0][warp] = fx; red[1][warp] = fy; }
		__syncthreads();
		if (threadIdx.x == 0) {
			double sx = 0, sy = 0;
			for (int w = 0; w < nwarps; w++) { sx += red[0][w]; sy += red[1][w]; }
			fpart[blockIdx.x].x += sx;
			fpart[blockIdx.x].y += sy;
		}
	}
}

// Reverse pass (complex64, FP32 FMAs) for unitary gates: from the state at the pass
// OUTPUT it rebuilds the state entering each gate with the adjoint gate (as k5_rev),
//   psi_k = G^+ psi_{k+1},  dpsi_k = G^+ dpsi_{k+1} - W psi_{k+1},  W = G^+ Z G^+,
// adds the outer sums dG_k += phi (x) psi_k, HZ_k += phi (x) dpsi_k + dphi (x) psi_k and
// moves phi, dphi through gate k, all in place in four tiles.  Per gate and tile the
// FP32 sums of a thread (eight group-columns) are reduced over the warp and added to
// FP64 per-warp sums in shared memory; partials leave in the k2 layout
// (part + k * nblk * 64 + blockIdx.x * 64: [0, 32) dG, [32, 64) HZ, re/im interleaved).
template <bool TAN, bool FIRST, bool LAST>
__global__ void __launch_bounds__(NT7, 2) k7_rev(const float2* __restrict__ psi, const float2* __restrict__ dpsi,
                                                 const float2* __restrict__ phi, const float2* __restrict__ dphi,
                                                 float2* __restrict__ phi_o, float2* __restrict__ dphi_o, PassGeom pg,
                                                 PassGates<float> gates, PassW<float> wg, double* __restrict__ part,
                                                 int nblk)
{
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int R = 1 << pg.NB, K = pg.K;
	float2* sg = reinterpret_cast<float2*>(smem_raw);   // [MAXK][48]: G, Z, W
	float2* Psi = sg + 48 * MAXK;
	float2* Phi = Psi + AMAX4;
	float2* dPsi = Phi + AMAX4;
	float2* dPhi = dPsi + AMAX4;
	double* accw = reinterpret_cast<double*>(dPhi + AMAX4);   // [warp][MAXK][4 rows][16]
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
	for (int e = threadIdx.x; e < 48 * MAXK; e += blockDim.x) {
		const int k = e / 48, w = e % 48;
		float2 v = make_float2(0.f, 0.f);
		if (k < K) {
			if (w < 16) v = gates.g[k].m[w];
			else if (TAN && w < 32) v = gates.z[k].m[w - 16];
			else if (TAN && w >= 32) v = wg.w[k].m[w - 32];
		}
		sg[e] = v;
	}
	for (int e = threadIdx.x; e < nwarps * MAXK * 64; e += blockDim.x) accw[e] = 0;
	const int q = lane & 3, cc = (lane >> 2) & 7;
	int ro[CPT7];
#pragma unroll
	for (int i = 0; i < CPT7; i++) {
		const int r = (threadIdx.x + i * NT7) >> 2;
		int o = 0;
		for (int b = 0; b < pg.NB; b++)
			if ((r >> b) & 1) o |= 1 << pg.tbit[b];
		ro[i] = o;
	}
	__syncthreads();
	for (int64_t tile = blockIdx.x; tile < pg.ntiles; tile += gridDim.x) {
		const int64_t rt = tile / pg.ncg, cgp = tile - rt * pg.ncg;
		const int64_t rowbase = deposit(rt, pg.rest_mask), colbase = cgp * CW4;
#pragma unroll
		for (int i = 0; i < CPT7; i++) {
			const int e = threadIdx.x + i * NT7;
			if (e >= 4 * R) continue;
			const int r = e >> 2, c2i = 2 * (e & 3);
			const int64_t a = (rowbase + ro[i]) * pg.C + colbase + c2i;
			const int pe = prow(r) * CW4 + c2i;
			cp_async16(Psi + pe, psi + a);
			cp_async16(Phi + pe, phi + a);
			if (TAN) {
				cp_async16(dPsi + pe, dpsi + a);
				if (FIRST) *reinterpret_cast<float4*>(dPhi + pe) = make_float4(0.f, 0.f, 0.f, 0.f);
				else cp_async16(dPhi + pe, dphi + a);
			}
		}
		cp_async_commit();
		cp_async_wait_all();
		__syncthreads();
#pragma unroll 1
		for (int k = K - 1; k >= 0; k--) {
			const bool first_gate = FIRST && k == K - 1;
			const bool last_gate = LAST && k == 0;
			float2 gcol[4], zcol[4], wrow[4];
#pragma unroll
			for (int m = 0; m < 4; m++) {
				gcol[m] = sg[48 * k + 4 * m + q];                                        // G[m][q]
				zcol[m] = TAN ? sg[48 * k + 16 + 4 * m + q] : make_float2(0.f, 0.f);     // Z[m][q]
				wrow[m] = TAN ? sg[48 * k + 32 + 4 * q + m] : make_float2(0.f, 0.f);     // W[q][m]
			}
			float2 ag[4], ah[4];   // row q of this gate's sums: dG[q][c], HZ[q][c]
#pragma unroll
			for (int c = 0; c < 4; c++) { ag[c] = make_float2(0.f, 0.f); ah[c] = make_float2(0.f, 0.f); }
			const int bi = pg.gi[k], bj = pg.gj[k];
			for (int b6 = warp; b6 < R / 4; b6 += nwarps) {
				int rows[4], pr[4];
				group_rows(b6, bi, bj, rows);
#pragma unroll
				for (int m = 0; m < 4; m++) pr[m] = prow(rows[m]) * CW4 + cc;
				float2 x[4], dx[4], p[4], dp[4];
#pragma unroll
				for (int m = 0; m < 4; m++) {
					x[m] = Psi[pr[m]];
					dx[m] = (TAN && !last_gate) ? dPsi[pr[m]] : make_float2(0.f, 0.f);
					p[m] = Phi[pr[m]];
					dp[m] = (TAN && !first_gate) ? dPhi[pr[m]] : make_float2(0.f, 0.f);
				}
				// 1. psi_k (and dpsi_k), component q, in place
				float2 y = make_float2(0.f, 0.f), dy = make_float2(0.f, 0.f);
#pragma unroll
				for (int m = 0; m < 4; m++) {
					y = c7fma_conj(gcol[m], x[m], y);
					if (TAN && !last_gate) {
						dy = c7fma_conj(gcol[m], dx[m], dy);
						dy = c7fma(make_float2(-wrow[m].x, -wrow[m].y), x[m], dy);
					}
				}
				__syncwarp();
				Psi[pr[q]] = y;
				if (TAN && !last_gate) dPsi[pr[q]] = dy;
				__syncwarp();
				// 2. row q of the outer sums with the rebuilt psi_k, dpsi_k
				const float2 pq = p[q], dpq = dp[q];
#pragma unroll
				for (int c = 0; c < 4; c++) {
					const float2 xc = Psi[pr[c]];
					ag[c] = c7fma(pq, xc, ag[c]);
					if (TAN) {
						if (!last_gate) ah[c] = c7fma(pq, dPsi[pr[c]], ah[c]);
						if (!first_gate) ah[c] = c7fma(dpq, xc, ah[c]);
					}
				}
				if (last_gate) continue;
				// 3. phi' = G^T phi, dphi' = G^T dphi + Z^T phi (component q, in place; every lane
				//    read phi before the __syncwarp above)
				float2 u = make_float2(0.f, 0.f), du = make_float2(0.f, 0.f);
#pragma unroll
				for (int m = 0; m < 4; m++) {
					u = c7fma(gcol[m], p[m], u);
					if (TAN) {
						du = c7fma(zcol[m], p[m], du);
						if (!first_gate) du = c7fma(gcol[m], dp[m], du);
					}
				}
				Phi[pr[q]] = u;
				if (TAN) dPhi[pr[q]] = du;
			}
			// sums over the eight columns of the warp (lanes with the same q), then into FP64
			float v[16];
#pragma unroll
			for (int c = 0; c < 4; c++) {
				v[2 * c] = ag[c].x;
				v[2 * c + 1] = ag[c].y;
				v[8 + 2 * c] = ah[c].x;
				v[8 + 2 * c + 1] = ah[c].y;
			}
#pragma unroll
			for (int t = 0; t < 16; t++) {
				if (!TAN && t >= 8) break;
				float x = v[t];
				x += __shfl_xor_sync(0xffffffffu, x, 4);
				x += __shfl_xor_sync(0xffffffffu, x, 8);
				x += __shfl_xor_sync(0xffffffffu, x, 16);
				v[t] = x;
			}
			if (lane < 4) {
				double* a = accw + ((size_t)(warp * MAXK + k) * 4 + q) * 16;
#pragma unroll
				for (int t = 0; t < 16; t++) a[t] += (double)v[t];
			}
			__syncthreads();
		}
		if (!LAST) {
#pragma unroll
			for (int i = 0; i < CPT7; i++) {
				const int e = threadIdx.x + i * NT7;
				if (e >= 4 * R) continue;
				const int r = e >> 2, c2i = 2 * (e & 3);
				const int64_t a = (rowbase + ro[i]) * pg.C + colbase + c2i;
				const int pe = prow(r) * CW4 + c2i;
				*reinterpret_cast<float4*>(phi_o + a) = *reinterpret_cast<const float4*>(Phi + pe);
				if (TAN) *reinterpret_cast<float4*>(dphi_o + a) = *reinterpret_cast<const float4*>(dPhi + pe);
			}
		}
		__syncthreads();
	}
	// block sums in the k2 layout: t < 32 dG (row t / 8, entry (t % 8) / 2, re/im t % 2), t >= 32 HZ
	for (int idx = threadIdx.x; idx < K * NPART2; idx += blockDim.x) {
		const int k = idx / NPART2, t = idx % NPART2;
		const int qq = (t & 31) >> 3, slot = (t >= 32 ? 8 : 0) + (t & 7);
		double sum = 0;
		for (int w = 0; w < nwarps; w++) sum += accw[((size_t)(w * MAXK + k) * 4 + qq) * 16 + slot];
		part[(size_t)k * nblk * NPART2 + (size_t)blockIdx.x * NPART2 + t] += sum;
	}
}

// Sum the complex64 engine's raw partials over blocks and fold them into complex dG, HZ.
// Lane (g, t) of an outer-sum MMA holds C[g][2t..2t+1] (v 0,1) and C[g+8][2t..2t+1]
// (v 2,3): dG raw R[g][2t+i] = v_i, HZ raw R[g][2t+i] = v_{2+i}.
__global__ void k4_reduce(const double* __restrict__ part, int nslots, int nblk, const double2* __restrict__ fpart,
                          int nblk_f, int with_hvp, double2* __restrict__ out)
{
	__shared__ double raw[NRAW4];
	__shared__ double R[2][64];
	const int s = blockIdx.x, t = threadIdx.x;
	if (s < nslots) {
		for (int v = t; v < NRAW4; v += blockDim.x) {
			double sum = 0, comp = 0;
			for (int b = 0; b < nblk; b++) {
				const double y = part[((size_t)s * nblk + b) * NRAW4 + v] - comp;
				const double u = sum + y;
				comp = (u - sum) - y;
				sum = u;
			}
			raw[v] = sum;
		}
		__syncthreads();
		if (t < 64) {
			const int ln = t >> 1, i = t & 1, gg = ln >> 2, tt = ln & 3;
			R[0][gg * 8 + 2 * tt + i] = raw[ln * 4 + i];
			R[1][gg * 8 + 2 * tt + i] = raw[ln * 4 + 2 + i];
		}
		__syncthreads();
		if (t < 32) {
			const int which = t >> 4, e = t & 15, r = e >> 2, c = e & 3;
			if (which == 1 && !with_hvp) return;
			const double* X = R[which];
			const double re = X[(2 * r) * 8 + 2 * c] - X[(2 * r + 1) * 8 + 2 * c + 1];
			const double im = X[(2 * r) * 8 + 2 * c + 1] + X[(2 * r + 1) * 8 + 2 * c];
			out[1 + 16 * (size_t)(which ? nslots + s : s) + e] = make_double2(re, im);
		}
	} else if (t < 2) {
		double sum = 0, comp = 0;
		for (int b = 0; b < nblk_f; b++) {
			const double y = (t == 0 ? fpart[b].x : fpart[b].y) - comp;
			const double u = sum + y;
			comp = (u - sum) - y;
			sum = u;
		}
		reinterpret_cast<double*>(out)[t] = sum;
	}
}

// -conj of host columns [Cc][N] (complex128) into the interleaved chunk [N][C]
template <typename T>
__global__ void k2_target_from_host(const double2* __restrict__ in, cplx<T>* __restrict__ out, int64_t N, int64_t Cc,
                                    int64_t C)
{
	for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N * C; i += (int64_t)gridDim.x * blockDim.x) {
		const int64_t row = i / C, col = i - row * C;
		if (col < Cc) {
			const double2 v = in[col * N + row];
			out[i] = mk<T>((T)(-v.x), (T)v.y);
		} else {
			out[i] = czero<cplx<T>>();
		}
	}
}

// f and per-gate sums over blocks; same record layout as the per-gate engine
__global__ void k2_reduce(const double* __restrict__ part, int nslots, int nblk, const double2* __restrict__ fpart,
                          int nblk_f, int with_hvp, double2* __restrict__ out)
{
	double* o = reinterpret_cast<double*>(out);
	const int s = blockIdx.x, t = threadIdx.x;
	if (s < nslots) {
		if (t >= NPART2 || (!with_hvp && t >= 32)) return;
		double sum = 0, comp = 0;
		for (int b = 0; b < nblk; b++) {
			const double y = part[((size_t)s * nblk + b) * NPART2 + t] - comp;
			const double u = sum + y;
			comp = (u - sum) - y;
			sum = u;
		}
		if (t < 32) o[2 * (1 + 16 * (size_t)s) + t] = sum;
		else o[2 * (1 + 16 * (size_t)nslots + 16 * (size_t)s) + (t - 32)] = sum;
	} else if (t < 2) {
		double sum = 0, comp = 0;
		for (int b = 0; b < nblk_f; b++) {
			const double y = (t == 0 ? fpart[b].x : fpart[b].y) - comp;
			const double u = sum + y;
			comp = (u - sum) - y;
			sum = u;
		}
		o[t] = sum;
	}
}

// ------------------------------------------------------------------------------ scheduling

struct Pass
{
	int first, K;
	PassGeom geom;   // chunk fields filled per launch
};

// Group consecutive gates into passes of up to MAXK gates; tile bits = the union of
// their wires (state bits), padded with the lowest other bits to min(8, L).
std::vector<Pass> schedule(int L, int G, const int* wires, int maxk)
{
	std::vector<Pass> out;
	const int NB = std::min(MAXNB, L);
	for (int i = 0; i < G;) {
		const int K = std::min(maxk, G - i);
		uint32_t bits = 0;
		for (int k = 0; k < K; k++) {
			bits |= 1u << (L - 1 - wires[2 * (i + k)]);
			bits |= 1u << (L - 1 - wires[2 * (i + k) + 1]);
		}
		for (int b = 0; __builtin_popcount(bits) < NB && b < L; b++) bits |= 1u << b;
		Pass p;
		memset(&p.geom, 0, sizeof(p.geom));
		p.first = i;
		p.K = K;
		p.geom.K = K;
		p.geom.NB = NB;
		p.geom.L = L;
		int local[32];
		int n = 0;
		for (int b = 0; b < L; b++)
			if ((bits >> b) & 1) { local[b] = n; p.geom.tbit[n++] = b; }
		for (int k = 0; k < K; k++) {
			p.geom.gi[k] = local[L - 1 - wires[2 * (i + k)]];
			p.geom.gj[k] = local[L - 1 - wires[2 * (i + k) + 1]];
		}
		const uint32_t all = L >= 32 ? 0xffffffffu : ((1u << L) - 1);
		p.geom.rest_mask = all & ~bits;
		out.push_back(p);
		i += K;
	}
	return out;
}

template <typename T>
PassGates<T> pass_gates(const Pass& p, const double2* gates, const double2* dirs)
{
	PassGates<T> pg;
	memset(&pg, 0, sizeof(pg));
	for (int k = 0; k < p.K; k++)
		for (int e = 0; e < 16; e++) {
			const double2 g = gates[16 * (p.first + k) + e];
			pg.g[k].m[e] = mk<T>((T)g.x, (T)g.y);
			if (dirs) {
				const double2 z = dirs[16 * (p.first + k) + e];
				pg.z[k].m[e] = mk<T>((T)z.x, (T)z.y);
			}
		}
	return pg;
}

template <typename T>
size_t fwd_smem(int NB)
{
	return 32 * MAXK * sizeof(cplx<T>) + (1 << MAXNB) * sizeof(int) + 2 * ((size_t)1 << NB) * ColsPer<T>::v * sizeof(cplx<T>);
}

template <typename T>
size_t rev_smem(int NB, int K, bool tan)
{
	if (!std::is_same<T, double>::value) return k4_rev_smem(NB, K, tan);
	const size_t A = ((size_t)1 << NB) * ColsPer<T>::v;
	const size_t tiles = (tan ? 2 * K + 2 : K + 1) * A * sizeof(cplx<T>);
	const size_t red = std::is_same<T, double>::value ? (size_t)(NTR / 32) * MAXK * NPART3 * sizeof(double)
	                                                  : (TPB2 / 32) * 4 * MAXK * (tan ? 16 : 8) * sizeof(double);
	return 32 * MAXK * sizeof(cplx<T>) + (1 << MAXNB) * sizeof(int) + std::max(tiles, red);
}

template <typename KernelT>
int prepare(KernelT kernel, size_t smem, int* per_sm, int threads = TPB2)
{
	if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
		cudaGetLastError();
		fprintf(stderr, "rqcopt_gpu: cannot reserve %zu bytes of shared memory\n", smem);
		return E_CUDA;
	}
	int n = 0;
	if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, smem) != cudaSuccess || n < 1) {
		cudaGetLastError();
		n = 1;
	}
	*per_sm = n;
	return OK;
}

#define RQC_LAUNCH2(RT, CLS, KERNEL, GRID, SMEM, ...)                             \
	do {                                                                           \
		cudaEvent_t ev__;                                                          \
		launch_begin((RT), (CLS), &ev__);                                          \
		KERNEL<<<(GRID), TPB2, (SMEM), (RT).stream>>>(__VA_ARGS__);                \
		launch_end((RT), (CLS), ev__);                                             \
		if (int e__ = RQC_CUDA(cudaGetLastError())) return e__;                    \
	} while (0)

#define RQC_LAUNCH3(RT, CLS, KERNEL, GRID, NT, SMEM, ...)                         \
	do {                                                                           \
		cudaEvent_t ev__;                                                          \
		launch_begin((RT), (CLS), &ev__);                                          \
		KERNEL<<<(GRID), (NT), (SMEM), (RT).stream>>>(__VA_ARGS__);                \
		launch_end((RT), (CLS), ev__);                                             \
		if (int e__ = RQC_CUDA(cudaGetLastError())) return e__;                    \
	} while (0)

template <typename T, bool TAN, int IN, int OUT>
int launch_fwd(Runtime& rt, const cplx<T>* psi, const cplx<T>* dpsi, cplx<T>* psi_o, cplx<T>* dpsi_o, const cplx<T>* phi,
               const PassGeom& pg, const PassGates<T>& gates, double2* fpart, int fgrid)
{
	const size_t smem = fwd_smem<T>(pg.NB);
	static int per_sm = 0;
	if constexpr (std::is_same<T, double>::value) {
		if (!per_sm) {
			int ret = prepare(k3_fwd<TAN, IN, OUT>, k3_fwd_smem(MAXNB, TAN), &per_sm, NTF);
			if (ret) return ret;
		}
		const int grid = OUT >= 2 ? fgrid : (int)std::max<int64_t>(1, std::min<int64_t>(pg.ntiles, (int64_t)rt.num_sms * per_sm));
		RQC_LAUNCH3(rt, KC_FUSED, (k3_fwd<TAN, IN, OUT>), grid, NTF, k3_fwd_smem(pg.NB, TAN), psi, dpsi, psi_o, dpsi_o, phi,
		            pg, gates, fpart);
	} else if (rt.c64_ffma) {
		static int per_sm7 = 0;
		if (!per_sm7) {
			int ret = prepare(k7_fwd<TAN, IN, OUT>, k7_fwd_smem(), &per_sm7, NT7);
			if (ret) return ret;
		}
		const int grid = OUT >= 2 ? fgrid : (int)std::max<int64_t>(1, std::min<int64_t>(pg.ntiles, (int64_t)rt.num_sms * per_sm7));
		RQC_LAUNCH3(rt, KC_FUSED, (k7_fwd<TAN, IN, OUT>), grid, NT7, k7_fwd_smem(), psi, dpsi, psi_o, dpsi_o, phi, pg, gates,
		            fpart);
	} else {
		if (!per_sm) {
			int ret = prepare(k4_fwd<TAN, IN, OUT>, k4_fwd_smem(MAXNB, TAN, OUT >= 2), &per_sm, NT4F);
			if (ret) return ret;
		}
		const int grid = OUT >= 2 ? fgrid : (int)std::max<int64_t>(1, std::min<int64_t>(pg.ntiles, (int64_t)rt.num_sms * per_sm));
		RQC_LAUNCH3(rt, KC_FUSED, (k4_fwd<TAN, IN, OUT>), grid, NT4F, k4_fwd_smem(pg.NB, TAN, OUT >= 2), psi, dpsi, psi_o,
		            dpsi_o, phi, pg, gates, fpart);
	}
	return OK;
}

template <typename T, bool TAN, bool FIRST, bool LAST>
int launch_rev(Runtime& rt, const cplx<T>* psi, const cplx<T>* dpsi, const cplx<T>* phi, const cplx<T>* dphi,
               cplx<T>* phi_o, cplx<T>* dphi_o, const PassGeom& pg, const PassGates<T>& gates, double* part, int nblk,
               double* scratch)
{
	const size_t smem = rev_smem<T>(pg.NB, pg.K, TAN);
	static bool ready = false;
	if constexpr (std::is_same<T, double>::value) {
		if (!ready) {
			int per_sm;
			int ret = prepare(k3_rev<TAN, FIRST, LAST>, rev_smem<T>(MAXNB, MAXK, TAN), &per_sm, NTR);
			if (ret) return ret;
			ready = true;
		}
		RQC_LAUNCH3(rt, KC_REVERSE, (k3_rev<TAN, FIRST, LAST>), nblk, NTR, smem, psi, dpsi, phi, dphi, phi_o, dphi_o, pg,
		            gates, part, nblk);
	} else {
		if (!ready) {
			int per_sm;
			int ret = prepare(k4_rev<TAN, FIRST, LAST>, rev_smem<T>(MAXNB, MAXK, TAN), &per_sm, NT4R);
			if (ret) return ret;
			ready = true;
		}
		RQC_LAUNCH3(rt, KC_REVERSE, (k4_rev<TAN, FIRST, LAST>), nblk, NT4R, smem, psi, dpsi, phi, dphi, phi_o, dphi_o, pg,
		            gates, part, nblk, scratch);
	}
	return OK;
}

template <typename T, bool TAN>
int launch_rev_any(Runtime& rt, bool first, bool last, const cplx<T>* psi, const cplx<T>* dpsi, const cplx<T>* phi,
                   const cplx<T>* dphi, cplx<T>* phi_o, cplx<T>* dphi_o, const PassGeom& pg, const PassGates<T>& gates,
                   double* part, int nblk, double* scratch)
{
	if (first && last)
		return launch_rev<T, TAN, true, true>(rt, psi, dpsi, phi, dphi, phi_o, dphi_o, pg, gates, part, nblk, scratch);
	if (first)
		return launch_rev<T, TAN, true, false>(rt, psi, dpsi, phi, dphi, phi_o, dphi_o, pg, gates, part, nblk, scratch);
	if (last)
		return launch_rev<T, TAN, false, true>(rt, psi, dpsi, phi, dphi, phi_o, dphi_o, pg, gates, part, nblk, scratch);
	return launch_rev<T, TAN, false, false>(rt, psi, dpsi, phi, dphi, phi_o, dphi_o, pg, gates, part, nblk, scratch);
}

template <bool TAN, bool FIRST, bool LAST>
int launch_rev5(Runtime& rt, const float2* psi, const float2* dpsi, const float2* phi, const float2* dphi, float2* phi_o,
                float2* dphi_o, const PassGeom& pg, const PassGates<float>& gates, const PassW<float>& wg, double* part,
                int nblk, double* scratch)
{
	static bool ready = false;
	if (!ready) {
		int per_sm;
		int ret = prepare(k5_rev<TAN, FIRST, LAST>, k5_rev_smem(TAN), &per_sm, NT5);
		if (ret) return ret;
		ready = true;
	}
	RQC_LAUNCH3(rt, KC_REVERSE, (k5_rev<TAN, FIRST, LAST>), nblk, NT5, k5_rev_smem(TAN), psi, dpsi, phi, dphi, phi_o,
	            dphi_o, pg, gates, wg, part, nblk, scratch);
	return OK;
}

template <bool TAN>
int launch_rev5_any(Runtime& rt, bool first, bool last, const float2* psi, const float2* dpsi, const float2* phi,
                    const float2* dphi, float2* phi_o, float2* dphi_o, const PassGeom& pg, const PassGates<float>& gates,
                    const PassW<float>& wg, double* part, int nblk, double* scratch)
{
	if (first && last)
		return launch_rev5<TAN, true, true>(rt, psi, dpsi, phi, dphi, phi_o, dphi_o, pg, gates, wg, part, nblk, scratch);
	if (first)
		return launch_rev5<TAN, true, false>(rt, psi, dpsi, phi, dphi, phi_o, dphi_o, pg, gates, wg, part, nblk, scratch);
	if (last)
		return launch_rev5<TAN, false, true>(rt, psi, dpsi, phi, dphi, phi_o, dphi_o, pg, gates, wg, part, nblk, scratch);
	return launch_rev5<TAN, false, false>(rt, psi, dpsi, phi, dphi, phi_o, dphi_o, pg, gates, wg, part, nblk, scratch);
}

template <bool TAN, bool FIRST, bool LAST>
int launch_rev6(Runtime& rt, const double2* psi, const double2* dpsi, const double2* phi, const double2* dphi,
                double2* phi_o, double2* dphi_o, const PassGeom& pg, const PassGates<double>& gates, const PassAdj& adj,
                double* part, int nblk)
{
	static bool ready = false;
	if (!ready) {
		int per_sm;
		int ret = prepare(k6_rev<TAN, FIRST, LAST>, k6_rev_smem(TAN), &per_sm, NT6);
		if (ret) return ret;
		ready = true;
	}
	RQC_LAUNCH3(rt, KC_REVERSE, (k6_rev<TAN, FIRST, LAST>), nblk, NT6, k6_rev_smem(TAN), psi, dpsi, phi, dphi, phi_o,
	            dphi_o, pg, gates, adj, part, nblk);
	return OK;
}

template <bool TAN>
int launch_rev6_any(Runtime& rt, bool first, bool last, const double2* psi, const double2* dpsi, const double2* phi,
                    const double2* dphi, double2* phi_o, double2* dphi_o, const PassGeom& pg,
                    const PassGates<double>& gates, const PassAdj& adj, double* part, int nblk)
{
	if (first && last)
		return launch_rev6<TAN, true, true>(rt, psi, dpsi, phi, dphi, phi_o, dphi_o, pg, gates, adj, part, nblk);
	if (first)
		return launch_rev6<TAN, true, false>(rt, psi, dpsi, phi, dphi, phi_o, dphi_o, pg, gates, adj, part, nblk);
	if (last)
		return launch_rev6<TAN, false, true>(rt, psi, dpsi, phi, dphi, phi_o, dphi_o, pg, gates, adj, part, nblk);
	return launch_rev6<TAN, false, false>(rt, psi, dpsi, phi, dphi, phi_o, dphi_o, pg, gates, adj, part, nblk);
}

int rev_grid6(Runtime& rt, bool tan)
{
	int per_sm = 1;
	const int ret = tan ? prepare(k6_rev<true, false, false>, k6_rev_smem(true), &per_sm, NT6)
	                    : prepare(k6_rev<false, false, false>, k6_rev_smem(false), &per_sm, NT6);
	if (ret) per_sm = 1;
	return rt.num_sms * per_sm;
}

template <bool TAN, bool FIRST, bool LAST>
int launch_rev7(Runtime& rt, const float2* psi, const float2* dpsi, const float2* phi, const float2* dphi, float2* phi_o,
                float2* dphi_o, const PassGeom& pg, const PassGates<float>& gates, const PassW<float>& wg, double* part,
                int nblk)
{
	static bool ready = false;
	if (!ready) {
		int per_sm;
		int ret = prepare(k7_rev<TAN, FIRST, LAST>, k7_rev_smem(), &per_sm, NT7);
		if (ret) return ret;
		ready = true;
	}
	RQC_LAUNCH3(rt, KC_REVERSE, (k7_rev<TAN, FIRST, LAST>), nblk, NT7, k7_rev_smem(), psi, dpsi, phi, dphi, phi_o, dphi_o,
	            pg, gates, wg, part, nblk);
	return OK;
}

template <bool TAN>
int launch_rev7_any(Runtime& rt, bool first, bool last, const float2* psi, const float2* dpsi, const float2* phi,
                    const float2* dphi, float2* phi_o, float2* dphi_o, const PassGeom& pg, const PassGates<float>& gates,
                    const PassW<float>& wg, double* part, int nblk)
{
	if (first && last)
		return launch_rev7<TAN, true, true>(rt, psi, dpsi, phi, dphi, phi_o, dphi_o, pg, gates, wg, part, nblk);
	if (first)
		return launch_rev7<TAN, true, false>(rt, psi, dpsi, phi, dphi, phi_o, dphi_o, pg, gates, wg, part, nblk);
	if (last)
		return launch_rev7<TAN, false, true>(rt, psi, dpsi, phi, dphi, phi_o, dphi_o, pg, gates, wg, part, nblk);
	return launch_rev7<TAN, false, false>(rt, psi, dpsi, phi, dphi, phi_o, dphi_o, pg, gates, wg, part, nblk);
}

int rev_grid7(Runtime& rt, bool tan)
{
	int per_sm = 1;
	const int ret = tan ? prepare(k7_rev<true, false, false>, k7_rev_smem(), &per_sm, NT7)
	                    : prepare(k7_rev<false, false, false>, k7_rev_smem(), &per_sm, NT7);
	if (ret) per_sm = 1;
	return rt.num_sms * per_sm;
}

int rev_grid5(Runtime& rt, bool tan)
{
	int per_sm = 1;
	const int ret = tan ? prepare(k5_rev<true, false, false>, k5_rev_smem(true), &per_sm, NT5)
	                    : prepare(k5_rev<false, false, false>, k5_rev_smem(false), &per_sm, NT5);
	if (ret) per_sm = 1;
	return rt.num_sms * per_sm;
}

// every gate unitary to `tol` (max |G^+ G - I|): the reverse pass may then rebuild
// states with adjoint gates (1e-10 for complex64 passes; complex128 passes, which must
// agree with the reference to 1e-12, ask for 1e-14)
bool gates_unitary(const double2* gates, int G, double tol = 1e-10)
{
	for (int k = 0; k < G; k++) {
		const double2* g = gates + 16 * (size_t)k;
		for (int r = 0; r < 4; r++)
			for (int c = 0; c < 4; c++) {
				double re = 0, im = 0;
				for (int q = 0; q < 4; q++) {   // (G^+ G)[r][c] = sum_q conj(G[q][r]) G[q][c]
					const double2 a = g[4 * q + r], b = g[4 * q + c];
					re += a.x * b.x + a.y * b.y;
					im += a.x * b.y - a.y * b.x;
				}
				if (fabs(re - (r == c ? 1.0 : 0.0)) > tol || fabs(im) > tol) return false;
			}
	}
	return true;
}

// conj(G) and -W = -G^+ Z G^+ of every gate of a pass, in FP64 (complex128 reconstruction)
PassAdj pass_adj(const Pass& p, const double2* gates, const double2* dirs)
{
	PassAdj pa;
	memset(&pa, 0, sizeof(pa));
	for (int k = 0; k < p.K; k++) {
		const double2* g = gates + 16 * (size_t)(p.first + k);
		for (int e = 0; e < 16; e++) pa.gc[k].m[e] = make_double2(g[e].x, -g[e].y);
		if (!dirs) continue;
		const double2* z = dirs + 16 * (size_t)(p.first + k);
		double2 gh[16], t[16], w[16];
		for (int r = 0; r < 4; r++)
			for (int c = 0; c < 4; c++) gh[4 * r + c] = make_double2(g[4 * c + r].x, -g[4 * c + r].y);
		auto mul = [](const double2* a, const double2* b, double2* o) {
			for (int r = 0; r < 4; r++)
				for (int c = 0; c < 4; c++) {
					double re = 0, im = 0;
					for (int q = 0; q < 4; q++) {
						const double2 x = a[4 * r + q], y = b[4 * q + c];
						re += x.x * y.x - x.y * y.y;
						im += x.x * y.y + x.y * y.x;
					}
					o[4 * r + c] = make_double2(re, im);
				}
		};
		mul(gh, z, t);
		mul(t, gh, w);
		for (int e = 0; e < 16; e++) pa.wn[k].m[e] = make_double2(-w[e].x, -w[e].y);
	}
	return pa;
}

// W = G^+ Z G^+ of every gate of a pass
PassW<float> pass_w(const Pass& p, const double2* gates, const double2* dirs)
{
	PassW<float> pw;
	memset(&pw, 0, sizeof(pw));
	for (int k = 0; k < p.K; k++) {
		const double2* g = gates + 16 * (size_t)(p.first + k);
		const double2* z = dirs + 16 * (size_t)(p.first + k);
		double2 gh[16], t[16];
		for (int r = 0; r < 4; r++)
			for (int c = 0; c < 4; c++) gh[4 * r + c] = make_double2(g[4 * c + r].x, -g[4 * c + r].y);
		auto mul = [](const double2* a, const double2* b, double2* o) {
			for (int r = 0; r < 4; r++)
				for (int c = 0; c < 4; c++) {
					double re = 0, im = 0;
					for (int q = 0; q < 4; q++) {
						const double2 x = a[4 * r + q], y = b[4 * q + c];
						re += x.x * y.x - x.y * y.y;
						im += x.x * y.y + x.y * y.x;
					}
					o[4 * r + c] = make_double2(re, im);
				}
		};
		mul(gh, z, t);
		double2 w[16];
		mul(t, gh, w);
		for (int e = 0; e < 16; e++) pw.w[k].m[e] = make_float2((float)w[e].x, (float)w[e].y);
	}
	return pw;
}

// grid of the partial-sum kernels: one resident wave of the reverse kernel
template <typename T>
int rev_grid(Runtime& rt, bool tan)
{
	int per_sm = 1;
	const size_t smem = rev_smem<T>(MAXNB, MAXK, tan);
	int ret;
	if constexpr (std::is_same<T, double>::value)
		ret = tan ? prepare(k3_rev<true, false, false>, smem, &per_sm, NTR)
		          : prepare(k3_rev<false, false, false>, smem, &per_sm, NTR);
	else
		ret = tan ? prepare(k4_rev<true, false, false>, smem, &per_sm, NT4R)
		          : prepare(k4_rev<false, false, false>, smem, &per_sm, NT4R);
	if (ret) per_sm = 1;
	return rt.num_sms * per_sm;
}

size_t workspace_limit2(Runtime& rt)
{
	if (rt.workspace_limit) return rt.workspace_limit;
	size_t free_b = 0, total_b = 0;
	if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
		cudaGetLastError();
		return (size_t)1 << 30;
	}
	return (size_t)((free_b + rt.work.bytes) * 0.75);
}

template <typename T>
int evaluate_fused_t(Runtime& rt, const CircuitSpec& c, const TargetSpec& t, int mode, int maxk, double2* d_out)
{
	using V = cplx<T>;
	constexpr int CW = ColsPer<T>::v;
	const int L = c.L, G = c.ngates;
	const int64_t N = (int64_t)1 << L;
	const int64_t ncols = rt.real_pairs ? N / 2 : N;   // (paired) basis columns
	const bool tan = mode == EVAL_HVP;
	const bool host_target = t.ufunc != nullptr;
	std::vector<Pass> passes = schedule(L, G, c.wires, maxk);
	std::vector<Pass> tpasses = host_target ? std::vector<Pass>() : schedule(L, t.ngates, t.wires, maxk);
	const int P = (int)passes.size(), Pt = (int)tpasses.size();
	std::vector<PassGates<T>> pgates(P), tgates(Pt);
	for (int p = 0; p < P; p++) pgates[p] = pass_gates<T>(passes[p], c.gates, tan ? c.dirs : nullptr);
	for (int p = 0; p < Pt; p++) tgates[p] = pass_gates<T>(tpasses[p], t.gates, nullptr);

	// complex64 with unitary gates: the reverse passes start from each pass's output
	// (the next checkpoint, or the final state) and rebuild states with adjoint gates
	bool recon = false;
	if constexpr (!std::is_same<T, double>::value) recon = mode != EVAL_F && gates_unitary(c.gates, G);
	else recon = mode != EVAL_F && rt.recon_c128 && gates_unitary(c.gates, G, 1e-14);
	std::vector<PassW<float>> pw(recon && tan && !std::is_same<T, double>::value ? P : 0);
	for (int p = 0; p < (int)pw.size(); p++) pw[p] = pass_w(passes[p], c.gates, c.dirs);
	std::vector<PassAdj> padj(recon && std::is_same<T, double>::value ? P : 0);
	for (int p = 0; p < (int)padj.size(); p++) padj[p] = pass_adj(passes[p], c.gates, tan ? c.dirs : nullptr);
	const int64_t nck = recon ? P : P - 1;   // checkpoints (recon: also the final state)

	// states per column: PHI, P0, P1 (+ D0, D1) and the pass checkpoints
	const int64_t nstates = mode == EVAL_F ? 3 : (mode == EVAL_GRAD ? 3 + nck : 5 + 2 * nck);
	const size_t col_bytes = (size_t)nstates * N * sizeof(V);
	const int64_t cbeg = std::min<int64_t>(rt.col_begin, ncols);
	const int64_t cend = rt.col_end > 0 ? std::min<int64_t>(rt.col_end, ncols) : ncols;
	const int64_t C_mem = (int64_t)(workspace_limit2(rt) / col_bytes);
	int64_t C = C_mem;
	if (rt.column_chunk > 0) C = std::min<int64_t>(C, ((rt.column_chunk + CW - 1) / CW) * CW);
	if (host_target) C = std::min<int64_t>(C, std::max<int64_t>(CW, ((int64_t)256 << 20) / (N * 16)));
	C = std::min<int64_t>(C, ((std::max<int64_t>(1, cend - cbeg) + CW - 1) / CW) * CW);
	C = (C / CW) * CW;
	if (C < CW || C > C_mem) {
		fprintf(stderr, "rqcopt_gpu: %d columns need %zu bytes of workspace, more than the limit\n", CW, CW * col_bytes);
		return E_ALLOC;
	}
	int ret = ensure_device(rt.work, (size_t)nstates * C * N * sizeof(V));
	if (ret) return ret;
	V* PHI = reinterpret_cast<V*>(rt.work.ptr);
	V* Pb[2] = { PHI + C * N, PHI + 2 * C * N };
	V* Db[2] = { tan ? PHI + 3 * C * N : nullptr, tan ? PHI + 4 * C * N : nullptr };
	V* ck = PHI + (tan ? 5 : 3) * C * N;                             // psi at the input of pass p = 1..nck
	V* dck = tan ? ck + nck * C * N : nullptr;                       // dpsi at the input of pass p
	auto ck_at = [&](int p) { return ck + (int64_t)(p - 1) * C * N; };
	auto dck_at = [&](int p) { return dck + (int64_t)(p - 1) * C * N; };

	// complex64 reverse passes on the FP32 pipe (k7_rev) or on the TF32 MMA (k5_rev)
	const bool ffma = !std::is_same<T, double>::value && recon && rt.c64_ffma;
	const int nblk = recon ? (std::is_same<T, double>::value ? rev_grid6(rt, tan) : (ffma ? rev_grid7(rt, tan) : rev_grid5(rt, tan)))
	                       : rev_grid<T>(rt, tan);
	// blocks of the forward launches that sum f (one FP64 partial each)
	const int nfb = std::is_same<T, double>::value ? nblk : 2 * rt.num_sms;
	const int nps = std::is_same<T, double>::value ? NPART3 : (ffma ? NPART2 : NRAW4);   // partial doubles per gate and block
	const size_t part_doubles = (size_t)G * nblk * nps + 2 * (size_t)nfb;
	if ((ret = ensure_device(rt.partials, part_doubles * sizeof(double)))) return ret;
	double* part = reinterpret_cast<double*>(rt.partials.ptr);
	double2* fpart = reinterpret_cast<double2*>(part + (size_t)G * nblk * nps);
	if ((ret = RQC_CUDA(cudaMemsetAsync(part, 0, part_doubles * sizeof(double), rt.stream)))) return ret;
	double* scratch = nullptr;
	if (!std::is_same<T, double>::value) {
		if ((ret = ensure_device(rt.scratch, (size_t)nblk * (NT4R / 32) * 32 * MAXK * 4 * sizeof(double)))) return ret;
		scratch = reinterpret_cast<double*>(rt.scratch.ptr);
	}

	double2* hcols = nullptr;
	double2* hbasis = nullptr;
	double2* dstage = nullptr;
	if (host_target) {
		if ((ret = ensure_host_pinned(rt.hpin, (size_t)(C + 1) * N * sizeof(double2)))) return ret;
		hcols = reinterpret_cast<double2*>(rt.hpin.ptr);
		hbasis = hcols + C * N;
		if ((ret = ensure_device(rt.stage[2], (size_t)C * N * sizeof(double2)))) return ret;
		dstage = reinterpret_cast<double2*>(rt.stage[2].ptr);
	}

	if (cend != rt.col_end_dev) {   // a copy from host memory waits for the stream: only when it changes
		if ((ret = RQC_CUDA(cudaMemcpyToSymbolAsync(c_col_end, &cend, sizeof(cend), 0, cudaMemcpyHostToDevice, rt.stream))))
			return ret;
		rt.col_end_dev = cend;
	}
	for (int64_t b0 = cbeg; b0 < cend; b0 += C) {
		const int64_t Cc = std::min(C, cend - b0);
		const int64_t ncg = (Cc + CW - 1) / CW;
		auto geom = [&](const Pass& p) {
			PassGeom g = p.geom;
			g.C = C;
			g.ncg = ncg;
			g.ntiles = ((int64_t)1 << (L - g.NB)) * ncg;
			g.b0 = b0;
			return g;
		};

		// target columns phi = -conj(U e_b)
		if (host_target) {
			const linear_func uf = reinterpret_cast<linear_func>(t.ufunc);
			for (int64_t j = 0; j < Cc; j++) {
				memset(hbasis, 0, N * sizeof(double2));
				hbasis[b0 + j].x = 1;
				if (rt.real_pairs) hbasis[b0 + j + N / 2].y = 1;
				statevector e = { reinterpret_cast<numeric*>(hbasis), L };
				statevector u = { reinterpret_cast<numeric*>(hcols + j * N), L };
				const int r = uf(&e, t.udata, &u);
				if (r < 0) {
					fprintf(stderr, "rqcopt_gpu: call of 'ufunc' failed, return value: %i\n", r);
					return E_UFUNC;
				}
			}
			if ((ret = RQC_CUDA(cudaMemcpyAsync(dstage, hcols, Cc * N * sizeof(double2), cudaMemcpyHostToDevice, rt.stream))))
				return ret;
			k2_target_from_host<T><<<rt.num_sms * 8, 256, 0, rt.stream>>>(dstage, PHI, N, Cc, C);
			rt.launches++;
			if ((ret = RQC_CUDA(cudaGetLastError()))) return ret;
			if ((ret = RQC_CUDA(cudaStreamSynchronize(rt.stream)))) return ret;
		} else {
			for (int p = 0; p < Pt; p++) {
				const PassGeom g = geom(tpasses[p]);
				const bool first = p == 0, last = p == Pt - 1;
				const V* in = first ? nullptr : Pb[(p - 1) & 1];
				V* out = last ? PHI : Pb[p & 1];
				if (first && last) ret = launch_fwd<T, false, 1, 1>(rt, in, nullptr, out, nullptr, nullptr, g, tgates[p], nullptr, 0);
				else if (first) ret = launch_fwd<T, false, 1, 0>(rt, in, nullptr, out, nullptr, nullptr, g, tgates[p], nullptr, 0);
				else if (last) ret = launch_fwd<T, false, 0, 1>(rt, in, nullptr, out, nullptr, nullptr, g, tgates[p], nullptr, 0);
				else ret = launch_fwd<T, false, 0, 0>(rt, in, nullptr, out, nullptr, nullptr, g, tgates[p], nullptr, 0);
				if (ret) return ret;
			}
		}

		// forward passes
		for (int p = 0; p < P; p++) {
			const PassGeom g = geom(passes[p]);
			const bool first = p == 0, last = p == P - 1;
			if (mode == EVAL_F) {
				const V* in = first ? nullptr : Pb[(p - 1) & 1];
				V* out = last ? nullptr : Pb[p & 1];
				if (first && last) ret = launch_fwd<T, false, 1, 2>(rt, in, nullptr, out, nullptr, PHI, g, pgates[p], fpart, nfb);
				else if (first) ret = launch_fwd<T, false, 1, 0>(rt, in, nullptr, out, nullptr, PHI, g, pgates[p], fpart, nfb);
				else if (last) ret = launch_fwd<T, false, 0, 2>(rt, in, nullptr, out, nullptr, PHI, g, pgates[p], fpart, nfb);
				else ret = launch_fwd<T, false, 0, 0>(rt, in, nullptr, out, nullptr, PHI, g, pgates[p], fpart, nfb);
			} else if (!tan) {
				const V* in = first ? nullptr : ck_at(p);
				V* out = (last && !recon) ? nullptr : ck_at(p + 1);
				if (recon && last) {
					if (first) ret = launch_fwd<T, false, 1, 3>(rt, in, nullptr, out, nullptr, PHI, g, pgates[p], fpart, nfb);
					else ret = launch_fwd<T, false, 0, 3>(rt, in, nullptr, out, nullptr, PHI, g, pgates[p], fpart, nfb);
				} else if (first && last) ret = launch_fwd<T, false, 1, 2>(rt, in, nullptr, out, nullptr, PHI, g, pgates[p], fpart, nfb);
				else if (first) ret = launch_fwd<T, false, 1, 0>(rt, in, nullptr, out, nullptr, PHI, g, pgates[p], fpart, nfb);
				else if (last) ret = launch_fwd<T, false, 0, 2>(rt, in, nullptr, out, nullptr, PHI, g, pgates[p], fpart, nfb);
				else ret = launch_fwd<T, false, 0, 0>(rt, in, nullptr, out, nullptr, PHI, g, pgates[p], fpart, nfb);
			} else {
				const V* in = first ? nullptr : ck_at(p);
				const V* din = first ? nullptr : dck_at(p);
				V* out = (last && !recon) ? nullptr : ck_at(p + 1);
				V* dout = (last && !recon) ? nullptr : dck_at(p + 1);
				if (recon && last) {
					if (first) ret = launch_fwd<T, true, 1, 3>(rt, in, din, out, dout, PHI, g, pgates[p], fpart, nfb);
					else ret = launch_fwd<T, true, 0, 3>(rt, in, din, out, dout, PHI, g, pgates[p], fpart, nfb);
				} else if (first && last) ret = launch_fwd<T, true, 1, 2>(rt, in, din, out, dout, PHI, g, pgates[p], fpart, nfb);
				else if (first) ret = launch_fwd<T, true, 1, 0>(rt, in, din, out, dout, PHI, g, pgates[p], fpart, nfb);
				else if (last) ret = launch_fwd<T, true, 0, 2>(rt, in, din, out, dout, PHI, g, pgates[p], fpart, nfb);
				else ret = launch_fwd<T, true, 0, 0>(rt, in, din, out, dout, PHI, g, pgates[p], fpart, nfb);
			}
			if (ret) return ret;
		}
		if (mode == EVAL_F) continue;

		// reverse passes
		for (int p = P - 1; p >= 0; p--) {
			const PassGeom g = geom(passes[p]);
			const bool first = p == P - 1, last = p == 0;
			const int cur = (P - 1 - p) & 1, nxt = cur ^ 1;
			const V* ph = first ? PHI : Pb[cur];
			const V* dph = (first || !tan) ? nullptr : Db[cur];
			double* pp = part + (size_t)passes[p].first * nblk * nps;
			if constexpr (std::is_same<T, double>::value) {
				if (recon) {
					if (tan)
						ret = launch_rev6_any<true>(rt, first, last, ck_at(p + 1), dck_at(p + 1), ph, dph,
						                            last ? nullptr : Pb[nxt], last ? nullptr : Db[nxt], g, pgates[p], padj[p],
						                            pp, nblk);
					else
						ret = launch_rev6_any<false>(rt, first, last, ck_at(p + 1), nullptr, ph, nullptr,
						                             last ? nullptr : Pb[nxt], nullptr, g, pgates[p], padj[p], pp, nblk);
					if (ret) return ret;
					continue;
				}
			}
			if constexpr (!std::is_same<T, double>::value) {
				if (ffma) {
					if (tan)
						ret = launch_rev7_any<true>(rt, first, last, ck_at(p + 1), dck_at(p + 1), ph, dph,
						                            last ? nullptr : Pb[nxt], last ? nullptr : Db[nxt], g, pgates[p], pw[p],
						                            pp, nblk);
					else
						ret = launch_rev7_any<false>(rt, first, last, ck_at(p + 1), nullptr, ph, nullptr,
						                             last ? nullptr : Pb[nxt], nullptr, g, pgates[p], PassW<float>{}, pp, nblk);
					if (ret) return ret;
					continue;
				}
				if (recon) {
					if (tan)
						ret = launch_rev5_any<true>(rt, first, last, ck_at(p + 1), dck_at(p + 1), ph, dph,
						                            last ? nullptr : Pb[nxt], last ? nullptr : Db[nxt], g, pgates[p], pw[p],
						                            pp, nblk, scratch);
					else
						ret = launch_rev5_any<false>(rt, first, last, ck_at(p + 1), nullptr, ph, nullptr,
						                             last ? nullptr : Pb[nxt], nullptr, g, pgates[p], PassW<float>{}, pp,
						                             nblk, scratch);
					if (ret) return ret;
					continue;
				}
			}
			if (tan)
				ret = launch_rev_any<T, true>(rt, first, last, last ? nullptr : ck_at(p), last ? nullptr : dck_at(p), ph, dph,
				                              last ? nullptr : Pb[nxt], last ? nullptr : Db[nxt], g, pgates[p], pp, nblk,
				                              scratch);
			else
				ret = launch_rev_any<T, false>(rt, first, last, last ? nullptr : ck_at(p), nullptr, ph, nullptr,
				                               last ? nullptr : Pb[nxt], nullptr, g, pgates[p], pp, nblk, scratch);
			if (ret) return ret;
		}
	}

	if (std::is_same<T, double>::value)
		k3_reduce<<<G + 1, NPART3, 0, rt.stream>>>(part, G, nblk, fpart, nfb, tan ? 1 : 0, d_out);
	else if (ffma)
		k2_reduce<<<G + 1, NPART2, 0, rt.stream>>>(part, G, nblk, fpart, nfb, tan ? 1 : 0, d_out);
	else
		k4_reduce<<<G + 1, NRAW4, 0, rt.stream>>>(part, G, nblk, fpart, nfb, tan ? 1 : 0, d_out);
	rt.launches++;
	return RQC_CUDA(cudaGetLastError());
}

}  // namespace

int set_pair_half_fused(Runtime& rt, int64_t half)
{
	return RQC_CUDA(cudaMemcpyToSymbolAsync(c_pair_half, &half, sizeof(half), 0, cudaMemcpyHostToDevice, rt.stream));
}

int evaluate_fused(Runtime& rt, const CircuitSpec& c, const TargetSpec& t, int mode, int precision, int maxk, double2* d_out)
{
	maxk = std::max(1, std::min(MAXK, maxk));
	int ret;
	if ((ret = RQC_CUDA(cudaMemsetAsync(d_out, 0, result_count(c.ngates) * sizeof(double2), rt.stream)))) return ret;
	if (mode != EVAL_GRAD && mode != EVAL_HVP) mode = EVAL_F;
	if (precision == PREC_C128) return evaluate_fused_t<double>(rt, c, t, mode, maxk, d_out);
	return evaluate_fused_t<float>(rt, c, t, mode, maxk, d_out);
}

}  // namespace rqc
