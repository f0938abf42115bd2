// Shared device helpers: complex arithmetic on double2/float2 and the
// amplitude-group index arithmetic of a two-qubit gate.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace rqc {

// ---------------------------------------------------------------- complex types

template <typename T> struct cplx_t;
template <> struct cplx_t<double> { using type = double2; };
template <> struct cplx_t<float>  { using type = float2; };
template <typename T> using cplx = typename cplx_t<T>::type;

template <typename T> __host__ __device__ __forceinline__ cplx<T> mk(T re, T im) { cplx<T> z; z.x = re; z.y = im; return z; }

// a * b + c
template <typename V> __host__ __device__ __forceinline__ V cfma(V a, V b, V c)
{
	V r;
	r.x = fma(a.x, b.x, fma(-a.y, b.y, c.x));
	r.y = fma(a.x, b.y, fma(a.y, b.x, c.y));
	return r;
}
template <typename V> __host__ __device__ __forceinline__ V cmul(V a, V b)
{
	V r;
	r.x = a.x * b.x - a.y * b.y;
	r.y = a.x * b.y + a.y * b.x;
	return r;
}
template <typename V> __host__ __device__ __forceinline__ V cadd(V a, V b) { V r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename V> __host__ __device__ __forceinline__ V csub(V a, V b) { V r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <typename V> __host__ __device__ __forceinline__ V cneg_conj(V a) { V r; r.x = -a.x; r.y = a.y; return r; }
template <typename V> __host__ __device__ __forceinline__ V czero() { V r; r.x = 0; r.y = 0; return r; }

__device__ __forceinline__ double2 to_d(double2 a) { return a; }
__device__ __forceinline__ double2 to_d(float2 a) { return make_double2(a.x, a.y); }

// ---------------------------------------------------------------- gates as kernel arguments

// One 4x4 gate in arithmetic precision T, row-major (row = 2*b_i + b_j).
template <typename T> struct Gate4 { cplx<T> m[16]; };

// ---------------------------------------------------------------- amplitude groups

// Wire pair of a gate acting on an L-qubit register: bit positions of the two
// wires (qubit q <-> index bit L-1-q) and the two positions sorted, for the
// insertion of zero bits into a rest index.
struct WirePair
{
	int64_t si, sj;   // strides of wire i and wire j
	int plo, phi;     // sorted bit positions
};

__host__ __device__ __forceinline__ WirePair make_pair_(int L, int i, int j)
{
	WirePair w;
	const int pi = L - 1 - i, pj = L - 1 - j;
	w.si = (int64_t)1 << pi;
	w.sj = (int64_t)1 << pj;
	w.plo = pi < pj ? pi : pj;
	w.phi = pi < pj ? pj : pi;
	return w;
}

// Base index (both wire bits zero) of the rest index r in [0, 2^(L-2)).
__host__ __device__ __forceinline__ int64_t group_base(int64_t r, const WirePair& w)
{
	const int64_t mlo = ((int64_t)1 << w.plo) - 1;
	r = ((r & ~mlo) << 1) | (r & mlo);
	const int64_t mhi = ((int64_t)1 << w.phi) - 1;
	r = ((r & ~mhi) << 1) | (r & mhi);
	return r;
}

// Offsets of the four group members in the order of the gate's row index.
__host__ __device__ __forceinline__ void group_offsets(const WirePair& w, int64_t off[4])
{
	off[0] = 0;
	off[1] = w.sj;
	off[2] = w.si;
	off[3] = w.si + w.sj;
}

// ---------------------------------------------------------------- 4x4 actions on a group

// y = G x
template <typename T>
__device__ __forceinline__ void gate_apply(const Gate4<T>& g, const cplx<T> x[4], cplx<T> y[4])
{
#pragma unroll
	for (int r = 0; r < 4; r++) {
		cplx<T> s = cmul(g.m[4*r], x[0]);
#pragma unroll
		for (int c = 1; c < 4; c++) s = cfma(g.m[4*r + c], x[c], s);
		y[r] = s;
	}
}

// y = G^T x
template <typename T>
__device__ __forceinline__ void gate_apply_t(const Gate4<T>& g, const cplx<T> x[4], cplx<T> y[4])
{
#pragma unroll
	for (int c = 0; c < 4; c++) {
		cplx<T> s = cmul(g.m[c], x[0]);
#pragma unroll
		for (int r = 1; r < 4; r++) s = cfma(g.m[4*r + c], x[r], s);
		y[c] = s;
	}
}

// y += G x
template <typename T>
__device__ __forceinline__ void gate_apply_acc(const Gate4<T>& g, const cplx<T> x[4], cplx<T> y[4])
{
#pragma unroll
	for (int r = 0; r < 4; r++) {
		cplx<T> s = y[r];
#pragma unroll
		for (int c = 0; c < 4; c++) s = cfma(g.m[4*r + c], x[c], s);
		y[r] = s;
	}
}

// y += G^T x
template <typename T>
__device__ __forceinline__ void gate_apply_t_acc(const Gate4<T>& g, const cplx<T> x[4], cplx<T> y[4])
{
#pragma unroll
	for (int c = 0; c < 4; c++) {
		cplx<T> s = y[c];
#pragma unroll
		for (int r = 0; r < 4; r++) s = cfma(g.m[4*r + c], x[r], s);
		y[c] = s;
	}
}

// acc[r][c] += a[r] * b[c]  (no conjugation)
template <typename A, typename V>
__device__ __forceinline__ void outer_acc(A acc[16], const V a[4], const V b[4])
{
#pragma unroll
	for (int r = 0; r < 4; r++)
#pragma unroll
		for (int c = 0; c < 4; c++) {
			A p;
			p.x = a[r].x * b[c].x - a[r].y * b[c].y;
			p.y = a[r].x * b[c].y + a[r].y * b[c].x;
			acc[4*r + c].x += p.x;
			acc[4*r + c].y += p.y;
		}
}

// ---------------------------------------------------------------- reductions

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	return v;
}

}  // namespace rqc
