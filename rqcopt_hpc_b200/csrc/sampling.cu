// Haar-random sample states and the sampled target value (see sampling.h).
//
// The reference draws sample b's amplitude j as crandn() = (randn() + i randn()) / sqrt(2)
// with randn() the Box-Muller transform of two uniforms u = 2^-64 * rand_uint64(),
// each rand_uint64() one step of both PCG32 generators (src/rng.c:100-157,
// src/pcg_basic.c:128-132), sequentially over samples and amplitudes, then
// normalises the state (src/statevector.c:47-66, 102-125).  Here every thread
// jumps both generators directly to its first amplitude's position in that
// stream (4 steps per amplitude; LCG jump-ahead as in F. Brown, "Random number
// generation with arbitrary strides", 1994) and draws a run of consecutive
// amplitudes, so the states are the reference's up to the last-bit differences of
// the device log and sin; one block per sample then normalises.
#include "sampling.h"

#include <stdio.h>
#include <algorithm>

#include "rqc_common.cuh"

namespace rqc {

namespace {

constexpr uint64_t PCG_MULT = 6364136223846793005ULL;
constexpr int HRUN = 8;     // consecutive amplitudes per thread
constexpr int HTPB = 256;

__host__ __device__ inline uint32_t pcg_output(uint64_t old)
{
	const uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
	const uint32_t rot = (uint32_t)(old >> 59u);
	return (xs >> rot) | (xs << ((32u - rot) & 31u));
}

// state after delta steps of state -> state * PCG_MULT + inc (mod 2^64)
__host__ __device__ inline uint64_t pcg_jump(uint64_t state, uint64_t inc, uint64_t delta)
{
	uint64_t acc_mult = 1, acc_plus = 0, cur_mult = PCG_MULT, cur_plus = inc;
	while (delta) {
		if (delta & 1) {
			acc_mult *= cur_mult;
			acc_plus = acc_plus * cur_mult + cur_plus;
		}
		cur_plus = (cur_mult + 1) * cur_plus;
		cur_mult *= cur_mult;
		delta >>= 1;
	}
	return acc_mult * state + acc_plus;
}

struct Gen2
{
	uint64_t s0, i0, s1, i1;

	__device__ uint64_t next64()
	{
		const uint64_t o0 = s0, o1 = s1;
		s0 = o0 * PCG_MULT + i0;
		s1 = o1 * PCG_MULT + i1;
		return ((uint64_t)pcg_output(o0) << 32) | pcg_output(o1);
	}

	// Box-Muller standard normal from two uniforms on [0, 1) (u1 = 0 replaced by 1)
	__device__ double randn()
	{
		double u1 = (double)next64() * 0x1p-64;
		const double u2 = (double)next64() * 0x1p-64;
		if (u1 == 0) u1 = 1;
		return sqrt(-2 * log(u1)) * sin(6.2831853071795864769 * u2);
	}
};

// unnormalised complex (or, with sp.real, real) normal amplitudes of samples s0 .. s0 + total / 2^L - 1
__global__ void __launch_bounds__(HTPB) k_haar(SampleSpec sp, int L, int64_t s0, int64_t total, double2* __restrict__ out)
{
	const double rs2 = sqrt(2.0);
	for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r * HRUN < total;
	     r += (int64_t)gridDim.x * blockDim.x) {
		const int64_t a0 = r * HRUN;
		const uint64_t d = (sp.real ? 2 : 4) * (uint64_t)((s0 << L) + a0);
		Gen2 g{ pcg_jump(sp.state[0], sp.inc[0], d), sp.inc[0], pcg_jump(sp.state[1], sp.inc[1], d), sp.inc[1] };
		const int n = (int)min((int64_t)HRUN, total - a0);
		if (sp.real) {
			for (int k = 0; k < n; k++) out[a0 + k] = make_double2(g.randn(), 0.0);
		} else {
			for (int k = 0; k < n; k++) {
				const double x = g.randn();
				const double y = g.randn();
				out[a0 + k] = make_double2(x / rs2, y / rs2);
			}
		}
	}
}

// one block per sample: divide by the 2-norm (unless zero)
__global__ void __launch_bounds__(HTPB) k_normalize(double2* __restrict__ psi, int L)
{
	__shared__ double red[HTPB / 32];
	const int64_t N = (int64_t)1 << L;
	double2* p = psi + (int64_t)blockIdx.x * N;
	double s = 0;
	for (int64_t j = threadIdx.x; j < N; j += HTPB) s += p[j].x * p[j].x + p[j].y * p[j].y;
	s = warp_sum(s);
	if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
	__syncthreads();
	double tot = 0;
	for (int k = 0; k < HTPB / 32; k++) tot += red[k];
	const double nrm = sqrt(tot);
	if (nrm > 0) {
		const double a = 1. / nrm;
		for (int64_t j = threadIdx.x; j < N; j += HTPB) p[j] = make_double2(p[j].x * a, p[j].y * a);
	}
}

// fpart[block] += sum over its elements of phi * cpsi (no conjugation)
__global__ void __launch_bounds__(HTPB) k_fdot(const double2* __restrict__ phi, const double2* __restrict__ cpsi, int64_t n,
                                                double2* __restrict__ fpart)
{
	__shared__ double red[2][HTPB / 32];
	double fx = 0, fy = 0;
	for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
		const double2 a = phi[i], b = cpsi[i];
		fx += a.x * b.x - a.y * b.y;
		fy += a.x * b.y + a.y * b.x;
	}
	fx = warp_sum(fx);
	fy = warp_sum(fy);
	if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = fx; red[1][threadIdx.x >> 5] = fy; }
	__syncthreads();
	if (threadIdx.x == 0) {
		double sx = 0, sy = 0;
		for (int k = 0; k < HTPB / 32; k++) { sx += red[0][k]; sy += red[1][k]; }
		fpart[blockIdx.x].x += sx;
		fpart[blockIdx.x].y += sy;
	}
}

// f = scale * sum over blocks
__global__ void k_fsum(const double2* __restrict__ fpart, int nblk, double scale, double2* __restrict__ f)
{
	if (threadIdx.x | blockIdx.x) return;
	double sx = 0, sy = 0;
	for (int b = 0; b < nblk; b++) { sx += fpart[b].x; sy += fpart[b].y; }
	f[0] = make_double2(sx * scale, sy * scale);
}

size_t sampling_workspace_limit(Runtime& rt)
{
	if (rt.workspace_limit) return rt.workspace_limit;
	size_t free_b = 0, total_b = 0;
	if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
		cudaGetLastError();
		return (size_t)1 << 30;
	}
	return (size_t)((free_b + rt.work.bytes) * 0.75);
}

int g_real_samples = 0;

}  // namespace

int real_samples() { return g_real_samples; }

void set_real_samples(int on) { g_real_samples = on ? 1 : 0; }

void pcg_advance_host(uint64_t& state, uint64_t inc, uint64_t delta)
{
	state = pcg_jump(state, inc, delta);
}

int haar_states_device(Runtime& rt, const SampleSpec& sp, int L, int64_t s0, int64_t ns, double2* d_out)
{
	const int64_t total = ns << L;
	const int64_t runs = (total + HRUN - 1) / HRUN;
	const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((runs + HTPB - 1) / HTPB, (int64_t)rt.num_sms * 16));
	k_haar<<<grid, HTPB, 0, rt.stream>>>(sp, L, s0, total, d_out);
	rt.launches++;
	int ret = RQC_CUDA(cudaGetLastError());
	if (ret) return ret;
	k_normalize<<<(unsigned)ns, HTPB, 0, rt.stream>>>(d_out, L);
	rt.launches++;
	return RQC_CUDA(cudaGetLastError());
}

int sampled_f_device(Runtime& rt, int L, int ngates, const double2* gates, const int* wires, const TargetSpec& t,
                     const SampleSpec& sp, double2* d_f)
{
	const int64_t N = (int64_t)1 << L;
	if (sp.nsamples < 1) return E_ARG;
	// chunk states: samples, target columns, C psi, two target scratch states
	const size_t col_bytes = 5 * (size_t)N * sizeof(double2);
	int64_t C = (int64_t)(sampling_workspace_limit(rt) / col_bytes);
	if (rt.column_chunk > 0) C = std::min<int64_t>(C, rt.column_chunk);
	if (t.ufunc) C = std::min<int64_t>(C, std::max<int64_t>(1, ((int64_t)256 << 20) / (N * 16)));
	C = std::min<int64_t>(C, sp.nsamples);
	if (C < 1) return E_ALLOC;
	int ret = ensure_device(rt.work, 5 * (size_t)C * N * sizeof(double2));
	if (ret) return ret;
	double2* states = reinterpret_cast<double2*>(rt.work.ptr);
	double2* phi = states + C * N;
	double2* cpsi = phi + C * N;
	double2* p0 = cpsi + C * N;
	double2* p1 = p0 + C * N;
	const int nblk = rt.num_sms * 4;
	if ((ret = ensure_device(rt.partials, (size_t)nblk * sizeof(double2)))) return ret;
	double2* fpart = reinterpret_cast<double2*>(rt.partials.ptr);
	if ((ret = RQC_CUDA(cudaMemsetAsync(fpart, 0, (size_t)nblk * sizeof(double2), rt.stream)))) return ret;
	for (int64_t s0 = 0; s0 < sp.nsamples; s0 += C) {
		const int64_t Cc = std::min(C, sp.nsamples - s0);
		if ((ret = haar_states_device(rt, sp, L, s0, Cc, states))) return ret;
		if ((ret = target_states_device(rt, t, L, states, Cc, phi, p0, p1))) return ret;
		if ((ret = apply_circuit_device(rt, L, ngates, gates, wires, states, cpsi, (long)Cc))) return ret;
		k_fdot<<<nblk, HTPB, 0, rt.stream>>>(phi, cpsi, Cc * N, fpart);
		rt.launches++;
		if ((ret = RQC_CUDA(cudaGetLastError()))) return ret;
	}
	k_fsum<<<1, 32, 0, rt.stream>>>(fpart, nblk, (double)N / (double)sp.nsamples, d_f);
	rt.launches++;
	return RQC_CUDA(cudaGetLastError());
}

}  // namespace rqc
