// Host random numbers and statevector normalisation of the reference's public C API
// (src/pcg_basic.h, src/rng.h, src/statevector.h:23).  The generator is PCG32
// (M. O'Neill, "PCG: a family of simple fast space-efficient statistically good
// algorithms for random number generation", 2014: a 64-bit LCG with multiplier
// 6364136223846793005 and the XSH-RR output permutation), which the reference
// vendors as src/pcg_basic.c; two generators with distinct streams form the 64-bit
// pair of struct rng_state.  Every function reproduces the reference's stream bit
// for bit (the normals up to the host libm, as in the reference); the device Haar
// generator (sampling.cu) draws from the same stream.
#include <math.h>
#include <string.h>
#include <vector>

#include "rqc_runtime.h"
#include "rqcopt_gpu.h"

using namespace rqc;

namespace {

constexpr uint64_t PCG_MULT = 6364136223846793005ULL;

}  // namespace

extern "C" {

// src/pcg_basic.c:30-37: stream from initseq, then two steps around adding initstate
void pcg32_srandom_r(const uint64_t initstate, const uint64_t initseq, struct pcg32_random* rng)
{
	rng->state = 0;
	rng->inc = (initseq << 1u) | 1u;
	pcg32_random_r(rng);
	rng->state += initstate;
	pcg32_random_r(rng);
}

// src/pcg_basic.c:44-51: LCG step, XSH-RR output of the old state
uint32_t pcg32_random_r(struct pcg32_random* rng)
{
	const uint64_t old = rng->state;
	rng->state = old * PCG_MULT + rng->inc;
	const uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
	const uint32_t rot = (uint32_t)(old >> 59u);
	return (xs >> rot) | (xs << ((32u - rot) & 31u));
}

// src/pcg_basic.c:58-83: unbiased r % bound by rejecting r below 2^32 mod bound
// (bound 0 returns 0)
uint32_t pcg32_boundedrand_r(const uint32_t bound, struct pcg32_random* rng)
{
	if (bound == 0) return 0;
	const uint32_t threshold = (0u - bound) % bound;
	for (;;) {
		const uint32_t r = pcg32_random_r(rng);
		if (r >= threshold) return r % bound;
	}
}

// src/pcg_basic.c:112-121: the two streams must differ (beyond the top bit)
void pcg32x2_srandom_r(uint64_t seed1, uint64_t seed2, uint64_t seq1, uint64_t seq2, struct pcg32x2_random* rng)
{
	const uint64_t mask = ~0ull >> 1;
	if ((seq1 & mask) == (seq2 & mask)) seq2 = ~seq2;
	pcg32_srandom_r(seed1, seq1, &rng->gen[0]);
	pcg32_srandom_r(seed2, seq2, &rng->gen[1]);
}

// src/pcg_basic.c:128-132: high word from the first generator, low word from the second
uint64_t pcg32x2_random_r(struct pcg32x2_random* rng)
{
	const uint64_t hi = pcg32_random_r(&rng->gen[0]);
	return (hi << 32) | pcg32_random_r(&rng->gen[1]);
}

// src/pcg_basic.c:139-148 (bound 0 returns 0)
uint64_t pcg32x2_boundedrand_r(const uint64_t bound, struct pcg32x2_random* rng)
{
	if (bound == 0) return 0;
	const uint64_t threshold = (0ull - bound) % bound;
	for (;;) {
		const uint64_t r = pcg32x2_random_r(rng);
		if (r >= threshold) return r % bound;
	}
}

// src/rng.c:13-25: a seeding generator on (seed, stream 6364136223846793005 seed +
// 1442695040888963407) yields the two seeds and two streams of the pair
void seed_rng_state(const uint64_t seed, struct rng_state* state)
{
	struct pcg32_random s;
	pcg32_srandom_r(seed, PCG_MULT * seed + 1442695040888963407ULL, &s);
	uint64_t v[4];
	for (int k = 0; k < 4; k++) {
		const uint64_t hi = pcg32_random_r(&s);
		v[k] = (hi << 32) | pcg32_random_r(&s);
	}
	pcg32x2_srandom_r(v[0], v[1], v[2], v[3], &state->pcgstate);
}

// src/rng.c:32-36: the first generator alone
uint32_t rand_uint32(struct rng_state* state) { return pcg32_random_r(&state->pcgstate.gen[0]); }

// src/rng.c:43-46
uint64_t rand_uint64(struct rng_state* state) { return pcg32x2_random_r(&state->pcgstate); }

// src/rng.c:53-56
uint64_t rand_interval(const uint64_t bound, struct rng_state* state) { return pcg32x2_boundedrand_r(bound, &state->pcgstate); }

// src/rng.c:63-85: Floyd's sampling of num_samples distinct values below bound
void rand_choice(const uint64_t bound, const uint64_t num_samples, struct rng_state* state, uint64_t* ret)
{
	if (num_samples > bound) {
		fail_arg("rand_choice", "more samples than values");
		return;
	}
	for (uint64_t i = 0; i < num_samples; i++) {
		const uint64_t j = bound - num_samples + 1 + i;
		const uint64_t t = rand_interval(j, state);
		bool drawn = false;
		for (uint64_t k = 0; k < i; k++)
			if (ret[k] == t) { drawn = true; break; }
		ret[i] = drawn ? j - 1 : t;
	}
}

// src/rng.c:91-94, 102-105: uniform on [0, 1) from 64 (32) random bits
double randu(struct rng_state* state) { return ldexp((double)rand_uint64(state), -64); }
float randuf(struct rng_state* state) { return ldexpf((float)rand_uint32(state), -32); }

// src/rng.c:114-126, 132-144: Box-Muller with log(u1) (u1 = 0 replaced by 1)
double randn(struct rng_state* state)
{
	double u1 = randu(state);
	const double u2 = randu(state);
	if (u1 == 0) u1 = 1;
	return sqrt(-2 * log(u1)) * sin(6.2831853071795864769 * u2);
}

float randnf(struct rng_state* state)
{
	float u1 = randuf(state);
	const float u2 = randuf(state);
	if (u1 == 0) u1 = 1;
	return sqrtf(-2 * logf(u1)) * sinf((float)6.2831853071795864769 * u2);
}

// src/rng.c:152-172: (x + i y) / sqrt(2) from two standard normals
numeric crandn(struct rng_state* state)
{
	const double x = randn(state);
	const double y = randn(state);
	return numeric(x / sqrt(2.0), y / sqrt(2.0));
}

std::complex<float> crandnf(struct rng_state* state)
{
	const float x = randnf(state);
	const float y = randnf(state);
	return std::complex<float>(x / sqrtf(2.f), y / sqrtf(2.f));
}

// src/statevector.c:47-66: divide by the 2-norm unless it is zero.  On the host, with
// device-memory statevectors copied through host memory.
void normalize_statevector(struct statevector* psi)
{
	if (!psi || !psi->data || psi->nqubits < 0 || psi->nqubits > 40) {
		fail_arg("normalize_statevector", "invalid statevector");
		return;
	}
	const int64_t n = (int64_t)1 << psi->nqubits;
	cudaPointerAttributes a;
	bool dev = false;
	if (cudaPointerGetAttributes(&a, psi->data) == cudaSuccess) dev = a.type == cudaMemoryTypeDevice;
	else cudaGetLastError();
	std::vector<double2> h(dev ? n : 0);
	if (dev && RQC_CUDA(cudaMemcpy(h.data(), psi->data, n * sizeof(double2), cudaMemcpyDeviceToHost))) {
		set_last_error(E_CUDA);
		return;
	}
	double2* x = dev ? h.data() : reinterpret_cast<double2*>(psi->data);
	// scaled sum of squares (no overflow or underflow for extreme amplitudes)
	double scale = 0, ssq = 1;
	for (int64_t k = 0; k < n; k++)
		for (double v : { x[k].x, x[k].y }) {
			if (v == 0) continue;
			const double av = fabs(v);
			if (scale < av) {
				ssq = 1 + ssq * (scale / av) * (scale / av);
				scale = av;
			} else {
				ssq += (av / scale) * (av / scale);
			}
		}
	const double nrm = scale * sqrt(ssq);
	if (nrm > 0) {
		const double s = 1. / nrm;
		for (int64_t k = 0; k < n; k++) x[k] = make_double2(x[k].x * s, x[k].y * s);
	}
	if (dev && RQC_CUDA(cudaMemcpy(psi->data, h.data(), n * sizeof(double2), cudaMemcpyHostToDevice)))
		set_last_error(E_CUDA);
}

}  // extern "C"
