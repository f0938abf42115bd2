// Random-state sampling estimator (src/target.c:85-149, 491-505, 807-928,
// 1050-1088): Haar-random states from the reference's PCG32x2 stream
// (src/rng.c, src/pcg_basic.c) generated on the device, in place of the basis
// columns of the exact sums.
#pragma once

#include <stdint.h>
#include "engine.h"
#include "rqc_runtime.h"
#include "rqcopt_gpu.h"

namespace rqc {

// The two PCG32 generators of `struct rng_state` at the start of a call.
// real: states of the reference's real build, one real normal per amplitude
// (src/statevector.c:115-121) instead of a complex one.
struct SampleSpec
{
	uint64_t state[2], inc[2];
	int64_t nsamples;
	int real;
};

// advance a PCG32 generator (64-bit LCG) by delta steps (jump-ahead)
void pcg_advance_host(uint64_t& state, uint64_t inc, uint64_t delta);

// process-wide choice of real sample states (rqcopt_gpu_set_real_samples)
int real_samples();

inline SampleSpec sample_spec(const struct rng_state* rng, long nsamples)
{
	SampleSpec sp;
	for (int k = 0; k < 2; k++) {
		sp.state[k] = rng->pcgstate.gen[k].state;
		sp.inc[k] = rng->pcgstate.gen[k].inc;
	}
	sp.nsamples = nsamples;
	sp.real = real_samples();
	return sp;
}

// past nsamples states of 2^L amplitudes: the reference draws 4 outputs of both
// generators per complex amplitude, 2 per real one (src/rng.c:114-157)
inline void advance_rng(struct rng_state* rng, long nsamples, int L)
{
	const uint64_t steps = (real_samples() ? 2 : 4) * (uint64_t)nsamples << L;
	for (int k = 0; k < 2; k++) pcg_advance_host(rng->pcgstate.gen[k].state, rng->pcgstate.gen[k].inc, steps);
}

// Haar-random states number s0 .. s0 + ns - 1 of the stream that starts at sp, one
// after another (2^L amplitudes each, normalised), into d_out.
int haar_states_device(Runtime& rt, const SampleSpec& sp, int L, int64_t s0, int64_t ns, double2* d_out);

// f = (2^L / nsamples) sum_b <-conj(U psi_b), C psi_b> for a sequential circuit (host
// gates and wires) -> d_f (one double2)
int sampled_f_device(Runtime& rt, int L, int ngates, const double2* gates, const int* wires, const TargetSpec& t,
                     const SampleSpec& sp, double2* d_f);

}  // namespace rqc
