// Autotuner of the basis-column evaluation engine.
//
// The column loop of the target functions (src/target.c:335-369) runs as passes over
// column chunks; how fast depends on three choices that interact with the problem
// shape and the GPU: gates fused per HBM round trip (1 = one kernel per gate, 2..4 =
// fused passes over eight-qubit tiles), columns per chunk (larger chunks amortise the
// per-launch cost, smaller ones keep more of the working set in L2), for complex128
// whether the reverse passes rebuild the states inside a pass with adjoint gates or
// recompute them from the pass input, and for complex64 whether the passes run on the
// FP32 FMA pipe or on the TF32 tensor-core MMA.
//
// On the first evaluation of a problem shape (qubits, gates, target gates, precision,
// mode, target kind, paired columns) large enough for the choice to matter, every
// candidate runs over the same contiguous sample of basis columns (the column range of
// rqcopt_gpu_set_column_range) and is timed with CUDA events on the library stream;
// the fastest per column is kept for the rest of the process.  A choice the caller made
// explicitly (rqcopt_gpu_set_gates_per_pass, _set_column_chunk, _set_reconstruct) stays
// fixed; rqcopt_gpu_set_autotune(1) releases them.  The search is
// coordinate-wise: gates per pass at the default chunk and reverse variant, then the
// chunk, then the reverse variant.  Every candidate computes the same sums (they differ
// in summation order only, to rounding), so tuning changes speed, not results.
#include <stdio.h>
#include <algorithm>
#include <vector>

#include "engine.h"
#include "rqc_runtime.h"

namespace rqc {

namespace {

// problems below this many amplitude x gate updates per evaluation run with the
// configured defaults (their evaluations take well under a millisecond)
constexpr double TUNE_MIN_WORK = 1 << 26;

struct Config { int gpp; long chunk; int recon; int ffma; };

struct Saved
{
	int gpp, recon, ffma;
	long chunk;
	int64_t b, e;
	explicit Saved(const Runtime& rt)
		: gpp(rt.gates_per_pass), recon(rt.recon_c128), ffma(rt.c64_ffma), chunk(rt.column_chunk), b(rt.col_begin),
		  e(rt.col_end) {}
	void restore(Runtime& rt) const
	{
		rt.gates_per_pass = gpp;
		rt.recon_c128 = recon;
		rt.c64_ffma = ffma;
		rt.column_chunk = chunk;
		rt.col_begin = b;
		rt.col_end = e;
	}
};

void apply(Runtime& rt, const Config& k)
{
	rt.gates_per_pass = k.gpp;
	rt.column_chunk = k.chunk;
	rt.recon_c128 = k.recon;
	rt.c64_ffma = k.ffma;
}

// milliseconds of one evaluation under configuration k over the sample [b, e) (the
// second of two runs: the first sets up kernels and workspace); negative on error
double time_config(Runtime& rt, const Config& k, const CircuitSpec& c, const TargetSpec& t, int mode, int precision,
                   double2* d_out, int64_t b, int64_t e, int* err)
{
	apply(rt, k);
	rt.col_begin = b;
	rt.col_end = e;
	cudaEvent_t e0, e1;
	if (RQC_CUDA(cudaEventCreate(&e0))) { *err = E_CUDA; return -1; }
	if (RQC_CUDA(cudaEventCreate(&e1))) { cudaEventDestroy(e0); *err = E_CUDA; return -1; }
	float ms = -1;
	int ret = evaluate_configured(rt, c, t, mode, precision, d_out);
	if (!ret) ret = RQC_CUDA(cudaEventRecord(e0, rt.stream));
	if (!ret) ret = evaluate_configured(rt, c, t, mode, precision, d_out);
	if (!ret) ret = RQC_CUDA(cudaEventRecord(e1, rt.stream));
	if (!ret) ret = RQC_CUDA(cudaEventSynchronize(e1));
	if (!ret) ret = RQC_CUDA(cudaEventElapsedTime(&ms, e0, e1));
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	if (ret) { *err = ret; return -1; }
	return ms;
}

}  // namespace

int evaluate_autotuned(Runtime& rt, const CircuitSpec& c, const TargetSpec& t, int mode, int precision, double2* d_out)
{
	const int64_t N = (int64_t)1 << c.L;
	const int64_t ncols = rt.real_pairs ? N / 2 : N;
	const double work = (double)ncols * (double)N * (double)(c.ngates + t.ngates);
	// host-callback targets are not tuned: the sample runs would call the caller's ufunc
	if (!rt.autotune || rt.tuning || c.L < 4 || work < TUNE_MIN_WORK || t.ufunc ||
	    (rt.pin_gpp && rt.pin_chunk && rt.pin_recon && rt.pin_ffma)) {
		rt.last_choice = {rt.gates_per_pass, rt.column_chunk, rt.recon_c128, rt.c64_ffma, 0.0, 0};
		return evaluate_configured(rt, c, t, mode, precision, d_out);
	}
	const std::array<long, 11> key = {c.L, c.ngates, t.ngates, precision, mode, t.ufunc ? 1 : 0, rt.real_pairs,
	                                  rt.pin_gpp ? rt.gates_per_pass : 0, rt.pin_chunk ? rt.column_chunk : -1,
	                                  rt.pin_recon ? rt.recon_c128 : -1, rt.pin_ffma ? rt.c64_ffma : -1};
	const Saved saved(rt);
	auto it = rt.tune_cache.find(key);
	if (it == rt.tune_cache.end()) {
		// the sample: the caller's column range (or all columns), at most 4096 columns
		const int64_t b = std::min<int64_t>(rt.col_begin, ncols);
		const int64_t e_all = rt.col_end > 0 ? std::min<int64_t>(rt.col_end, ncols) : ncols;
		const int64_t e = std::min<int64_t>(e_all, b + 4096);
		const int64_t ns = std::max<int64_t>(1, e - b);
		rt.tuning = true;
		int err = 0;
		Config best = {saved.gpp, saved.chunk, saved.recon, saved.ffma};
		double best_ms = time_config(rt, best, c, t, mode, precision, d_out, b, e, &err);
		auto consider = [&](const Config& k) {
			if (err) return;
			const double ms = time_config(rt, k, c, t, mode, precision, d_out, b, e, &err);
			if (!err && ms >= 0 && ms < best_ms) { best_ms = ms; best = k; }
		};
		// gates per pass (unless the caller set it)
		const Config base = best;
		if (!rt.pin_gpp)
			for (int g = 1; g <= 4; g++)
				if (g != base.gpp) consider({g, base.chunk, base.recon, base.ffma});
		// columns per chunk (0: as many as the workspace holds)
		const Config after_gpp = best;
		if (!rt.pin_chunk)
			for (long ch : {0L, 2048L, 1024L, 512L, 256L, 128L})
				if (ch != after_gpp.chunk && (ch == 0 || ch < ns))
					consider({after_gpp.gpp, ch, after_gpp.recon, after_gpp.ffma});
		// reverse variant (complex128 fused passes of HVP / gradient evaluations)
		if (!rt.pin_recon && precision == PREC_C128 && best.gpp > 1 && mode != EVAL_F)
			consider({best.gpp, best.chunk, 1 - best.recon, best.ffma});
		// complex64 passes on the FP32 pipe or the TF32 MMA
		if (!rt.pin_ffma && precision != PREC_C128 && best.gpp > 1)
			consider({best.gpp, best.chunk, best.recon, 1 - best.ffma});
		rt.tuning = false;
		saved.restore(rt);
		if (err) return err;
		it = rt.tune_cache.emplace(key, Runtime::TuneChoice{best.gpp, best.chunk, best.recon, best.ffma, best_ms / (double)ns, 1})
		         .first;
	}
	const Runtime::TuneChoice& ch = it->second;
	apply(rt, {ch.gates_per_pass, ch.column_chunk, ch.recon, ch.ffma});
	rt.last_choice = ch;
	const int ret = evaluate_configured(rt, c, t, mode, precision, d_out);
	saved.restore(rt);
	return ret;
}

}  // namespace rqc
