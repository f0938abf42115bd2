// Per-device runtime state of the library: the stream every call issues its
// work on, device workspaces that grow on demand and are reused across calls,
// staging of host buffers, error reporting, launch counting and per-kernel
// event timing.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>
#include <array>
#include <map>
#include <vector>

namespace rqc {

enum ErrorCode { OK = 0, E_ALLOC = -1, E_UFUNC = -2, E_PASS = -3, E_PASS2 = -4, E_CUDA = -5, E_ARG = -6 };

enum KernelClass { KC_APPLY = 0, KC_FORWARD = 1, KC_REVERSE = 2, KC_FUSED = 3, KC_HESS = 4, KC_COUNT = 5 };

struct Buffer
{
	void* ptr = nullptr;
	size_t bytes = 0;
};

struct Runtime
{
	int device = -1;
	int num_sms = 0;
	cudaStream_t stream = nullptr;

	// device buffers, grown on demand
	Buffer work;          // evaluation-engine column chunks and caches
	Buffer partials;      // per-block partial sums
	Buffer small;         // inputs of the exported calls (gates, directions)
	Buffer result;        // reduction results of the engine and single-gate passes
	Buffer opt;           // optimiser vectors
	Buffer scratch;       // FP64 per-lane sums of the complex64 reverse passes
	Buffer stage[4];      // staging of host statevectors
	Buffer arrays;        // statevector arrays and gate-input caches of the full-Hessian calls
	Buffer hpin;          // pinned host scratch
	Buffer status;        // device status word of kernels with bounded waits (non-zero: a wait gave up)

	// configuration
	int precision = 0;
	double refine_threshold = 1e-5;
	size_t workspace_limit = 0;
	long column_chunk = 0;
	// basis columns the target sums run over: [col_begin, col_end), col_end 0 = to the last
	// column (rqcopt_gpu_set_column_range)
	int64_t col_begin = 0, col_end = 0;
	int64_t col_end_dev = -1;    // the column end the fused kernels hold (__constant__), -1 unset
	int real_pairs = 0;          // evaluate(): paired basis columns of a real problem (rqcopt_gpu_set_real_pairs)
	int gates_per_pass = 4;   // 1: one kernel per gate; 2..4: fused passes
	int recon_c128 = 1;       // complex128 reverse passes rebuild states with adjoint gates (unitary gates)
	int c64_ffma = 0;         // complex64 fused passes on the FP32 pipe (k7) rather than the TF32 MMA (k4 / k5)

	// autotuning of the basis-column engine (autotune.cu): the configuration chosen per
	// problem shape, and the one the last evaluation ran with
	struct TuneChoice { int gates_per_pass; long column_chunk; int recon; int ffma; double ms_per_column; int tuned; };
	int autotune = 1;
	bool tuning = false;
	bool pin_gpp = false, pin_chunk = false, pin_recon = false, pin_ffma = false;   // set explicitly by the caller
	std::map<std::array<long, 11>, TuneChoice> tune_cache;
	TuneChoice last_choice = {0, 0, 0, 0, 0.0, 0};

	// instrumentation
	unsigned long long launches = 0;
	// per-iteration record of the last optimize_* call with Hessian-vector products:
	// step accepted, tCG ended on the trust-region boundary, tCG inner iterations,
	// Hessian-vector products in complex128 (1) or complex64 (0)
	struct IterTrace { int accepted, on_boundary, inner, refined; };
	std::vector<IterTrace> opt_trace;
	bool timing = false;
	double time_ms[KC_COUNT] = {0, 0, 0, 0, 0};
	long time_count[KC_COUNT] = {0, 0, 0, 0, 0};
	std::vector<cudaEvent_t> event_pool;
	struct Pending { cudaEvent_t a, b; int cls; };
	std::vector<Pending> pending;
};

// runtime of the current device; initialises it on first use (nullptr if no usable GPU)
Runtime* runtime();

// report a CUDA error (prints to stderr); returns E_CUDA if e != cudaSuccess
int cuda_check(cudaError_t e, const char* what, const char* file, int line);
#define RQC_CUDA(call) ::rqc::cuda_check((call), #call, __FILE__, __LINE__)

// record an error of a void entry point (readable through rqcopt_gpu_last_error)
void set_last_error(int code);
void fail_arg(const char* fn, const char* msg);

// ensure a buffer holds at least `bytes` (device or pinned host); returns 0 or E_ALLOC
int ensure_device(Buffer& b, size_t bytes);
int ensure_host_pinned(Buffer& b, size_t bytes);

// true if the pointer is device-accessible memory of this context (device or managed)
bool is_device_pointer(const void* p);

// A statevector-sized span on the device: either the caller's pointer (device or
// managed memory) or a staging buffer filled from / written back to host memory.
struct DeviceSpan
{
	void* dev = nullptr;
	void* host = nullptr;   // non-null if staged
	size_t bytes = 0;
};
int span_in(Runtime& rt, const void* p, size_t bytes, int slot, DeviceSpan& s);
int span_out(Runtime& rt, void* p, size_t bytes, int slot, DeviceSpan& s);
int span_finish(Runtime& rt, DeviceSpan& s);   // copy back if staged (async on rt.stream)

// synchronise the stream and fold pending kernel timings; returns 0 or E_CUDA
int sync(Runtime& rt);

// kernel launch bookkeeping
void launch_begin(Runtime& rt, int cls, cudaEvent_t* ev_start);
void launch_end(Runtime& rt, int cls, cudaEvent_t ev_start);

}  // namespace rqc
