// Exported configuration and instrumentation entry points (additions; no
// counterpart in the reference).
#include "rqc_runtime.h"
#include "rqcopt_gpu.h"

using namespace rqc;

namespace rqc { int take_last_error(); void set_real_samples(int on); }

extern "C" {

int rqcopt_gpu_set_precision(int precision)
{
	if (precision < RQCOPT_PRECISION_C128 || precision > RQCOPT_PRECISION_C64) return E_ARG;
	Runtime* rt = runtime();
	if (!rt) return E_CUDA;
	rt->precision = precision;
	return 0;
}

int rqcopt_gpu_get_precision(void)
{
	Runtime* rt = runtime();
	return rt ? rt->precision : E_CUDA;
}

void rqcopt_gpu_set_refine_threshold(double gnorm)
{
	if (Runtime* rt = runtime()) rt->refine_threshold = gnorm;
}

void rqcopt_gpu_set_workspace_limit(size_t bytes)
{
	if (Runtime* rt = runtime()) rt->workspace_limit = bytes;
}

void rqcopt_gpu_set_column_chunk(long columns)
{
	if (Runtime* rt = runtime()) {
		rt->column_chunk = columns > 0 ? columns : 0;
		rt->pin_chunk = columns > 0;
	}
}

int rqcopt_gpu_set_autotune(int on)
{
	Runtime* rt = runtime();
	if (!rt) return E_CUDA;
	rt->autotune = on ? 1 : 0;
	if (on) {
		rt->pin_gpp = rt->pin_chunk = rt->pin_recon = rt->pin_ffma = false;
		rt->gates_per_pass = 4;
		rt->column_chunk = 0;
		rt->recon_c128 = 1;
		rt->c64_ffma = 0;
	}
	return 0;
}

int rqcopt_gpu_last_config(int* gates_per_pass, long* column_chunk, int* reconstruct, int* c64_fp32_pipe,
                           double* ms_per_column)
{
	Runtime* rt = runtime();
	if (!rt) return E_CUDA;
	const Runtime::TuneChoice& c = rt->last_choice;
	if (gates_per_pass) *gates_per_pass = c.gates_per_pass;
	if (column_chunk) *column_chunk = c.column_chunk;
	if (reconstruct) *reconstruct = c.recon;
	if (c64_fp32_pipe) *c64_fp32_pipe = c.ffma;
	if (ms_per_column) *ms_per_column = c.ms_per_column;
	return c.tuned;
}

int rqcopt_gpu_set_column_range(long begin, long end)
{
	if (begin < 0 || end < 0 || (end != 0 && end <= begin)) return E_ARG;
	Runtime* rt = runtime();
	if (!rt) return E_CUDA;
	rt->col_begin = begin;
	rt->col_end = end;
	return 0;
}

void rqcopt_gpu_set_c64_fp32_pipe(int on)
{
	if (Runtime* rt = runtime()) {
		rt->c64_ffma = on ? 1 : 0;
		rt->pin_ffma = true;
	}
}

void rqcopt_gpu_set_reconstruct(int on)
{
	if (Runtime* rt = runtime()) {
		rt->recon_c128 = on ? 1 : 0;
		rt->pin_recon = true;
	}
}

int rqcopt_gpu_set_gates_per_pass(int gates)
{
	if (gates < 1 || gates > 4) return E_ARG;
	Runtime* rt = runtime();
	if (!rt) return E_CUDA;
	rt->gates_per_pass = gates;
	rt->pin_gpp = true;
	return 0;
}

int rqcopt_gpu_optimizer_trace(int* accepted, int* on_boundary, int* inner_iterations, int* refined, int capacity)
{
	Runtime* rt = runtime();
	if (!rt) return E_CUDA;
	const int n = (int)rt->opt_trace.size();
	for (int k = 0; k < n && k < capacity; k++) {
		const Runtime::IterTrace& t = rt->opt_trace[k];
		if (accepted) accepted[k] = t.accepted;
		if (on_boundary) on_boundary[k] = t.on_boundary;
		if (inner_iterations) inner_iterations[k] = t.inner;
		if (refined) refined[k] = t.refined;
	}
	return n;
}

int rqcopt_gpu_last_error(void) { return take_last_error(); }

void rqcopt_gpu_set_real_samples(int on) { set_real_samples(on); }

void rqcopt_gpu_set_real_pairs(int on)
{
	if (Runtime* rt = runtime()) rt->real_pairs = on ? 1 : 0;
}

unsigned long long rqcopt_gpu_launch_count(void)
{
	Runtime* rt = runtime();
	return rt ? rt->launches : 0;
}

void rqcopt_gpu_reset_launch_count(void)
{
	if (Runtime* rt = runtime()) rt->launches = 0;
}

void rqcopt_gpu_enable_kernel_timing(int enable)
{
	Runtime* rt = runtime();
	if (!rt) return;
	sync(*rt);
	rt->timing = enable != 0;
	for (int k = 0; k < KC_COUNT; k++) { rt->time_ms[k] = 0; rt->time_count[k] = 0; }
}

int rqcopt_gpu_kernel_time(int kernel_class, double* total_ms, long* launches)
{
	Runtime* rt = runtime();
	if (!rt) return E_CUDA;
	if (kernel_class < 0 || kernel_class >= KC_COUNT) return E_ARG;
	int ret = sync(*rt);
	*total_ms = rt->time_ms[kernel_class];
	*launches = rt->time_count[kernel_class];
	return ret;
}

void* rqcopt_gpu_stream(void)
{
	Runtime* rt = runtime();
	return rt ? (void*)rt->stream : nullptr;
}

}  // extern "C"
