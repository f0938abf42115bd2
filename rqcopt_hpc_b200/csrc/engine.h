// Basis-column evaluation engine: f = -sum_b <U e_b | C e_b>, the per-gate
// gradients sum_b dG and the Hessian-vector products, for a sequential circuit
// of two-qubit gates, over all 2^L basis columns processed in chunks.
#pragma once

#include <cuda_runtime.h>
#include "rqc_runtime.h"

namespace rqc {

enum EvalMode { EVAL_F = 0, EVAL_GRAD = 1, EVAL_HVP = 2 };
enum Precision { PREC_C128 = 0, PREC_MIXED = 1, PREC_C64 = 2 };

// A sequential circuit; arrays are host memory.
struct CircuitSpec
{
	int L = 0;
	int ngates = 0;
	const double2* gates = nullptr;   // [ngates][16]
	const double2* dirs = nullptr;    // [ngates][16], EVAL_HVP only
	const int* wires = nullptr;       // [2 * ngates]
};

// The target U: either a circuit evaluated on the device (gates, wires) or a
// host callback `linear_func` applied to one basis column at a time.
struct TargetSpec
{
	int ngates = 0;
	const double2* gates = nullptr;
	const int* wires = nullptr;
	void* ufunc = nullptr;
	void* udata = nullptr;
};

// Device result layout (double2): [0] f, [1 + 16 g + e] dG_g[e], [1 + 16 G + 16 g + e] (H Z)_g[e]
inline size_t result_count(int ngates) { return 1 + 32 * (size_t)ngates; }

// Evaluates on rt.stream into the device array d_out (result_count(ngates) entries).
// Returns 0, E_UFUNC if the host callback fails, E_ALLOC or E_CUDA.
int evaluate(Runtime& rt, const CircuitSpec& c, const TargetSpec& t, int mode, int precision, double2* d_out);

// evaluate() with the configuration in rt as it stands (no autotuning)
int evaluate_configured(Runtime& rt, const CircuitSpec& c, const TargetSpec& t, int mode, int precision, double2* d_out);

// evaluate_configured() under the configuration the autotuner picked for this problem
// shape (autotune.cu), tuning on first use when rt.autotune is set and the problem is
// large enough for the choice to matter
int evaluate_autotuned(Runtime& rt, const CircuitSpec& c, const TargetSpec& t, int mode, int precision, double2* d_out);

// Apply a circuit to a batch of states: out = C in, for `ncols` states of 2^L
// amplitudes stored one after another (device pointers; in and out distinct).
int apply_circuit_device(Runtime& rt, int L, int ngates, const double2* gates, const int* wires,
                         const double2* d_in, double2* d_out, long ncols);

// Same for one statevector with up to maxk consecutive gates per HBM round trip
// (shared-memory tiles over the gates' qubits plus the lowest amplitude bits).
int apply_circuit_fused_device(Runtime& rt, int L, int ngates, const double2* gates, const int* wires,
                               const double2* d_in, double2* d_out, int maxk);
int apply_circuit_fused_device_c64(Runtime& rt, int L, int ngates, const double2* gates, const int* wires,
                                   const float2* d_in, float2* d_out, int maxk);
// out = C in for one complex64 statevector (per-gate passes, or fused passes of
// up to gates_per_pass gates for L >= 10)
int apply_circuit_device_c64(Runtime& rt, int L, int ngates, const double2* gates, const int* wires, const float2* d_in,
                             float2* d_out);

// Single-gate kernels on device statevectors (ncols states one after another).
int gate_apply_device(Runtime& rt, int L, const double2* gate, int i, int j,
                      const double2* d_in, double2* d_out, long ncols);
// dpsi = G^T dpsi_out; d_dgate[16] = sum dpsi_out (x) psi (device output)
int gate_backward_device(Runtime& rt, int L, const double2* gate, int i, int j, const double2* d_psi,
                         const double2* d_dout, double2* d_dpsi, double2* d_dgate);
// Forward / reverse / tangent passes of one column with explicit input states
// (psi arbitrary, phi the adjoint vector at the circuit output): psi_out = C psi,
// per-gate dG and HZ into d_dgates / d_hess ([ngates][16] each, device).
// dirs may be null (gradient only, d_hess untouched).
int column_passes_device(Runtime& rt, int L, int ngates, const double2* gates, const double2* dirs, const int* wires,
                         const double2* d_psi, const double2* d_phi, double2* d_psi_out, double2* d_dgates,
                         double2* d_hess);
// Target columns of one chunk: phi[c] = -conj(U e_{b0 + c}) for c < ncols (states of
// 2^L amplitudes one after another), through the device circuit of t or its host
// callback; p0 and p1 are two chunk-sized scratch arrays.
int target_columns_device(Runtime& rt, const TargetSpec& t, int L, int64_t b0, int64_t ncols, double2* phi,
                          double2* p0, double2* p1);
// The same for given input states: phi[c] = -conj(U states[c]).
int target_states_device(Runtime& rt, const TargetSpec& t, int L, const double2* states, int64_t ncols, double2* phi,
                         double2* p0, double2* p1);
// c = a + b elementwise, n complex entries
int add_device(Runtime& rt, const double2* a, const double2* b, double2* c, long n);

}  // namespace rqc
