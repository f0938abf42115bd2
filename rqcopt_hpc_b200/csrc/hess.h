// Full (16 nlayers)^2 Hessian of the brickwall target and of one brickwall
// backward pass (src/brickwall_circuit.c:134-255, src/target.c:687-1035), and
// the dense-Hessian trust-region kernels (src/trust_region.c:83-141, 230-293).
#pragma once

#include <cuda_runtime.h>
#include "engine.h"
#include "rqc_runtime.h"

namespace rqc {

// A brickwall as sequential gates: layer l holds gates l*per .. l*per + per - 1, all
// copies of the layer gate ugates[l]; arrays are host memory.
struct HessCircuit
{
	int L = 0;
	int nlayers = 0;
	const double2* ugates = nullptr;   // [nlayers][16]
	const int* wires = nullptr;        // [2 * nlayers * L/2]
};

// Device output record of the Hessian engine (double2 entries):
// [0] f, [1 + 16 l + e] sum dV_l[e], then the row-major m x m complex Hessian, m = 16 nlayers.
inline size_t hess_record_count(int nlayers) { return 1 + 16 * (size_t)nlayers + 256 * (size_t)nlayers * nlayers; }

struct SampleSpec;

// f, per-layer gradients and the complex Hessian summed over all basis columns, or,
// with samp, over samp->nsamples Haar-random states scaled by 2^L / nsamples.
int hessian_target_device(Runtime& rt, const HessCircuit& c, const TargetSpec& t, double2* d_rec,
                          const SampleSpec* samp = nullptr);

// One state: cache holds the input state of every sequential gate (device, one after
// another), dout the cotangent of the circuit output; dpsi (device) receives the
// cotangent of the input; d_rec gets the gradient and Hessian (f slot zero).
int hessian_single_device(Runtime& rt, const HessCircuit& c, const double2* d_cache, const double2* d_dout,
                          double2* d_dpsi, double2* d_rec);

// Riemannian gradient vector and real Hessian matrix from a record (src/target.c:937-1035);
// d_ugates: the layer gates on the device.
// With d_hess2 (block encoding) the projected matrix is that of conj(hess1 Z) + hess2 Z.
int project_hessian_device(Runtime& rt, int nlayers, const double2* d_ugates, const double2* d_rec, double* d_grad,
                           double* d_H, const double2* d_hess2 = nullptr);

// Block-encoding target || P^dag W P - H ||_F^2 / 2 (src/target.c:1100-1623), H given by t on
// L/2 qubits.  mode 0: f; 1: f and gradients; 2: f, gradients, hess1 (in the record) and
// hess2 (m x m, device, may be null otherwise).  The record's f slot holds f (real).
int blockenc_device(Runtime& rt, const HessCircuit& c, const TargetSpec& t, int mode, double2* d_rec, double2* d_hess2);

// Truncated CG on a dense n x n Hessian in one single-block kernel; d_status[0]
// receives 1 if the solution stopped on the trust-region boundary.
int tcg_hmat_device(Runtime& rt, int n, const double* d_grad, const double* d_hess, double radius, int maxiter,
                    double abstol, double reltol, double* d_work /* 3 n */, double* d_z, int* d_status);

// y = A x for a row-major n x n matrix (sequential row sums)
int gemv_device(Runtime& rt, int n, const double* d_a, const double* d_x, double* d_y);

// Interleaved arrays of ns states (amplitude a of state s at a*ns + s), device memory.
int gate_to_array_device(Runtime& rt, int L, int ns, const double2* gate, int i, int j, const double2* d_in,
                         double2* d_out);
// d_dgates[s] = sum dout (x) psi_s (device, ns x 16)
int gate_backward_array_device(Runtime& rt, int L, int ns, int i, int j, const double2* d_psi, const double2* d_dout,
                               double2* d_dgates);
// 16 states E_rc psi, state 4 r + c
int gate_placeholder_device(Runtime& rt, int L, int i, int j, const double2* d_psi, double2* d_out);

}  // namespace rqc
