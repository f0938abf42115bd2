// Host description of an optimisation problem: the sequential circuit the
// engine evaluates, its optimisation units (one gate per brickwall layer, or
// every gate of a general circuit) and the target.
#pragma once

#include <vector>

#include "engine.h"
#include "rqcopt_gpu.h"

namespace rqc {

struct Problem
{
	int L = 0;
	int G = 0;        // sequential gates
	int nunits = 0;   // optimisation units
	int per = 1;      // sequential gates per unit (brickwall: L/2 copies of the layer gate)
	std::vector<double2> gates, dirs;     // [G][16]
	std::vector<int> wires;               // [2G]
	std::vector<double2> ugates, udirs;   // [nunits][16]

	bool set_brickwall(int L, int nlayers, const struct mat4x4* vlist, const struct mat4x4* vdirs, const int* const* perms);
	bool set_circuit(int L, int ngates, const struct mat4x4* gates, const struct mat4x4* dirs, const int* wires);
	bool valid() const;
	void set_gates_from_units(const double2* ugates);
	void set_dirs_from_units(const double2* udirs);
};

// Target of the basis-column sums: a device-native brickwall / circuit, or a host callback.
struct TargetHolder
{
	std::vector<double2> gates;
	std::vector<int> wires;
	TargetSpec spec;
	bool set(linear_func ufunc, void* udata, int L);
};

int post_launch(Runtime& rt, const double2* d_res, const Problem& pb, const double2* d_ugates, const double2* d_udirs,
                int with_hvp, double2* d_dunits, double2* d_hunits, double* d_grad, double* d_hvp);

int run_target(const Problem& pb, const TargetHolder& th, int mode, numeric* fval, struct mat4x4* dunits,
               struct mat4x4* hunits, double* grad_vec, double* hvp_vec);

}  // namespace rqc
