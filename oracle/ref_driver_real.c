/*
 * Small driver compiled together with the unmodified reference sources, WITHOUT
 * COMPLEX_CIRCUIT (the reference's real-orthogonal build), into
 * oracle/_ref/librqcopt_ref_real.so.  It calls only the reference's own public
 * functions; it adds a matrix-free brickwall target as a `linear_func` and a
 * column-range form of the grad+HVP column loop, so that a bounded sample of a large
 * evaluation can be timed.
 *
 * TEST / BASELINE INFRASTRUCTURE ONLY.
 */
#include <stdlib.h>
#include <string.h>
#include "config.h"
#include "matrix.h"
#include "statevector.h"
#include "quantum_circuit.h"
#include "brickwall_circuit.h"

struct refdrv_brickwall
{
	const struct mat4x4* vlist;
	int nlayers;
	const int** perms;
};

/* psi_out = W psi via the reference's apply_brickwall_unitary (real build) */
int refdrv_real_brickwall_ufunc(const struct statevector* psi, void* udata, struct statevector* psi_out)
{
	const struct refdrv_brickwall* t = udata;
	return apply_brickwall_unitary(t->vlist, t->nlayers, t->perms, psi, psi_out);
}

/*
 * Grad+HVP basis-column sum of the real build restricted to columns [b0, b1), for a
 * brickwall circuit against a brickwall target, through the reference's per-column
 * function quantum_circuit_gates_hessian_vector_product (the loop body of
 * src/target.c:335-369).  Outputs are per-gate sums, ngates = nlayers * L / 2.
 */
int refdrv_real_brickwall_hvp_columns(const struct mat4x4* vlist, const struct mat4x4* vdirs, int nlayers,
                                      const int* perms_flat, int L,
                                      const struct mat4x4* tvlist, int tnlayers, const int* tperms_flat,
                                      long b0, long b1, double* fval, struct mat4x4* dgates, struct mat4x4* hess)
{
	const int per = L / 2, G = nlayers * per;
	struct mat4x4* gates = malloc(G * sizeof(struct mat4x4));
	struct mat4x4* dirs = malloc(G * sizeof(struct mat4x4));
	struct mat4x4* dg = malloc(G * sizeof(struct mat4x4));
	struct mat4x4* hg = malloc(G * sizeof(struct mat4x4));
	int* wires = malloc(2 * G * sizeof(int));
	for (int l = 0; l < nlayers; l++)
		for (int p = 0; p < per; p++) {
			gates[l*per + p] = vlist[l];
			dirs[l*per + p] = vdirs[l];
			wires[2*(l*per + p)] = perms_flat[l*L + 2*p];
			wires[2*(l*per + p) + 1] = perms_flat[l*L + 2*p + 1];
		}
	const int** tp = malloc(tnlayers * sizeof(int*));
	for (int l = 0; l < tnlayers; l++) tp[l] = &tperms_flat[l * L];
	struct refdrv_brickwall target = { tvlist, tnlayers, tp };

	struct statevector psi, upsi, cpsi;
	allocate_statevector(L, &psi);
	allocate_statevector(L, &upsi);
	allocate_statevector(L, &cpsi);
	memset(dgates, 0, G * sizeof(struct mat4x4));
	memset(hess, 0, G * sizeof(struct mat4x4));
	double f = 0;
	const intqs n = (intqs)1 << L;
	int ret = 0;
	for (long b = b0; b < b1; b++) {
		memset(psi.data, 0, n * sizeof(numeric));
		psi.data[b] = 1;
		refdrv_real_brickwall_ufunc(&psi, &target, &upsi);
		for (intqs a = 0; a < n; a++) upsi.data[a] = -upsi.data[a];
		if (quantum_circuit_gates_hessian_vector_product(gates, dirs, G, wires, &psi, &upsi, &cpsi, dg, hg) < 0) { ret = -3; break; }
		for (intqs a = 0; a < n; a++) f += upsi.data[a] * cpsi.data[a];
		for (int k = 0; k < G; k++) { add_matrix(&dgates[k], &dg[k]); add_matrix(&hess[k], &hg[k]); }
	}
	fval[0] = f;
	free_statevector(&psi); free_statevector(&upsi); free_statevector(&cpsi);
	free(tp); free(gates); free(dirs); free(dg); free(hg); free(wires);
	return ret;
}
