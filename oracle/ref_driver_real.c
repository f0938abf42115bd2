/*
 * Small driver compiled together with the unmodified reference sources, WITHOUT
 * COMPLEX_CIRCUIT (the reference's real-orthogonal build), into
 * oracle/_ref/librqcopt_ref_real.so.  It calls only the reference's own public
 * functions and adds a matrix-free brickwall target as a `linear_func`.
 *
 * TEST / BASELINE INFRASTRUCTURE ONLY.
 */
#include "config.h"
#include "statevector.h"
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
