/*
 * Small driver compiled together with the unmodified reference sources into
 * oracle/_ref/librqcopt_ref.so.  It calls only the reference's own public
 * functions; it adds a matrix-free brickwall target as a `linear_func`, the
 * synthetic target map of the reference tests, and a column-range form of the
 * grad+HVP column loop (the loop body of src/target.c:335-369) so that a
 * bounded sample of a large evaluation can be timed.
 *
 * TEST / BASELINE INFRASTRUCTURE ONLY.
 */
#include <stdlib.h>
#include <string.h>
#include "config.h"
#include "matrix.h"
#include "statevector.h"
#include "gate.h"
#include "quantum_circuit.h"
#include "brickwall_circuit.h"
#include "target.h"
#include "trust_region.h"
#include "brickwall_opt.h"
#include "circuit_opt.h"
#include "rng.h"

struct refdrv_brickwall
{
	const struct mat4x4* vlist;
	int nlayers;
	const int** perms;
};

/* matrix-free brickwall target: psi_out = W psi via the reference's apply_brickwall_unitary */
int refdrv_brickwall_ufunc(const struct statevector* psi, void* udata, struct statevector* psi_out)
{
	const struct refdrv_brickwall* t = udata;
	return apply_brickwall_unitary(t->vlist, t->nlayers, t->perms, psi, psi_out);
}

/* synthetic sparse target of the reference tests (test/test_target.c:16-34) */
int refdrv_fixture_ufunc(const struct statevector* psi, void* udata, struct statevector* psi_out)
{
	(void)udata;
	const intqs n = (intqs)1 << psi->nqubits;
	for (intqs i = 0; i < n; i++)
		psi_out->data[i] = (-1.1 + 0.8*I) * psi->data[((i + 3) * 113) % n]
		                 + ( 0.4 - 0.7*I) * psi->data[((i + 9) * 173) % n]
		                 + ( 0.5 + 0.1*I) * psi->data[i]
		                 + (-0.3 + 0.2*I) * psi->data[((i + 4) * 199) % n];
	return 0;
}

static const int** perm_ptrs(const int* flat, int nlayers, int L)
{
	const int** p = malloc(nlayers * sizeof(int*));
	for (int l = 0; l < nlayers; l++) p[l] = flat + (size_t)l * L;
	return p;
}

/*
 * Grad+HVP basis-column sum restricted to columns [b0, b1) for a brickwall
 * circuit against a brickwall target, through the reference's per-column
 * function quantum_circuit_gates_hessian_vector_product.  Outputs are the
 * per-gate sums (not yet folded per layer), ngates = nlayers * L / 2.
 */
int refdrv_brickwall_hvp_columns(const struct mat4x4* vlist, const struct mat4x4* vdirs, int nlayers,
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
	const int** tp = perm_ptrs(tperms_flat, tnlayers, L);
	struct refdrv_brickwall target = { tvlist, tnlayers, tp };

	struct statevector psi, upsi, cpsi;
	allocate_statevector(L, &psi);
	allocate_statevector(L, &upsi);
	allocate_statevector(L, &cpsi);
	memset(dgates, 0, G * sizeof(struct mat4x4));
	memset(hess, 0, G * sizeof(struct mat4x4));
	numeric f = 0;
	const intqs n = (intqs)1 << L;
	int ret = 0;
	for (long b = b0; b < b1; b++) {
		memset(psi.data, 0, n * sizeof(numeric));
		psi.data[b] = 1;
		refdrv_brickwall_ufunc(&psi, &target, &upsi);
		for (intqs a = 0; a < n; a++) upsi.data[a] = -conj(upsi.data[a]);
		if (quantum_circuit_gates_hessian_vector_product(gates, dirs, G, wires, &psi, &upsi, &cpsi, dg, hg) < 0) { ret = -3; break; }
		for (intqs a = 0; a < n; a++) f += upsi.data[a] * cpsi.data[a];
		for (int k = 0; k < G; k++) { add_matrix(&dgates[k], &dg[k]); add_matrix(&hess[k], &hg[k]); }
	}
	fval[0] = creal(f);
	fval[1] = cimag(f);
	free_statevector(&psi); free_statevector(&upsi); free_statevector(&cpsi);
	free(tp); free(gates); free(dirs); free(dg); free(hg); free(wires);
	return ret;
}

/* one f + projected gradient + projected HVP evaluation with a brickwall target */
int refdrv_brickwall_projected_hvp(const struct mat4x4* vlist, const struct mat4x4* vdirs, int nlayers,
                                   const int* perms_flat, int L,
                                   const struct mat4x4* tvlist, int tnlayers, const int* tperms_flat,
                                   double* fval, double* grad_vec, double* hvp_vec)
{
	const int** p = perm_ptrs(perms_flat, nlayers, L);
	const int** tp = perm_ptrs(tperms_flat, tnlayers, L);
	struct refdrv_brickwall target = { tvlist, tnlayers, tp };
	numeric f;
	int ret = brickwall_unitary_target_projected_hessian_vector_product(refdrv_brickwall_ufunc, &target, vlist, vdirs,
		nlayers, p, L, &f, grad_vec, hvp_vec);
	fval[0] = creal(f);
	fval[1] = cimag(f);
	free(p); free(tp);
	return ret;
}

/* optimize_brickwall_circuit_hvp with a brickwall target and default RTR parameters */
void refdrv_optimize_brickwall(const struct mat4x4* vstart, int nlayers, int L, const int* perms_flat,
                               const struct mat4x4* tvlist, int tnlayers, const int* tperms_flat,
                               int niter, double* f_iter, struct mat4x4* vopt)
{
	const int** p = perm_ptrs(perms_flat, nlayers, L);
	const int** tp = perm_ptrs(tperms_flat, tnlayers, L);
	struct refdrv_brickwall target = { tvlist, tnlayers, tp };
	struct rtr_params params;
	set_rtr_default_params(nlayers * num_tangent_params, &params);
	optimize_brickwall_circuit_hvp(refdrv_brickwall_ufunc, &target, vstart, nlayers, L, p, &params, niter, f_iter, vopt);
	free(p); free(tp);
}

/* f, projected gradient and projected Hessian matrix with a brickwall target
 * (src/target.c:996-1035) */
int refdrv_gradient_vector_hessian_matrix(const struct mat4x4* vlist, int nlayers, const int* perms_flat, int L,
                                          const struct mat4x4* tvlist, int tnlayers, const int* tperms_flat,
                                          double* fval, double* grad_vec, double* H)
{
	const int** p = perm_ptrs(perms_flat, nlayers, L);
	const int** tp = perm_ptrs(tperms_flat, tnlayers, L);
	struct refdrv_brickwall target = { tvlist, tnlayers, tp };
	numeric f;
	int ret = brickwall_unitary_target_gradient_vector_hessian_matrix(refdrv_brickwall_ufunc, &target, vlist, nlayers,
		L, p, &f, grad_vec, H);
	fval[0] = creal(f);
	fval[1] = cimag(f);
	free(p); free(tp);
	return ret;
}

/* f, gradients and complex Hessian with a brickwall target (src/target.c:687-806) */
int refdrv_gradient_hessian(const struct mat4x4* vlist, int nlayers, const int* perms_flat, int L,
                            const struct mat4x4* tvlist, int tnlayers, const int* tperms_flat,
                            double* fval, struct mat4x4* dvlist, numeric* hess)
{
	const int** p = perm_ptrs(perms_flat, nlayers, L);
	const int** tp = perm_ptrs(tperms_flat, tnlayers, L);
	struct refdrv_brickwall target = { tvlist, tnlayers, tp };
	numeric f;
	int ret = brickwall_unitary_target_gradient_hessian(refdrv_brickwall_ufunc, &target, vlist, nlayers, L, p, &f,
		dvlist, hess);
	fval[0] = creal(f);
	fval[1] = cimag(f);
	free(p); free(tp);
	return ret;
}

/* the full-Hessian driver with a brickwall target and default RTR parameters */
void refdrv_optimize_brickwall_hmat(const struct mat4x4* vstart, int nlayers, int L, const int* perms_flat,
                                    const struct mat4x4* tvlist, int tnlayers, const int* tperms_flat,
                                    int niter, double* f_iter, struct mat4x4* vopt)
{
	const int** p = perm_ptrs(perms_flat, nlayers, L);
	const int** tp = perm_ptrs(tperms_flat, tnlayers, L);
	struct refdrv_brickwall target = { tvlist, tnlayers, tp };
	struct rtr_params params;
	set_rtr_default_params(nlayers * num_tangent_params, &params);
	optimize_brickwall_circuit_hmat(refdrv_brickwall_ufunc, &target, vstart, nlayers, L, p, &params, niter, f_iter, vopt);
	free(p); free(tp);
}

/* one forward pass and one backward pass with Hessian of a single state, as in
 * examples/benchmark/benchmark_16_qubits.c:66-80 */
int refdrv_forward_backward_hessian(const struct mat4x4* vlist, int nlayers, const int* perms_flat, int L,
                                    const numeric* psi_in, const numeric* dpsi_out_in, numeric* psi_out_o,
                                    numeric* dpsi_o, struct mat4x4* dvlist, numeric* hess)
{
	const int** p = perm_ptrs(perms_flat, nlayers, L);
	const intqs n = (intqs)1 << L;
	struct statevector psi, psi_out, dpsi_out, dpsi;
	allocate_statevector(L, &psi);
	allocate_statevector(L, &psi_out);
	allocate_statevector(L, &dpsi_out);
	allocate_statevector(L, &dpsi);
	memcpy(psi.data, psi_in, n * sizeof(numeric));
	memcpy(dpsi_out.data, dpsi_out_in, n * sizeof(numeric));
	struct quantum_circuit_cache cache;
	int ret = allocate_quantum_circuit_cache(L, nlayers * (L / 2), &cache);
	if (!ret) ret = brickwall_unitary_forward(vlist, nlayers, p, &psi, &cache, &psi_out);
	if (!ret) ret = brickwall_unitary_backward_hessian(vlist, nlayers, p, &cache, &dpsi_out, &dpsi, dvlist, hess);
	memcpy(psi_out_o, psi_out.data, n * sizeof(numeric));
	memcpy(dpsi_o, dpsi.data, n * sizeof(numeric));
	free_quantum_circuit_cache(&cache);
	free_statevector(&psi); free_statevector(&psi_out); free_statevector(&dpsi_out); free_statevector(&dpsi);
	free(p);
	return ret;
}

/*
 * The basis-column loop of brickwall_unitary_target_gradient_hessian
 * (src/target.c:733-790) restricted to columns [b0, b1), with a brickwall target,
 * through the reference's brickwall_unitary_forward and
 * brickwall_unitary_backward_hessian, so that a bounded sample of a large
 * evaluation can be timed.  Outputs are the sums over the sampled columns.
 */
int refdrv_hessian_columns(const struct mat4x4* vlist, int nlayers, const int* perms_flat, int L,
                           const struct mat4x4* tvlist, int tnlayers, const int* tperms_flat,
                           long b0, long b1, double* fval, struct mat4x4* dvlist, numeric* hess)
{
	const int** p = perm_ptrs(perms_flat, nlayers, L);
	const int** tp = perm_ptrs(tperms_flat, tnlayers, L);
	struct refdrv_brickwall target = { tvlist, tnlayers, tp };
	const int m = 16 * nlayers;
	const intqs n = (intqs)1 << L;
	struct statevector psi, upsi, wpsi;
	allocate_statevector(L, &psi);
	allocate_statevector(L, &upsi);
	allocate_statevector(L, &wpsi);
	struct quantum_circuit_cache cache;
	int ret = allocate_quantum_circuit_cache(L, nlayers * (L / 2), &cache);
	struct mat4x4* dv = malloc(nlayers * sizeof(struct mat4x4));
	numeric* hu = malloc((size_t)m * m * sizeof(numeric));
	memset(dvlist, 0, nlayers * sizeof(struct mat4x4));
	memset(hess, 0, (size_t)m * m * sizeof(numeric));
	numeric f = 0;
	for (long b = b0; b < b1 && !ret; b++) {
		memset(psi.data, 0, n * sizeof(numeric));
		psi.data[b] = 1;
		refdrv_brickwall_ufunc(&psi, &target, &upsi);
		for (intqs a = 0; a < n; a++) upsi.data[a] = -conj(upsi.data[a]);
		if ((ret = brickwall_unitary_forward(vlist, nlayers, p, &psi, &cache, &wpsi)) < 0) break;
		for (intqs a = 0; a < n; a++) f += upsi.data[a] * wpsi.data[a];
		if ((ret = brickwall_unitary_backward_hessian(vlist, nlayers, p, &cache, &upsi, &psi, dv, hu)) < 0) break;
		for (int i = 0; i < nlayers; i++) add_matrix(&dvlist[i], &dv[i]);
		for (long i = 0; i < (long)m * m; i++) hess[i] += hu[i];
	}
	fval[0] = creal(f);
	fval[1] = cimag(f);
	free(dv); free(hu);
	free_quantum_circuit_cache(&cache);
	free_statevector(&psi); free_statevector(&upsi); free_statevector(&wpsi);
	free(p); free(tp);
	return ret;
}

/* dense row-major target matrix U as a linear_func (udata: the 2^L x 2^L matrix) */
int refdrv_dense_ufunc(const struct statevector* psi, void* udata, struct statevector* psi_out)
{
	const numeric* u = udata;
	const intqs n = (intqs)1 << psi->nqubits;
	for (intqs r = 0; r < n; r++) {
		numeric s = 0;
		for (intqs c = 0; c < n; c++) s += u[r*n + c] * psi->data[c];
		psi_out->data[r] = s;
	}
	return 0;
}

/* sampling estimator with a brickwall target (tvlist, tperms) or, if tvlist is NULL,
 * the dense target matrix tdense: f only (mode 0), f + gradients + complex Hessian
 * (mode 1) or f + gradient vector + real Hessian (mode 2) */
int refdrv_sampling(int mode, const struct mat4x4* vlist, int nlayers, const int* perms_flat, int L,
                    const struct mat4x4* tvlist, int tnlayers, const int* tperms_flat, const numeric* tdense,
                    long nsamples, struct rng_state* rng, double* fval, void* out1, void* out2)
{
	const int** p = perm_ptrs(perms_flat, nlayers, L);
	const int** tp = tvlist ? perm_ptrs(tperms_flat, tnlayers, L) : NULL;
	struct refdrv_brickwall target = { tvlist, tnlayers, tp };
	linear_func uf = tvlist ? refdrv_brickwall_ufunc : refdrv_dense_ufunc;
	void* ud = tvlist ? (void*)&target : (void*)tdense;
	numeric f = 0;
	int ret;
	if (mode == 0) ret = brickwall_unitary_target_sampling(uf, ud, vlist, nlayers, L, p, nsamples, rng, &f);
	else if (mode == 1) ret = brickwall_unitary_target_gradient_hessian_sampling(uf, ud, vlist, nlayers, L, p, nsamples, rng, &f, out1, out2);
	else ret = brickwall_unitary_target_gradient_vector_hessian_matrix_sampling(uf, ud, vlist, nlayers, L, p, nsamples, rng, &f, out1, out2);
	fval[0] = creal(f);
	fval[1] = cimag(f);
	free(p); free(tp);
	return ret;
}

/* the sampling full-Hessian driver with default RTR parameters */
void refdrv_optimize_brickwall_hmat_sampling(const struct mat4x4* vstart, int nlayers, int L, const int* perms_flat,
                                             const struct mat4x4* tvlist, int tnlayers, const int* tperms_flat,
                                             long nsamples, struct rng_state* rng, int niter, double* f_iter,
                                             struct mat4x4* vopt)
{
	const int** p = perm_ptrs(perms_flat, nlayers, L);
	const int** tp = perm_ptrs(tperms_flat, tnlayers, L);
	struct refdrv_brickwall target = { tvlist, tnlayers, tp };
	struct rtr_params params;
	set_rtr_default_params(nlayers * num_tangent_params, &params);
	optimize_brickwall_circuit_hmat_sampling(refdrv_brickwall_ufunc, &target, vstart, nlayers, L, p, nsamples, rng,
		&params, niter, f_iter, vopt);
	free(p); free(tp);
}

/* block-encoding target with a brickwall H on L / 2 qubits (hvlist, hperms_flat [hnlayers][L/2]):
 * mode 0 f, 1 f + dvlist, 2 f + grad_vec, 3 f + dvlist + hess1 + hess2, 4 f + grad_vec + H */
int refdrv_blockenc(int mode, const struct mat4x4* vlist, int nlayers, const int* perms_flat, int L,
                    const struct mat4x4* hvlist, int hnlayers, const int* hperms_flat, double* fval,
                    void* o1, void* o2, void* o3)
{
	const int** p = perm_ptrs(perms_flat, nlayers, L);
	const int** hp = perm_ptrs(hperms_flat, hnlayers, L / 2);
	struct refdrv_brickwall hop = { hvlist, hnlayers, hp };
	int ret;
	switch (mode) {
	case 0: ret = brickwall_blockenc_target(refdrv_brickwall_ufunc, &hop, vlist, nlayers, L, p, fval); break;
	case 1: ret = brickwall_blockenc_target_and_gradient(refdrv_brickwall_ufunc, &hop, vlist, nlayers, L, p, fval, o1); break;
	case 2: ret = brickwall_blockenc_target_and_gradient_vector(refdrv_brickwall_ufunc, &hop, vlist, nlayers, L, p, fval, o1); break;
	case 3: ret = brickwall_blockenc_target_gradient_hessian(refdrv_brickwall_ufunc, &hop, vlist, nlayers, L, p, fval, o1, o2, o3); break;
	default: ret = brickwall_blockenc_target_gradient_vector_hessian_matrix(refdrv_brickwall_ufunc, &hop, vlist, nlayers, L, p, fval, o1, o2); break;
	}
	free(p); free(hp);
	return ret;
}

/*
 * The column loop of brickwall_blockenc_target_gradient_hessian (src/target.c:1441-1600)
 * restricted to columns [b0, b1) of the half register, with a brickwall H on L/2 qubits,
 * through the reference's brickwall_unitary_forward, brickwall_unitary_backward_hessian and
 * apply_brickwall_unitary_gate_placeholder, so that a bounded sample can be timed.
 */
int refdrv_blockenc_hessian_columns(const struct mat4x4* vlist, int nlayers, const int* perms_flat, int L,
                                    const struct mat4x4* hvlist, int hnlayers, const int* hperms_flat, long b0, long b1,
                                    double* fval)
{
	const int** p = perm_ptrs(perms_flat, nlayers, L);
	const int** hp = perm_ptrs(hperms_flat, hnlayers, L / 2);
	struct refdrv_brickwall hop = { hvlist, hnlayers, hp };
	const int half = L / 2, m = 16 * nlayers;
	const intqs s = (intqs)1 << half, n = (intqs)1 << L;
	struct statevector psi, hpsi, chi, wchi;
	allocate_statevector(half, &psi);
	allocate_statevector(half, &hpsi);
	allocate_statevector(L, &chi);
	allocate_statevector(L, &wchi);
	struct quantum_circuit_cache cache;
	int ret = allocate_quantum_circuit_cache(L, nlayers * (L / 2), &cache);
	struct statevector_array tmp;
	allocate_statevector_array(L, 16, &tmp);
	struct mat4x4* dv = malloc(nlayers * sizeof(struct mat4x4));
	numeric* h1 = malloc((size_t)m * m * sizeof(numeric));
	numeric* phi = malloc((size_t)nlayers * s * 16 * sizeof(numeric));
	numeric* h2 = calloc((size_t)m * m, sizeof(numeric));
	double f = 0;
	for (long b = b0; b < b1 && !ret; b++) {
		memset(psi.data, 0, s * sizeof(numeric));
		psi.data[b] = 1;
		refdrv_brickwall_ufunc(&psi, &hop, &hpsi);
		memset(chi.data, 0, n * sizeof(numeric));
		intqs c = 0;
		for (int i = 0; i < half; i++) { intqs t = b & ((intqs)1 << i); c += 2 * t * t; }
		chi.data[c] = 1;
		if ((ret = brickwall_unitary_forward(vlist, nlayers, p, &chi, &cache, &wchi)) < 0) break;
		memset(chi.data, 0, n * sizeof(numeric));
		for (intqs a = 0; a < s; a++) {
			intqs ca = 0;
			for (int i = 0; i < half; i++) { intqs t = a & ((intqs)1 << i); ca += 2 * t * t; }
			const numeric d = wchi.data[ca] - hpsi.data[a];
			f += 0.5 * (creal(d) * creal(d) + cimag(d) * cimag(d));
			chi.data[ca] = conj(d);
		}
		if ((ret = brickwall_unitary_backward_hessian(vlist, nlayers, p, &cache, &chi, &wchi, dv, h1)) < 0) break;
		for (int l = 0; l < nlayers; l++) {
			if ((ret = apply_brickwall_unitary_gate_placeholder(vlist, nlayers, p, l, &cache, &tmp)) < 0) break;
			for (intqs a = 0; a < s; a++) {
				intqs ca = 0;
				for (int i = 0; i < half; i++) { intqs t = a & ((intqs)1 << i); ca += 2 * t * t; }
				memcpy(&phi[((size_t)l * s + a) * 16], &tmp.data[ca * 16], 16 * sizeof(numeric));
			}
		}
		for (int l = 0; l < nlayers; l++)
			for (int k = 0; k <= l; k++)
				for (intqs a = 0; a < s; a++)
					for (int i = 0; i < 16; i++)
						for (int j = 0; j < 16; j++)
							h2[((l*16 + i)*nlayers + k)*16 + j] += conj(phi[((size_t)l * s + a) * 16 + i]) * phi[((size_t)k * s + a) * 16 + j];
	}
	*fval = f;
	free(dv); free(h1); free(phi); free(h2);
	free_statevector_array(&tmp);
	free_quantum_circuit_cache(&cache);
	free_statevector(&psi); free_statevector(&hpsi); free_statevector(&chi); free_statevector(&wchi);
	free(p); free(hp);
	return ret;
}
