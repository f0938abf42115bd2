/* Batched evaluation and optimisation of many independent brickwall circuits
 * on one GPU (additions beside the reference interface; no counterpart in the
 * reference, whose optimisers take one problem per call:
 * src/brickwall_opt.h:8-10 optimize_brickwall_circuit_hvp).
 *
 * Every problem is one brickwall circuit (nlayers layer gates on the pairs of
 * perms[l], as apply_brickwall_unitary, src/brickwall_circuit.c:14-43) fitted to
 * a brickwall target applied matrix-free, i.e. the objective of
 * brickwall_unitary_target* with the target as the linear function
 * (src/target.c:467-678).  Limits: 2 <= nqubits <= 14 (even), nlayers and
 * target_nlayers <= 16.
 *
 * Precision: RQCOPT_PRECISION_C128 (complex128 passes), RQCOPT_PRECISION_C64
 * (complex64 passes with FP64 sums) or RQCOPT_PRECISION_MIXED (f and gradient in
 * complex128, Hessian-vector products in complex64 until the gradient norm falls
 * below the refinement threshold, rqcopt_gpu_set_refine_threshold).
 *
 * Return codes: >= 0 success (slot, count), -1 allocation, -5 CUDA, -6 invalid
 * argument. */
#ifndef RQCOPT_BATCH_H
#define RQCOPT_BATCH_H

#include <stddef.h>
#include "rqcopt_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

struct rqcopt_batch_problem
{
	int nqubits;
	int nlayers;
	const struct mat4x4* vlist;          /* circuit layer gates (start point) [nlayers] */
	const int* const* perms;             /* [nlayers][nqubits] */
	int target_nlayers;
	const struct mat4x4* target_vlist;   /* target layer gates [target_nlayers] */
	const int* const* target_perms;      /* [target_nlayers][nqubits] */
};

/* f (complex: f[2k], f[2k+1]), projected gradient and projected Hessian-vector
 * product of every problem in one batched pass, as
 * brickwall_unitary_target_projected_hessian_vector_product (src/target.c:631-678)
 * per problem; mode 0 f, 1 f + gradient, 2 f + gradient + HVP in direction
 * vdirs[k] (tangent matrices, [nlayers]).  grad_vec and hvp_vec hold
 * 16 nlayers doubles per problem, concatenated. */
int rqcopt_brickwall_batch_evaluate(const struct rqcopt_batch_problem* problems, int count,
                                    const struct mat4x4* const* vdirs, int mode, int precision, double* f,
                                    double* grad_vec, double* hvp_vec);

/* optimize_brickwall_circuit_hvp for every problem, all advancing together:
 * niter trust-region iterations each (params: one per problem, or NULL for the
 * reference defaults of set_rtr_default_params), f_iter [count][niter + 1],
 * vlist_opt concatenated [sum nlayers]. */
int rqcopt_optimize_brickwall_batch(const struct rqcopt_batch_problem* problems, int count,
                                    const struct rtr_params* params, int niter, int precision, double* f_iter,
                                    struct mat4x4* vlist_opt);

/* Slot interface for a request loop: problems join and leave between rounds;
 * one round evaluates every active problem once and advances its trust-region
 * state. */
struct rqcopt_batch;
struct rqcopt_batch* rqcopt_batch_create(int capacity, int max_iterations);
void rqcopt_batch_destroy(struct rqcopt_batch* batch);
/* admit a problem: returns its slot; it stops after niter trust-region iterations
 * or, with grad_tol > 0, at the first iteration whose gradient norm is at most
 * grad_tol (f_iter then ends at that iteration) */
int rqcopt_batch_add(struct rqcopt_batch* batch, const struct rqcopt_batch_problem* problem,
                     const struct rtr_params* params, int niter, int precision, double grad_tol);
/* run up to max_rounds rounds (fewer if every slot finishes): active slots left */
int rqcopt_batch_run(struct rqcopt_batch* batch, int max_rounds);
/* slots that finished since the last call (at most max_slots) */
int rqcopt_batch_finished(struct rqcopt_batch* batch, int* slots, int max_slots);
/* 1 and the results of a finished slot, 0 while it runs; iterations: trust-region
 * iterations completed (f_iter holds iterations + 1 values) */
int rqcopt_batch_result(struct rqcopt_batch* batch, int slot, double* f_iter, struct mat4x4* vlist_opt,
                        int* iterations);
/* free a slot */
int rqcopt_batch_release(struct rqcopt_batch* batch, int slot);
/* cost-weighted sharing for problems added from now on: a problem is evaluated
 * only every p-th round, p growing with its cost per evaluation (off by default) */
int rqcopt_batch_set_sharing(struct rqcopt_batch* batch, int on);
/* rounds run so far */
long rqcopt_batch_rounds(const struct rqcopt_batch* batch);
/* evaluations run so far (one per active problem and round), and of them the
 * Hessian-vector products */
long rqcopt_batch_evaluations(const struct rqcopt_batch* batch, long* hvp_evaluations);
/* device bytes held for one problem of this size (admission accounting) */
size_t rqcopt_batch_footprint(int nqubits, int nlayers);

#ifdef __cplusplus
}
#endif

#endif
