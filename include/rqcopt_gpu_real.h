/*
 * rqcopt_gpu_real.h -- C ABI of librqcopt_gpu_real.so, the real-orthogonal build.
 *
 * The reference compiles its sources either for complex unitary circuits
 * (COMPLEX_CIRCUIT, declared in rqcopt_gpu.h) or, without that definition, for
 * real orthogonal circuits: `numeric` is double, gates are real 4x4 matrices,
 * a tangent direction of a gate is a real antisymmetric matrix with 6
 * parameters (src/matrix.h:42-46, src/matrix.c:245-271, 288-300), and the
 * full-Hessian "matrix" forms and their optimiser do not exist
 * (src/target.h:79-90, 106-110, 123-127; src/brickwall_opt.c:81-100, 152-269).
 * This header declares that function set with the reference's names and
 * signatures; a program written against the reference's real build includes
 * it instead of the reference headers and links -lrqcopt_gpu_real.
 *
 * Conventions are those of rqcopt_gpu.h (synchronous calls, 0 / negative return
 * codes, rqcopt_gpu_last_error for void functions), except:
 *   - statevectors returned by allocate_statevector are host memory;
 *   - the library evaluates through the complex GPU engine of librqcopt_gpu.so
 *     (loaded from the same directory) on states with zero imaginary part,
 *     which gives the real build's results: every sum the real build forms is
 *     the real part of the complex one for real inputs.
 */
#pragma once

#ifdef __cplusplus
extern "C" {
#else
#include <stdbool.h>
#endif

#include <stddef.h>
#include <stdint.h>

/* src/config.h:20 (real build) */
typedef double numeric;

/* src/config.h:62 */
typedef long int intqs;

/* src/matrix.h:10-13 */
struct mat4x4
{
	numeric data[16];
};

/* src/statevector.h:11-15 */
struct statevector
{
	numeric* data;
	int nqubits;
};

/* src/statevector.h:39-44 -- states interleaved: amplitude a of state s at data[a*nstates + s] */
struct statevector_array
{
	numeric* data;
	int nqubits;
	int nstates;
};

/* src/pcg_basic.h:32-36 */
struct pcg32_random
{
	uint64_t state;
	uint64_t inc;
};

/* src/pcg_basic.h:50-53 */
struct pcg32x2_random
{
	struct pcg32_random gen[2];
};

/* src/rng.h:15-18 */
struct rng_state
{
	struct pcg32x2_random pcgstate;
};

/* src/quantum_circuit.h:16-21 */
struct quantum_circuit_cache
{
	struct statevector* psi_list;
	int nqubits;
	int ngates;
};

/* src/target.h:7 */
typedef int (*linear_func)(const struct statevector* psi, void* fdata, struct statevector* psi_out);

/* ------------------------------------------------------------------ statevector.h */

int allocate_statevector(int nqubits, struct statevector* psi);                      /* src/statevector.h:18 */
void free_statevector(struct statevector* psi);                                       /* src/statevector.h:20 */
void add_statevectors(const struct statevector* psi1, const struct statevector* psi2,
	struct statevector* psi_sum);                                                     /* src/statevector.h:32 */
void transpose_statevector(const struct statevector* psi, const int* perm,
	struct statevector* psi_trans);                                                   /* src/statevector.h:26 */
void seed_rng_state(const uint64_t seed, struct rng_state* state);                    /* src/rng.h:21 */
/* src/pcg_basic.h:38-60 and src/rng.h:29-61 -- host random numbers, the reference's stream */
void pcg32_srandom_r(const uint64_t initstate, const uint64_t initseq, struct pcg32_random* rng);
uint32_t pcg32_random_r(struct pcg32_random* rng);
uint32_t pcg32_boundedrand_r(const uint32_t bound, struct pcg32_random* rng);
void pcg32x2_srandom_r(uint64_t seed1, uint64_t seed2, uint64_t seq1, uint64_t seq2, struct pcg32x2_random* rng);
uint64_t pcg32x2_random_r(struct pcg32x2_random* rng);
uint64_t pcg32x2_boundedrand_r(const uint64_t bound, struct pcg32x2_random* rng);
uint32_t rand_uint32(struct rng_state* state);
uint64_t rand_uint64(struct rng_state* state);
uint64_t rand_interval(const uint64_t bound, struct rng_state* state);
void rand_choice(const uint64_t bound, const uint64_t num_samples, struct rng_state* state, uint64_t* ret);
double randu(struct rng_state* state);
float randuf(struct rng_state* state);
double randn(struct rng_state* state);
float randnf(struct rng_state* state);
void normalize_statevector(struct statevector* psi);                                  /* src/statevector.h:23 */
/* src/statevector.h:29 -- real normal entries (src/statevector.c:115-121), drawn on the GPU */
void haar_random_statevector(struct statevector* psi, struct rng_state* rng);
int allocate_statevector_array(int nqubits, int nstates, struct statevector_array* psi_list);  /* src/statevector.h:47 */
void free_statevector_array(struct statevector_array* psi_list);                               /* src/statevector.h:49 */

/* ------------------------------------------------------------------ gate.h */

void apply_gate(const struct mat4x4* gate, const int i, const int j,
	const struct statevector* psi, struct statevector* psi_out);                      /* src/gate.h:7 */
void apply_gate_backward(const struct mat4x4* gate, const int i, const int j, const struct statevector* psi,
	const struct statevector* dpsi_out, struct statevector* dpsi, struct mat4x4* dgate);  /* src/gate.h:9-10 */
void apply_gate_to_array(const struct mat4x4* gate, const int i, const int j, const struct statevector_array* psi,
	struct statevector_array* psi_out);                                               /* src/gate.h:13 */
void apply_gate_backward_array(const struct mat4x4* gate, const int i, const int j, const struct statevector_array* psi,
	const struct statevector* dpsi_out, struct mat4x4* dgates);                       /* src/gate.h:15-16 */
void apply_gate_placeholder(const int i, const int j, const struct statevector* psi,
	struct statevector_array* psi_out);                                               /* src/gate.h:19 */

/* ------------------------------------------------------------------ quantum_circuit.h */

int apply_quantum_circuit(const struct mat4x4 gates[], const int ngates, const int wires[],
	const struct statevector* psi, struct statevector* psi_out);                      /* src/quantum_circuit.h:7-8 */
int allocate_quantum_circuit_cache(const int nqubits, const int ngates, struct quantum_circuit_cache* cache);  /* :23 */
void free_quantum_circuit_cache(struct quantum_circuit_cache* cache);                /* src/quantum_circuit.h:25 */
int quantum_circuit_forward(const struct mat4x4 gates[], const int ngates, const int wires[],
	const struct statevector* psi, struct quantum_circuit_cache* cache, struct statevector* psi_out);  /* :27-28 */
int quantum_circuit_backward(const struct mat4x4 gates[], const int ngates, const int wires[], const struct quantum_circuit_cache* cache,
	const struct statevector* dpsi_out, struct statevector* dpsi, struct mat4x4 dgates[]);  /* :30-31 */
int quantum_circuit_gates_hessian_vector_product(const struct mat4x4 gates[], const struct mat4x4 gatedirs[], const int ngates, const int wires[],
	const struct statevector* psi, const struct statevector* phi,
	struct statevector* psi_out, struct mat4x4 dgates[], struct mat4x4 hess_gatedirs[]);  /* :34-36 */

/* ------------------------------------------------------------------ brickwall_circuit.h */

int apply_brickwall_unitary(const struct mat4x4 vlist[], const int nlayers, const int* perms[],
	const struct statevector* psi, struct statevector* psi_out);                      /* src/brickwall_circuit.h:8-9 */
int brickwall_unitary_forward(const struct mat4x4 vlist[], int nlayers, const int* perms[],
	const struct statevector* psi, struct quantum_circuit_cache* cache, struct statevector* psi_out);  /* :11-12 */
int brickwall_unitary_backward(const struct mat4x4 vlist[], int nlayers, const int* perms[], const struct quantum_circuit_cache* cache,
	const struct statevector* dpsi_out, struct statevector* dpsi, struct mat4x4 dvlist[]);  /* :14-15 */
/* src/brickwall_circuit.h:17-18 -- hess: (16 nlayers)^2, entry ((i*16 + x)*nlayers + j)*16 + y */
int brickwall_unitary_backward_hessian(const struct mat4x4 vlist[], int nlayers, const int* perms[], const struct quantum_circuit_cache* cache,
	const struct statevector* dpsi_out, struct statevector* dpsi, struct mat4x4 dvlist[], numeric* hess);
int apply_brickwall_unitary_gate_placeholder(const struct mat4x4 vlist[], int nlayers, const int* perms[], int l,
	const struct quantum_circuit_cache* cache, struct statevector_array* psi_out);   /* src/brickwall_circuit.h:21-22 */

/* ------------------------------------------------------------------ target.h (real build) */

int circuit_unitary_target(linear_func ufunc, void* udata,
	const struct mat4x4 gates[], const int ngates, const int wires[], const int nqubits,
	numeric* fval);                                                                   /* src/target.h:10-12 */
int circuit_unitary_target_sampling(linear_func ufunc, void* udata,
	const struct mat4x4 gates[], const int ngates, const int wires[], const int nqubits,
	const long nsamples, struct rng_state* rng, numeric* fval);                      /* src/target.h:14-17 */
int circuit_unitary_target_and_gradient(linear_func ufunc, void* udata,
	const struct mat4x4 gates[], const int ngates, const int wires[], const int nqubits,
	numeric* fval, struct mat4x4 dgates[]);                                           /* src/target.h:20-22 */
/* src/target.h:24-26 -- grad_vec: 6 per gate */
int circuit_unitary_target_and_projected_gradient(linear_func ufunc, void* udata,
	const struct mat4x4 gates[], const int ngates, const int wires[], const int nqubits,
	numeric* fval, double* grad_vec);
int circuit_unitary_target_hessian_vector_product(linear_func ufunc, void* udata,
	const struct mat4x4 gates[], const struct mat4x4 gatedirs[], const int ngates, const int wires[], const int nqubits,
	numeric* fval, struct mat4x4 dgates[], struct mat4x4 hess_gatedirs[]);           /* src/target.h:29-31 */
int circuit_unitary_target_projected_hessian_vector_product(linear_func ufunc, void* udata,
	const struct mat4x4 gates[], const struct mat4x4 gatedirs[], const int ngates, const int wires[], const int nqubits,
	numeric* fval, double* grad_vec, double* hvp_vec);                               /* src/target.h:33-35 */
int brickwall_unitary_target(linear_func ufunc, void* udata,
	const struct mat4x4 vlist[], const int nlayers, const int nqubits, const int* perms[],
	numeric* fval);                                                                   /* src/target.h:42-44 */
int brickwall_unitary_target_sampling(linear_func ufunc, void* udata,
	const struct mat4x4 vlist[], const int nlayers, const int nqubits, const int* perms[],
	const long nsamples, struct rng_state* rng, numeric* fval);                      /* src/target.h:46-49 */
int brickwall_unitary_target_and_gradient(linear_func ufunc, void* udata,
	const struct mat4x4 vlist[], const int nlayers, const int nqubits, const int* perms[],
	numeric* fval, struct mat4x4 dvlist[]);                                           /* src/target.h:52-54 */
int brickwall_unitary_target_and_projected_gradient(linear_func ufunc, void* udata,
	const struct mat4x4 vlist[], const int nlayers, const int nqubits, const int* perms[],
	numeric* fval, double* grad_vec);                                                 /* src/target.h:56-58 */
int brickwall_unitary_target_hessian_vector_product(linear_func ufunc, void* udata,
	const struct mat4x4 vlist[], const struct mat4x4 vdirs[], const int nlayers, const int* perms[], const int nqubits,
	numeric* fval, struct mat4x4 dvlist[], struct mat4x4 hess_vdirs[]);              /* src/target.h:61-63 */
int brickwall_unitary_target_projected_hessian_vector_product(linear_func ufunc, void* udata,
	const struct mat4x4 vlist[], const struct mat4x4 vdirs[], const int nlayers, const int* perms[], const int nqubits,
	numeric* fval, double* grad_vec, double* hvp_vec);                               /* src/target.h:65-67 */
int brickwall_unitary_target_gradient_hessian(linear_func ufunc, void* udata,
	const struct mat4x4 vlist[], const int nlayers, const int nqubits, const int* perms[],
	numeric* fval, struct mat4x4 dvlist[], numeric* hess);                           /* src/target.h:70-72 */
int brickwall_unitary_target_gradient_hessian_sampling(linear_func ufunc, void* udata,
	const struct mat4x4 vlist[], const int nlayers, const int nqubits, const int* perms[],
	const long nsamples, struct rng_state* rng,
	numeric* fval, struct mat4x4 dvlist[], numeric* hess);                           /* src/target.h:74-77 */
int brickwall_blockenc_target(linear_func hfunc, void* hdata,
	const struct mat4x4 vlist[], const int nlayers, const int nqubits, const int* perms[],
	double* fval);                                                                    /* src/target.h:96-98 */
int brickwall_blockenc_target_and_gradient(linear_func hfunc, void* hdata,
	const struct mat4x4 vlist[], const int nlayers, const int nqubits, const int* perms[],
	double* fval, struct mat4x4 dvlist[]);                                            /* src/target.h:101-103 */
/* src/target.h:113-121 (real build: one Hessian, the sum of the two terms, src/target.c:1595-1597) */
int brickwall_blockenc_target_gradient_hessian(linear_func hfunc, void* hdata,
	const struct mat4x4 vlist[], const int nlayers, const int nqubits, const int* perms[],
	double* fval, struct mat4x4 dvlist[], numeric* hess);

/* ------------------------------------------------------------------ trust_region.h */

struct truncated_cg_params
{
	int maxiter;
	double abstol;
	double reltol;
};                                                                                    /* src/trust_region.h:10-16 */

static inline void set_truncated_cg_default_params(int n, struct truncated_cg_params* params)
{
	params->maxiter = 2 * n;
	params->abstol  = 1e-8;
	params->reltol  = 1e-6;
}                                                                                     /* src/trust_region.h:23-28 */

bool truncated_cg_hmat(const double* grad, const double* hess, int n, double radius,
	const struct truncated_cg_params* params, double* z);                            /* src/trust_region.h:31 */

typedef void (*hessian_vector_product_func)(const double* x, void* fdata, double* vec, double* hvp);  /* :34 */
typedef double (*target_func)(const double* x, void* fdata);                          /* src/trust_region.h:39 */
typedef double (*target_gradient_func)(const double* x, void* fdata, double* grad);   /* src/trust_region.h:41 */
typedef double (*target_gradient_hessian_func)(const double* x, void* fdata, double* grad, double* hess);  /* :43 */
typedef void (*retract_func)(const double* x, const double* eta, void* rdata, double* xs);  /* :45 */

struct rtr_params
{
	struct truncated_cg_params tcg_params;
	double rho_trust;
	double radius_init;
	double maxradius;
	target_func g_func;
	void*       g_data;
	double*     g_iter;
};                                                                                    /* src/trust_region.h:52-61 */

static inline void set_rtr_default_params(int n, struct rtr_params* params)
{
	set_truncated_cg_default_params(n, &params->tcg_params);
	params->rho_trust   = 0.125;
	params->radius_init = 0.01;
	params->maxradius   = 0.1;
	params->g_func      = NULL;
	params->g_data      = NULL;
	params->g_iter      = NULL;
}                                                                                     /* src/trust_region.h:68-77 */

bool truncated_cg_hvp(const double* x, const double* grad, const hessian_vector_product_func f_hvp, void* fdata,
	const int n, const double radius, const struct truncated_cg_params* params, double* z);  /* :36 */
void riemannian_trust_region_optimize_hmat(target_func f, target_gradient_hessian_func f_deriv_hess, void* fdata,
	retract_func retract, void* rdata, const int n, const double* x_init, const int m,
	const struct rtr_params* params, const int niter, double* f_iter, double* x_final);  /* :80-81 */
void riemannian_trust_region_optimize_hvp(const target_func f, const target_gradient_func f_deriv,
	const hessian_vector_product_func f_hvp, void* fdata, retract_func retract, void* rdata,
	const int n, const double* x_init, const int m, const struct rtr_params* params, const int niter,
	double* f_iter, double* x_final);                                                 /* src/trust_region.h:83-85 */

/* ------------------------------------------------------------------ brickwall_opt.h, circuit_opt.h */

/* src/brickwall_opt.h:8-10 -- 6 nlayers tangent parameters */
void optimize_brickwall_circuit_hvp(linear_func ufunc, void* udata,
	const struct mat4x4 vlist_start[], const int nlayers, const int nqubits, const int* perms[],
	struct rtr_params* params, const int niter, double* f_iter, struct mat4x4 vlist_opt[]);
/* src/circuit_opt.h:8 */
void optimize_quantum_circuit(linear_func ufunc, void* udata, const struct mat4x4 gates_start[], const int ngates,
	const int nqubits, const int wires[], struct rtr_params* params, const int niter, double* f_iter,
	struct mat4x4 gates_opt[]);

/* ------------------------------------------------------------------ matrix.h (real build) */

/* src/matrix.h:44-46 */
static const int num_tangent_params = 6;

void zero_matrix(struct mat4x4* a);                                          /* src/matrix.h:16 */
void identity_matrix(struct mat4x4* a);                                      /* src/matrix.h:18 */
void scale_matrix(struct mat4x4* a, const double x);                         /* src/matrix.h:21 */
void conjugate_matrix(struct mat4x4* a);                                     /* src/matrix.h:24 -- no-op */
void add_matrix(struct mat4x4* a, const struct mat4x4* b);                   /* src/matrix.h:27 */
void sub_matrix(struct mat4x4* a, const struct mat4x4* b);                   /* src/matrix.h:28 */
void add_matrices(const struct mat4x4* a, const struct mat4x4* b, struct mat4x4* c);  /* src/matrix.h:30 */
void sub_matrices(const struct mat4x4* a, const struct mat4x4* b, struct mat4x4* c);  /* src/matrix.h:31 */
void transpose(const struct mat4x4* a, struct mat4x4* at);                   /* src/matrix.h:34 */
void adjoint(const struct mat4x4* a, struct mat4x4* ah);                     /* src/matrix.h:35 */
void symm(const struct mat4x4* w, struct mat4x4* z);                         /* src/matrix.h:38 */
void antisymm(const struct mat4x4* w, struct mat4x4* z);                     /* src/matrix.h:39 */
void real_to_antisymm(const double* r, struct mat4x4* w);                    /* src/matrix.h:48 -- 6 entries */
void antisymm_to_real(const struct mat4x4* w, double* r);                    /* src/matrix.h:49 -- 6 entries */
void real_to_tangent(const double* r, const struct mat4x4* v, struct mat4x4* z);       /* src/matrix.h:51 */
void tangent_to_real(const struct mat4x4* v, const struct mat4x4* z, double* r);       /* src/matrix.h:52 */
void project_tangent(const struct mat4x4* u, const struct mat4x4* z, struct mat4x4* p); /* src/matrix.h:55 */
void multiply_matrices(const struct mat4x4* a, const struct mat4x4* b, struct mat4x4* c); /* src/matrix.h:58 */
void symmetric_triple_matrix_product(const struct mat4x4* a, const struct mat4x4* b,
	const struct mat4x4* c, struct mat4x4* ret);                                 /* src/matrix.h:61 */
int inverse_matrix(const struct mat4x4* a, struct mat4x4* ainv);            /* src/matrix.h:64 */
void polar_factor(const struct mat4x4* a, struct mat4x4* u);                 /* src/matrix.h:67 */
void retract(const struct mat4x4* u, const double* eta, struct mat4x4* v);   /* src/matrix.h:70 -- 6 entries */

/* ------------------------------------------------------------------ util.h */

double uniform_distance_real(long n, const double* x, const double* y);     /* src/util.h:19 */
double uniform_distance(long n, const numeric* x, const numeric* y);        /* src/util.h:21 */
double relative_distance(long n, const numeric* x, const numeric* y, double eps);  /* src/util.h:23 */

/* ==================================================================================
 * Additions (no counterpart in the reference), as in rqcopt_gpu.h with real gates
 * ================================================================================== */

struct rqcopt_brickwall_target
{
	const struct mat4x4* vlist;
	int nlayers;
	const int* const* perms;
};
int rqcopt_brickwall_ufunc(const struct statevector* psi, void* udata, struct statevector* psi_out);

struct rqcopt_circuit_target
{
	const struct mat4x4* gates;
	int ngates;
	const int* wires;
};
int rqcopt_circuit_ufunc(const struct statevector* psi, void* udata, struct statevector* psi_out);

struct rqcopt_dense_target
{
	const numeric* u;
	int nqubits;
};
int rqcopt_dense_ufunc(const struct statevector* psi, void* udata, struct statevector* psi_out);

/* forwarded to librqcopt_gpu.so (see rqcopt_gpu.h) */
int rqcopt_gpu_set_precision(int precision);
int rqcopt_gpu_last_error(void);
unsigned long long rqcopt_gpu_launch_count(void);
void rqcopt_gpu_reset_launch_count(void);

#ifdef __cplusplus
}
#endif
