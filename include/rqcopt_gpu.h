/*
 * rqcopt_gpu.h -- C ABI of the B200 library librqcopt_gpu.so.
 *
 * The first part declares, with identical names, argument types and meaning,
 * the functions of cmendl/rqcopt_hpc on the matrix-free circuit-optimisation
 * path, so that C host code written against the reference headers links
 * against this library unchanged.  Every declaration names the reference
 * declaration it replaces (path:line within the reference project).  The
 * second part declares additions that have no counterpart in the reference.
 *
 * Conventions (as in the reference, COMPLEX_CIRCUIT build):
 *   - `numeric` is double complex; a statevector holds 2^nqubits amplitudes,
 *     qubit 0 is the most significant bit of the amplitude index;
 *   - `struct mat4x4` is a row-major 4x4 gate whose row/column index is
 *     2*b_i + b_j for the bits of its wires (i, j);
 *   - every call is synchronous: when it returns, all GPU work it issued has
 *     finished and its outputs are visible to the host;
 *   - statevector data pointers may be host memory (pageable or pinned),
 *     CUDA managed memory (what allocate_statevector returns) or device
 *     memory of the current device; host buffers are staged through HBM;
 *   - int-returning functions return 0 on success and a negative code on
 *     failure: -1 allocation, -2 target-callback failure, -3/-4 internal pass
 *     failure, -5 CUDA error, -6 invalid argument (the last two are additions);
 *   - void functions that receive invalid arguments print a message to stderr,
 *     leave their outputs untouched and record the error, readable through
 *     rqcopt_gpu_last_error().
 */
#pragma once

#ifdef __cplusplus
#include <complex>
typedef std::complex<double> numeric;
extern "C" {
#else
#include <complex.h>
#include <stdbool.h>
typedef double complex numeric;
#endif

#include <stddef.h>
#include <stdint.h>

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

/* src/pcg_basic.h:32-36 -- the PCG32 generator (state, stream) */
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

/* src/statevector.h:18 -- returns CUDA managed memory (host- and device-accessible) */
int allocate_statevector(int nqubits, struct statevector* psi);
/* src/statevector.h:20 */
void free_statevector(struct statevector* psi);
/* src/statevector.h:32 */
void add_statevectors(const struct statevector* psi1, const struct statevector* psi2, struct statevector* psi_sum);
/* src/statevector.h:26 -- permutes qubit wires on the host (device statevectors through host copies) */
void transpose_statevector(const struct statevector* psi, const int* perm, struct statevector* psi_trans);
/* src/rng.h:21 */
void seed_rng_state(const uint64_t seed, struct rng_state* state);

/* src/pcg_basic.h:38-60 -- the PCG32 generator and its pair (host) */
void pcg32_srandom_r(const uint64_t initstate, const uint64_t initseq, struct pcg32_random* rng);
uint32_t pcg32_random_r(struct pcg32_random* rng);
uint32_t pcg32_boundedrand_r(const uint32_t bound, struct pcg32_random* rng);
void pcg32x2_srandom_r(uint64_t seed1, uint64_t seed2, uint64_t seq1, uint64_t seq2, struct pcg32x2_random* rng);
uint64_t pcg32x2_random_r(struct pcg32x2_random* rng);
uint64_t pcg32x2_boundedrand_r(const uint64_t bound, struct pcg32x2_random* rng);
/* src/rng.h:29-67 -- random numbers from rng_state (host, the reference's stream) */
uint32_t rand_uint32(struct rng_state* state);
uint64_t rand_uint64(struct rng_state* state);
uint64_t rand_interval(const uint64_t bound, struct rng_state* state);
void rand_choice(const uint64_t bound, const uint64_t num_samples, struct rng_state* state, uint64_t* ret);
double randu(struct rng_state* state);
float randuf(struct rng_state* state);
double randn(struct rng_state* state);
float randnf(struct rng_state* state);
#ifdef __cplusplus
std::complex<double> crandn(struct rng_state* state);
std::complex<float> crandnf(struct rng_state* state);
#else
double complex crandn(struct rng_state* state);
float complex crandnf(struct rng_state* state);
#endif
/* src/statevector.h:23 -- on the host (device statevectors through host copies) */
void normalize_statevector(struct statevector* psi);
/* src/statevector.h:29 -- generated on the GPU; advances rng exactly as the reference does */
void haar_random_statevector(struct statevector* psi, struct rng_state* rng);
/* src/statevector.h:47 -- returns CUDA managed memory */
int allocate_statevector_array(int nqubits, int nstates, struct statevector_array* psi_list);
/* src/statevector.h:49 */
void free_statevector_array(struct statevector_array* psi_list);

/* ------------------------------------------------------------------ gate.h */

/* src/gate.h:7 */
void apply_gate(const struct mat4x4* gate, const int i, const int j,
	const struct statevector* psi, struct statevector* psi_out);
/* src/gate.h:9-10 */
void apply_gate_backward(const struct mat4x4* gate, const int i, const int j, const struct statevector* psi,
	const struct statevector* dpsi_out, struct statevector* dpsi, struct mat4x4* dgate);
/* src/gate.h:13 */
void apply_gate_to_array(const struct mat4x4* gate, const int i, const int j, const struct statevector_array* psi, struct statevector_array* psi_out);
/* src/gate.h:15-16 */
void apply_gate_backward_array(const struct mat4x4* gate, const int i, const int j, const struct statevector_array* psi,
	const struct statevector* dpsi_out, struct mat4x4* dgates);
/* src/gate.h:19 -- psi_out->nstates must be 16 */
void apply_gate_placeholder(const int i, const int j, const struct statevector* psi, struct statevector_array* psi_out);

/* ------------------------------------------------------------------ quantum_circuit.h */

/* src/quantum_circuit.h:7-8 */
int apply_quantum_circuit(const struct mat4x4 gates[], const int ngates, const int wires[],
	const struct statevector* psi, struct statevector* psi_out);
/* src/quantum_circuit.h:23 -- cache states are CUDA managed memory */
int allocate_quantum_circuit_cache(const int nqubits, const int ngates, struct quantum_circuit_cache* cache);
/* src/quantum_circuit.h:25 */
void free_quantum_circuit_cache(struct quantum_circuit_cache* cache);
/* src/quantum_circuit.h:27-28 */
int quantum_circuit_forward(const struct mat4x4 gates[], const int ngates, const int wires[],
	const struct statevector* psi, struct quantum_circuit_cache* cache, struct statevector* psi_out);
/* src/quantum_circuit.h:30-31 */
int quantum_circuit_backward(const struct mat4x4 gates[], const int ngates, const int wires[], const struct quantum_circuit_cache* cache,
	const struct statevector* dpsi_out, struct statevector* dpsi, struct mat4x4 dgates[]);
/* src/quantum_circuit.h:34-36 */
int quantum_circuit_gates_hessian_vector_product(const struct mat4x4 gates[], const struct mat4x4 gatedirs[], const int ngates, const int wires[],
	const struct statevector* psi, const struct statevector* phi,
	struct statevector* psi_out, struct mat4x4 dgates[], struct mat4x4 hess_gatedirs[]);

/* ------------------------------------------------------------------ brickwall_circuit.h */

/* src/brickwall_circuit.h:8-9 */
int apply_brickwall_unitary(const struct mat4x4 vlist[], const int nlayers, const int* perms[],
	const struct statevector* psi, struct statevector* psi_out);
/* src/brickwall_circuit.h:11-12 */
int brickwall_unitary_forward(const struct mat4x4 vlist[], int nlayers, const int* perms[],
	const struct statevector* psi, struct quantum_circuit_cache* cache, struct statevector* psi_out);
/* src/brickwall_circuit.h:14-15 */
int brickwall_unitary_backward(const struct mat4x4 vlist[], int nlayers, const int* perms[], const struct quantum_circuit_cache* cache,
	const struct statevector* dpsi_out, struct statevector* dpsi, struct mat4x4 dvlist[]);
/* src/brickwall_circuit.h:17-18 -- hess: (16 nlayers)^2 row-major, entry ((i*16 + x)*nlayers + j)*16 + y */
int brickwall_unitary_backward_hessian(const struct mat4x4 vlist[], int nlayers, const int* perms[], const struct quantum_circuit_cache* cache,
	const struct statevector* dpsi_out, struct statevector* dpsi, struct mat4x4 dvlist[], numeric* hess);
/* src/brickwall_circuit.h:21-22 */
int apply_brickwall_unitary_gate_placeholder(const struct mat4x4 vlist[], int nlayers, const int* perms[], int l,
	const struct quantum_circuit_cache* cache, struct statevector_array* psi_out);

/* ------------------------------------------------------------------ target.h */

/* src/target.h:10-12 */
int circuit_unitary_target(linear_func ufunc, void* udata,
	const struct mat4x4 gates[], const int ngates, const int wires[], const int nqubits,
	numeric* fval);
/* src/target.h:14-17 -- Haar-random sample states drawn on the GPU from rng's stream */
int circuit_unitary_target_sampling(linear_func ufunc, void* udata,
	const struct mat4x4 gates[], const int ngates, const int wires[], const int nqubits,
	const long nsamples, struct rng_state* rng,
	numeric* fval);
/* src/target.h:20-22 */
int circuit_unitary_target_and_gradient(linear_func ufunc, void* udata,
	const struct mat4x4 gates[], const int ngates, const int wires[], const int nqubits,
	numeric* fval, struct mat4x4 dgates[]);
/* src/target.h:24-26 */
int circuit_unitary_target_and_projected_gradient(linear_func ufunc, void* udata,
	const struct mat4x4 gates[], const int ngates, const int wires[], const int nqubits,
	numeric* fval, double* grad_vec);
/* src/target.h:29-31 */
int circuit_unitary_target_hessian_vector_product(linear_func ufunc, void* udata,
	const struct mat4x4 gates[], const struct mat4x4 gatedirs[], const int ngates, const int wires[], const int nqubits,
	numeric* fval, struct mat4x4 dgates[], struct mat4x4 hess_gatedirs[]);
/* src/target.h:33-35 */
int circuit_unitary_target_projected_hessian_vector_product(linear_func ufunc, void* udata,
	const struct mat4x4 gates[], const struct mat4x4 gatedirs[], const int ngates, const int wires[], const int nqubits,
	numeric* fval, double* grad_vec, double* hvp_vec);
/* src/target.h:42-44 */
int brickwall_unitary_target(linear_func ufunc, void* udata,
	const struct mat4x4 vlist[], const int nlayers, const int nqubits, const int* perms[],
	numeric* fval);
/* src/target.h:46-49 */
int brickwall_unitary_target_sampling(linear_func ufunc, void* udata,
	const struct mat4x4 vlist[], const int nlayers, const int nqubits, const int* perms[],
	const long nsamples, struct rng_state* rng,
	numeric* fval);
/* src/target.h:52-54 */
int brickwall_unitary_target_and_gradient(linear_func ufunc, void* udata,
	const struct mat4x4 vlist[], const int nlayers, const int nqubits, const int* perms[],
	numeric* fval, struct mat4x4 dvlist[]);
/* src/target.h:56-58 */
int brickwall_unitary_target_and_projected_gradient(linear_func ufunc, void* udata,
	const struct mat4x4 vlist[], const int nlayers, const int nqubits, const int* perms[],
	numeric* fval, double* grad_vec);
/* src/target.h:61-63 */
int brickwall_unitary_target_hessian_vector_product(linear_func ufunc, void* udata,
	const struct mat4x4 vlist[], const struct mat4x4 vdirs[], const int nlayers, const int* perms[], const int nqubits,
	numeric* fval, struct mat4x4 dvlist[], struct mat4x4 hess_vdirs[]);
/* src/target.h:65-67 */
int brickwall_unitary_target_projected_hessian_vector_product(linear_func ufunc, void* udata,
	const struct mat4x4 vlist[], const struct mat4x4 vdirs[], const int nlayers, const int* perms[], const int nqubits,
	numeric* fval, double* grad_vec, double* hvp_vec);

/* src/target.h:70-72 -- complex (16 nlayers)^2 Hessian, layout as brickwall_unitary_backward_hessian */
int brickwall_unitary_target_gradient_hessian(linear_func ufunc, void* udata,
	const struct mat4x4 vlist[], const int nlayers, const int nqubits, const int* perms[],
	numeric* fval, struct mat4x4 dvlist[], numeric* hess);
/* src/target.h:81-83 -- real symmetric (16 nlayers)^2 Riemannian Hessian H */
int brickwall_unitary_target_gradient_vector_hessian_matrix(linear_func ufunc, void* udata,
	const struct mat4x4 vlist[], const int nlayers, const int nqubits, const int* perms[],
	numeric* fval, double* grad_vec, double* H);
/* src/target.h:74-77 */
int brickwall_unitary_target_gradient_hessian_sampling(linear_func ufunc, void* udata,
	const struct mat4x4 vlist[], const int nlayers, const int nqubits, const int* perms[],
	const long nsamples, struct rng_state* rng,
	numeric* fval, struct mat4x4 dvlist[], numeric* hess);
/* src/target.h:85-88 */
int brickwall_unitary_target_gradient_vector_hessian_matrix_sampling(linear_func ufunc, void* udata,
	const struct mat4x4 vlist[], const int nlayers, const int nqubits, const int* perms[],
	const long nsamples, struct rng_state* rng,
	numeric* fval, double* grad_vec, double* H);

/* src/target.h:96-98 -- block-encoding target || P^dag W P - H ||_F^2 / 2; hfunc acts on
 * nqubits / 2 qubits (the even-numbered ones; P puts the odd ones in |0>) */
int brickwall_blockenc_target(linear_func hfunc, void* hdata,
	const struct mat4x4 vlist[], const int nlayers, const int nqubits, const int* perms[],
	double* fval);
/* src/target.h:101-103 */
int brickwall_blockenc_target_and_gradient(linear_func hfunc, void* hdata,
	const struct mat4x4 vlist[], const int nlayers, const int nqubits, const int* perms[],
	double* fval, struct mat4x4 dvlist[]);
/* src/target.h:106-108 */
int brickwall_blockenc_target_and_gradient_vector(linear_func hfunc, void* hdata,
	const struct mat4x4 vlist[], const int nlayers, const int nqubits, const int* perms[],
	double* fval, double* grad_vec);
/* src/target.h:113-121 (COMPLEX_CIRCUIT form: hess1 the second derivative of the residual's
 * backward pass, hess2 the Gauss-Newton term) */
int brickwall_blockenc_target_gradient_hessian(linear_func hfunc, void* hdata,
	const struct mat4x4 vlist[], const int nlayers, const int nqubits, const int* perms[],
	double* fval, struct mat4x4 dvlist[], numeric* hess1, numeric* hess2);
/* src/target.h:124-126 */
int brickwall_blockenc_target_gradient_vector_hessian_matrix(linear_func hfunc, void* hdata,
	const struct mat4x4 vlist[], const int nlayers, const int nqubits, const int* perms[],
	double* fval, double* grad_vec, double* H);

/* ------------------------------------------------------------------ trust_region.h */

/* src/trust_region.h:10-16 */
struct truncated_cg_params
{
	int maxiter;
	double abstol;
	double reltol;
};

/* src/trust_region.h:23-28 */
static inline void set_truncated_cg_default_params(int n, struct truncated_cg_params* params)
{
	params->maxiter = 2 * n;
	params->abstol  = 1e-8;
	params->reltol  = 1e-6;
}

/* src/trust_region.h:31 */
bool truncated_cg_hmat(const double* grad, const double* hess, int n, double radius, const struct truncated_cg_params* params, double* z);

/* src/trust_region.h:34 */
typedef void (*hessian_vector_product_func)(const double* x, void* fdata, double* vec, double* hvp);
/* src/trust_region.h:39 */
typedef double (*target_func)(const double* x, void* fdata);
/* src/trust_region.h:41 */
typedef double (*target_gradient_func)(const double* x, void* fdata, double* grad);
/* src/trust_region.h:43 */
typedef double (*target_gradient_hessian_func)(const double* x, void* fdata, double* grad, double* hess);
/* src/trust_region.h:45 */
typedef void (*retract_func)(const double* x, const double* eta, void* rdata, double* xs);

/* src/trust_region.h:52-61 */
struct rtr_params
{
	struct truncated_cg_params tcg_params;
	double rho_trust;
	double radius_init;
	double maxradius;
	target_func g_func;
	void*       g_data;
	double*     g_iter;
};

/* src/trust_region.h:68-77 */
static inline void set_rtr_default_params(int n, struct rtr_params* params)
{
	set_truncated_cg_default_params(n, &params->tcg_params);
	params->rho_trust   = 0.125;
	params->radius_init = 0.01;
	params->maxradius   = 0.1;
	params->g_func      = NULL;
	params->g_data      = NULL;
	params->g_iter      = NULL;
}

/* src/trust_region.h:36 */
bool truncated_cg_hvp(const double* x, const double* grad, const hessian_vector_product_func f_hvp, void* fdata,
	const int n, const double radius, const struct truncated_cg_params* params, double* z);
/* src/trust_region.h:80-81 */
void riemannian_trust_region_optimize_hmat(target_func f, target_gradient_hessian_func f_deriv_hess, void* fdata, retract_func retract, void* rdata,
	const int n, const double* x_init, const int m, const struct rtr_params* params, const int niter, double* f_iter, double* x_final);
/* src/trust_region.h:83-85 */
void riemannian_trust_region_optimize_hvp(const target_func f, const target_gradient_func f_deriv,
	const hessian_vector_product_func f_hvp, void* fdata, retract_func retract, void* rdata,
	const int n, const double* x_init, const int m, const struct rtr_params* params, const int niter,
	double* f_iter, double* x_final);

/* ------------------------------------------------------------------ brickwall_opt.h, circuit_opt.h */

/* src/brickwall_opt.h:8-10 */
void optimize_brickwall_circuit_hvp(linear_func ufunc, void* udata,
	const struct mat4x4 vlist_start[], const int nlayers, const int nqubits, const int* perms[],
	struct rtr_params* params, const int niter, double* f_iter, struct mat4x4 vlist_opt[]);
/* src/brickwall_opt.h:15-17 -- complex128 regardless of rqcopt_gpu_set_precision */
void optimize_brickwall_circuit_hmat(linear_func ufunc, void* udata,
	const struct mat4x4 vlist_start[], const int nlayers, const int nqubits, const int* perms[],
	struct rtr_params* params, const int niter, double* f_iter, struct mat4x4 vlist_opt[]);
/* src/brickwall_opt.h:19-22 */
void optimize_brickwall_circuit_hmat_sampling(linear_func ufunc, void* udata,
	const struct mat4x4 vlist_start[], const int nlayers, const int nqubits, const int* perms[],
	const long nsamples, struct rng_state* rng,
	struct rtr_params* params, const int niter, double* f_iter, struct mat4x4 vlist_opt[]);
/* src/circuit_opt.h:8 */
void optimize_quantum_circuit(linear_func ufunc, void* udata, const struct mat4x4 gates_start[], const int ngates,
	const int nqubits, const int wires[], struct rtr_params* params, const int niter, double* f_iter,
	struct mat4x4 gates_opt[]);

/* ------------------------------------------------------------------ matrix.h */

/* src/matrix.h:42-46 (COMPLEX_CIRCUIT) */
static const int num_tangent_params = 16;

void zero_matrix(struct mat4x4* a);                                          /* src/matrix.h:16 */
void identity_matrix(struct mat4x4* a);                                      /* src/matrix.h:18 */
void scale_matrix(struct mat4x4* a, const double x);                         /* src/matrix.h:21 */
void conjugate_matrix(struct mat4x4* a);                                     /* src/matrix.h:24 */
void add_matrix(struct mat4x4* a, const struct mat4x4* b);                   /* src/matrix.h:27 */
void sub_matrix(struct mat4x4* a, const struct mat4x4* b);                   /* src/matrix.h:28 */
void add_matrices(const struct mat4x4* a, const struct mat4x4* b, struct mat4x4* c);  /* src/matrix.h:30 */
void sub_matrices(const struct mat4x4* a, const struct mat4x4* b, struct mat4x4* c);  /* src/matrix.h:31 */
void transpose(const struct mat4x4* a, struct mat4x4* at);                   /* src/matrix.h:34 */
void adjoint(const struct mat4x4* a, struct mat4x4* ah);                     /* src/matrix.h:35 */
void symm(const struct mat4x4* w, struct mat4x4* z);                         /* src/matrix.h:38 */
void antisymm(const struct mat4x4* w, struct mat4x4* z);                     /* src/matrix.h:39 */
void real_to_antisymm(const double* r, struct mat4x4* w);                    /* src/matrix.h:48 */
void antisymm_to_real(const struct mat4x4* w, double* r);                    /* src/matrix.h:49 */
void real_to_tangent(const double* r, const struct mat4x4* v, struct mat4x4* z);       /* src/matrix.h:51 */
void tangent_to_real(const struct mat4x4* v, const struct mat4x4* z, double* r);       /* src/matrix.h:52 */
void project_tangent(const struct mat4x4* u, const struct mat4x4* z, struct mat4x4* p); /* src/matrix.h:55 */
void multiply_matrices(const struct mat4x4* a, const struct mat4x4* b, struct mat4x4* c); /* src/matrix.h:58 */
void symmetric_triple_matrix_product(const struct mat4x4* a, const struct mat4x4* b,
	const struct mat4x4* c, struct mat4x4* ret);                                 /* src/matrix.h:61 */
int inverse_matrix(const struct mat4x4* a, struct mat4x4* ainv);            /* src/matrix.h:64 */
void polar_factor(const struct mat4x4* a, struct mat4x4* u);                 /* src/matrix.h:67 */
void retract(const struct mat4x4* u, const double* eta, struct mat4x4* v);   /* src/matrix.h:70 */

/* ------------------------------------------------------------------ util.h */

double uniform_distance_real(long n, const double* x, const double* y);     /* src/util.h:19 */
double uniform_distance(long n, const numeric* x, const numeric* y);        /* src/util.h:21 */
double relative_distance(long n, const numeric* x, const numeric* y, double eps);  /* src/util.h:23 */

/* ==================================================================================
 * Additions (no counterpart in the reference)
 * ================================================================================== */

/*
 * Device-native targets.  These are ordinary `linear_func`s (applying a
 * brickwall or a general circuit to one column through the GPU), and the
 * target functions and optimisers recognise them by address: given one of
 * them as `ufunc`, the basis-column sums evaluate the target on the GPU next
 * to the circuit, without one host callback per column.
 */
struct rqcopt_brickwall_target
{
	const struct mat4x4* vlist;  /* nlayers gates, one per layer */
	int nlayers;
	const int* const* perms;     /* nlayers permutations of [0, nqubits) */
};
int rqcopt_brickwall_ufunc(const struct statevector* psi, void* udata, struct statevector* psi_out);

struct rqcopt_circuit_target
{
	const struct mat4x4* gates;
	int ngates;
	const int* wires;            /* 2 * ngates wire indices */
};
int rqcopt_circuit_ufunc(const struct statevector* psi, void* udata, struct statevector* psi_out);

/* Dense row-major 2^nqubits x 2^nqubits target (the Python module's U, whose `ufunc` is
 * a zgemv, pymodule/rqcopt_module.c:16-28): psi_out = U psi on the host; a basis
 * vector (one entry 1, all others 0) costs one column copy instead of the product. */
struct rqcopt_dense_target
{
	const numeric* u;
	int nqubits;
};
int rqcopt_dense_ufunc(const struct statevector* psi, void* udata, struct statevector* psi_out);

/* precision of the basis-column passes */
enum rqcopt_precision
{
	RQCOPT_PRECISION_C128  = 0,  /* complex128 end to end (the drop-in default) */
	RQCOPT_PRECISION_MIXED = 1,  /* complex64 passes, FP64 sums; optimisers switch to
	                                complex128 once the gradient norm falls below the
	                                refinement threshold */
	RQCOPT_PRECISION_C64   = 2   /* complex64 passes, FP64 sums, no refinement */
};
int rqcopt_gpu_set_precision(int precision);
int rqcopt_gpu_get_precision(void);
/* gradient-norm threshold for the switch from complex64 to complex128 (default 1e-5) */
void rqcopt_gpu_set_refine_threshold(double gnorm);

/* upper bound on the device memory (bytes) the evaluation engine may use for
 * column chunks and caches; 0 selects 75 % of the free memory at first use */
void rqcopt_gpu_set_workspace_limit(size_t bytes);
/* number of basis columns per chunk; 0 selects it from the workspace limit */
void rqcopt_gpu_set_column_chunk(long columns);

/* Restrict the basis-column sums of the target functions (circuit_unitary_target*,
 * brickwall_unitary_target* and the optimisers that call them) to the columns
 * [begin, end); end = 0 means up to the last column, and (0, 0), the default, restores
 * the full sums.  It is the column loop of src/target.c:335-369 run over a contiguous
 * sample, so that a large evaluation can be checked column by column against a CPU
 * implementation of the same range.  Returns 0, or -6 if begin < 0, end < 0 or
 * 0 < end <= begin. */
int rqcopt_gpu_set_column_range(long begin, long end);

/* gates fused per HBM round trip in the basis-column passes: 1 runs one kernel
 * per gate, 2..4 (default 4) group consecutive gates into passes over
 * eight-qubit tiles of column-interleaved chunks.  Setting it fixes it for the
 * autotuner too (as do rqcopt_gpu_set_column_chunk with a positive count and
 * rqcopt_gpu_set_reconstruct). */
int rqcopt_gpu_set_gates_per_pass(int gates);

/* Autotuning of the basis-column sums (on by default): on the first evaluation of a
 * problem shape (qubits, gates, target gates, precision, mode, paired columns) with at
 * least 2^26 amplitude x gate updates and a device-native target, the library times the
 * candidate gates-per-pass (1-4), column chunks and complex128 reverse variants on a
 * sample of up to 4096 basis columns with CUDA events and keeps the fastest for the rest
 * of the process; choices fixed by the setters above are kept.  Results are the same to
 * rounding whichever configuration runs.  rqcopt_gpu_set_autotune(1) also releases the
 * fixed choices and restores the defaults; 0 turns tuning off.  Returns 0 or -5. */
int rqcopt_gpu_set_autotune(int on);
/* configuration of the last target evaluation on this device: gates per pass, column
 * chunk (0: from the workspace), complex128 reconstruction, complex64 passes on the FP32
 * pipe (1) or the TF32 MMA (0), and the tuned sample's time per basis column in ms;
 * returns 1 if the autotuner chose it, 0 if the defaults / fixed settings ran, -5 without
 * a device */
int rqcopt_gpu_last_config(int* gates_per_pass, long* column_chunk, int* reconstruct, int* c64_fp32_pipe,
                           double* ms_per_column);
/* complex64 fused passes: 1 in FP32 FMAs, four threads per amplitude group and the gate
 * coefficients in registers; 0 (default) on the TF32 tensor-core MMA with the three-term
 * split (FP32 accuracy), which issues about half the instructions and measured faster on
 * B200.  Both meet the complex64 bar; fixing it keeps it for the autotuner. */
void rqcopt_gpu_set_c64_fp32_pipe(int on);

/* complex128 reverse passes over fused gates: 1 (default) rebuilds the state entering
 * each gate from the pass output with the adjoint gate when every gate is unitary to
 * 1e-14 (four tiles in shared memory, two blocks per SM); 0 recomputes those states
 * from the pass input.  Both give the same sums to rounding. */
void rqcopt_gpu_set_reconstruct(int on);

/* last error recorded by a void function (0 if none); reading clears it */
int rqcopt_gpu_last_error(void);

/* Per-iteration record of the last optimize_brickwall_circuit_hvp / optimize_quantum_circuit
 * call on this device (the decisions of src/trust_region.c:330-352): step accepted (rho >
 * rho_trust), tCG ended on the trust-region boundary, tCG inner iterations (Hessian-vector
 * products), and whether those products ran in complex128 (1) or complex64 (0).  Fills up to
 * `capacity` entries of each non-null array and returns the number of iterations recorded. */
int rqcopt_gpu_optimizer_trace(int* accepted, int* on_boundary, int* inner_iterations, int* refined, int capacity);

/* Haar-random sample states with real normal entries, one draw of randn() per
 * amplitude as in the reference's real build (src/statevector.c:115-121), instead
 * of complex ones; used by librqcopt_gpu_real.so (rqcopt_gpu_real.h) around its
 * sampling calls.  The generator state advances by 2 instead of 4 steps per amplitude. */
void rqcopt_gpu_set_real_samples(int on);

/* Real problems (real gates and a real target, as in librqcopt_gpu_real.so): the
 * basis-column sums of the f / gradient / HVP target functions run over the 2^(n-1)
 * paired columns e_b + i e_{b + 2^(n-1)} and keep the real parts, which are the sums
 * over all 2^n real columns (half the passes).  Results of complex problems are wrong
 * in this mode; librqcopt_gpu_real.so sets it around its calls only. */
void rqcopt_gpu_set_real_pairs(int on);

/* number of kernels this library launched since the counter was last reset */
unsigned long long rqcopt_gpu_launch_count(void);
void rqcopt_gpu_reset_launch_count(void);

/*
 * Per-kernel timing with CUDA events recorded on the launching stream.  While
 * enabled, each launch of a kernel class is bracketed by events; the totals
 * are read with rqcopt_gpu_kernel_time (milliseconds summed over launches and
 * number of launches).  Kernel classes: 0 gate apply, 1 forward tangent pass,
 * 2 reverse (gradient/HVP) pass, 3 fused multi-gate apply, 4 full-Hessian
 * tangent sweep.
 */
void rqcopt_gpu_enable_kernel_timing(int enable);
int  rqcopt_gpu_kernel_time(int kernel_class, double* total_ms, long* launches);

/* the CUDA stream (cudaStream_t) all library work is issued on */
void* rqcopt_gpu_stream(void);

/* Addition (no counterpart in the reference): apply_quantum_circuit
 * (src/quantum_circuit.h:7, src/quantum_circuit.c:13-35) on complex64 states
 * already in device memory (psi, psi_out: 2^nqubits float2 each, distinct);
 * gates are complex128 host matrices, rounded to complex64 for the passes.
 * Returns 0, or -5 (CUDA) / -6 (invalid argument, host pointers). */
int rqcopt_apply_quantum_circuit_c64(const struct mat4x4 gates[], int ngates, const int wires[], const void* psi,
                                     void* psi_out, int nqubits);

/*
 * Allocation-free gate backward pass.  No counterpart in the reference; it
 * computes what apply_gate_backward (src/gate.h:9-10) computes, without any
 * device allocation, for callers that cannot call cudaMalloc at that point (a
 * process whose device memory belongs to its own pool, a latency-critical
 * thread that must not take the device-wide synchronisation an allocation or
 * free can imply, a host callback such as a target's linear_func that another
 * library's column loop calls on an ordinary host thread while it holds the
 * device memory).  It makes CUDA calls and waits for its stream, so it must not
 * be called from a stream host function (cudaLaunchHostFunc,
 * cudaStreamAddCallback), where CUDA calls are not allowed.
 *
 * Its only scratch (per-tile partial sums of dgate) is a static device array
 * of 2 MiB + 256 B that every GPU loading the library keeps until exit.
 *   - psi, dpsi_out and dpsi must hold managed memory or device memory of the
 *     current device (host buffers would need staging, i.e. allocation; memory
 *     of another GPU is refused); dgate may be host or device memory;
 *   - at most RQCOPT_NOALLOC_MAX_QUBITS qubits; larger states are rejected
 *     with -6 and a message on stderr;
 *   - work is issued on `stream` (a cudaStream_t, NULL for the legacy default
 *     stream) and the call returns after the stream has finished it;
 *   - the first call on a device does the set-up there: it resolves the
 *     scratch address (cudaGetSymbolAddress) with that device current, so
 *     make that first call before any stream capture;
 *   - all calls share the scratch: calls whose GPU work overlaps (other
 *     streams, other host threads) race on it.
 * Returns 0, -5 (CUDA error) or -6 (invalid argument).
 */
#define RQCOPT_NOALLOC_MAX_QUBITS 25
int rqcopt_apply_gate_backward_noalloc(const struct mat4x4* gate, const int i, const int j,
	const struct statevector* psi, const struct statevector* dpsi_out, struct statevector* dpsi,
	struct mat4x4* dgate, void* stream);

#ifdef __cplusplus
}
#endif
