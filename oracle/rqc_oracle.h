/*
 * CPU oracle for the rqcopt_hpc matrix-free circuit-optimisation path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithm (the C sources of cmendl/rqcopt_hpc, src/) used as the checker for the GPU
 * library.  Only the tests, the smoke check and the CPU-baseline leg of the
 * benchmark load it; the product library never links or calls it.
 *
 * Every function states the reference file:line it restates.  Types are
 * layout-identical to the reference's `struct mat4x4` / `struct statevector`
 * (src/matrix.h:10-13, src/statevector.h:11-15): 16 row-major double-complex
 * gate entries, and a 2^nqubits double-complex amplitude vector with qubit 0
 * the most significant index bit.
 */
#pragma once

#include <complex.h>
#include <stdbool.h>
#include <stdint.h>

typedef double complex orc_cplx;

typedef struct { orc_cplx data[16]; } orc_mat4;

typedef struct { orc_cplx* data; int nqubits; } orc_sv;

/* same calling convention as the reference's `linear_func` (src/target.h:7) */
typedef int (*orc_linear_func)(const orc_sv* psi, void* udata, orc_sv* psi_out);

typedef void (*orc_hvp_func)(const double* x, void* fdata, double* vec, double* hvp);
typedef double (*orc_target_func)(const double* x, void* fdata);
typedef double (*orc_target_grad_func)(const double* x, void* fdata, double* grad);
typedef void (*orc_retract_func)(const double* x, const double* eta, void* rdata, double* xs);
typedef double (*orc_target_grad_hess_func)(const double* x, void* fdata, double* grad, double* hess);

typedef struct { int maxiter; double abstol; double reltol; } orc_tcg_params;
typedef struct { orc_tcg_params tcg; double rho_trust, radius_init, maxradius; } orc_rtr_params;

/* ---- 4x4 algebra (src/matrix.c) ---- */
void orc_multiply(const orc_mat4* a, const orc_mat4* b, orc_mat4* c);
void orc_adjoint(const orc_mat4* a, orc_mat4* ah);
void orc_transpose(const orc_mat4* a, orc_mat4* at);
void orc_symm(const orc_mat4* w, orc_mat4* z);
void orc_antisymm(const orc_mat4* w, orc_mat4* z);
void orc_real_to_antisymm(const double* r, orc_mat4* w);
void orc_antisymm_to_real(const orc_mat4* w, double* r);
void orc_real_to_tangent(const double* r, const orc_mat4* v, orc_mat4* z);
void orc_tangent_to_real(const orc_mat4* v, const orc_mat4* z, double* r);
void orc_project_tangent(const orc_mat4* u, const orc_mat4* z, orc_mat4* p);
void orc_symmetric_triple_product(const orc_mat4* a, const orc_mat4* b, const orc_mat4* c, orc_mat4* ret);
int  orc_inverse(const orc_mat4* a, orc_mat4* ainv);
void orc_polar_factor(const orc_mat4* a, orc_mat4* u);
void orc_retract(const orc_mat4* u, const double* eta, orc_mat4* v);

/* ---- gates and circuits (src/gate.c, src/quantum_circuit.c, src/brickwall_circuit.c) ---- */
void orc_add_statevectors(const orc_sv* psi1, const orc_sv* psi2, orc_sv* psi_sum);
void orc_apply_gate(const orc_mat4* g, int i, int j, const orc_sv* psi, orc_sv* out);
void orc_apply_gate_backward(const orc_mat4* g, int i, int j, const orc_sv* psi,
                             const orc_sv* dpsi_out, orc_sv* dpsi, orc_mat4* dg);
int  orc_apply_circuit(const orc_mat4* gates, int ngates, const int* wires, const orc_sv* psi, orc_sv* out);
int  orc_circuit_forward(const orc_mat4* gates, int ngates, const int* wires, const orc_sv* psi,
                         orc_sv* cache /* ngates states */, orc_sv* out);
int  orc_circuit_backward(const orc_mat4* gates, int ngates, const int* wires, const orc_sv* cache,
                          const orc_sv* dpsi_out, orc_sv* dpsi, orc_mat4* dgates);
int  orc_circuit_gates_hvp(const orc_mat4* gates, const orc_mat4* gatedirs, int ngates, const int* wires,
                           const orc_sv* psi, const orc_sv* phi, orc_sv* psi_out,
                           orc_mat4* dgates, orc_mat4* hess_gatedirs);
int  orc_apply_brickwall(const orc_mat4* vlist, int nlayers, const int* perms /* [nlayers][L] */,
                         const orc_sv* psi, orc_sv* out);
int  orc_brickwall_forward(const orc_mat4* vlist, int nlayers, const int* perms, const orc_sv* psi,
                           orc_sv* cache, orc_sv* out);
int  orc_brickwall_backward(const orc_mat4* vlist, int nlayers, const int* perms, const orc_sv* cache,
                            const orc_sv* dpsi_out, orc_sv* dpsi, orc_mat4* dvlist);

/* ---- targets (src/target.c); column range [b_begin, b_end) of the basis-column sum ---- */
int orc_circuit_target(orc_linear_func uf, void* ud, const orc_mat4* gates, int ngates, const int* wires,
                       int nqubits, long b_begin, long b_end, orc_cplx* fval);
int orc_circuit_target_and_gradient(orc_linear_func uf, void* ud, const orc_mat4* gates, int ngates,
                                    const int* wires, int nqubits, long b_begin, long b_end,
                                    orc_cplx* fval, orc_mat4* dgates);
int orc_circuit_target_hvp(orc_linear_func uf, void* ud, const orc_mat4* gates, const orc_mat4* gatedirs,
                           int ngates, const int* wires, int nqubits, long b_begin, long b_end,
                           orc_cplx* fval, orc_mat4* dgates, orc_mat4* hess);
int orc_circuit_target_projected_gradient(orc_linear_func uf, void* ud, const orc_mat4* gates, int ngates,
                                          const int* wires, int nqubits, orc_cplx* fval, double* grad_vec);
int orc_circuit_target_projected_hvp(orc_linear_func uf, void* ud, const orc_mat4* gates, const orc_mat4* gatedirs,
                                     int ngates, const int* wires, int nqubits,
                                     orc_cplx* fval, double* grad_vec, double* hvp_vec);
int orc_brickwall_target(orc_linear_func uf, void* ud, const orc_mat4* vlist, int nlayers, int nqubits,
                         const int* perms, orc_cplx* fval);
int orc_brickwall_target_and_gradient(orc_linear_func uf, void* ud, const orc_mat4* vlist, int nlayers,
                                      int nqubits, const int* perms, orc_cplx* fval, orc_mat4* dvlist);
int orc_brickwall_target_projected_gradient(orc_linear_func uf, void* ud, const orc_mat4* vlist, int nlayers,
                                            int nqubits, const int* perms, orc_cplx* fval, double* grad_vec);
int orc_brickwall_target_hvp(orc_linear_func uf, void* ud, const orc_mat4* vlist, const orc_mat4* vdirs,
                             int nlayers, const int* perms, int nqubits, long b_begin, long b_end,
                             orc_cplx* fval, orc_mat4* dvlist, orc_mat4* hess_vdirs);
int orc_brickwall_target_projected_hvp(orc_linear_func uf, void* ud, const orc_mat4* vlist, const orc_mat4* vdirs,
                                       int nlayers, const int* perms, int nqubits,
                                       orc_cplx* fval, double* grad_vec, double* hvp_vec);

/* ---- trust region (src/trust_region.c) ---- */
bool orc_truncated_cg_hvp(const double* x, const double* grad, orc_hvp_func f_hvp, void* fdata, int n,
                          double radius, const orc_tcg_params* params, double* z);
void orc_rtr_optimize_hvp(orc_target_func f, orc_target_grad_func f_deriv, orc_hvp_func f_hvp, void* fdata,
                          orc_retract_func retract, void* rdata, int n, const double* x_init, int m,
                          const orc_rtr_params* params, int niter, double* f_iter, double* x_final,
                          int* accepted /* niter entries or NULL */, int* on_boundary /* niter or NULL */);
void orc_optimize_brickwall_hvp(orc_linear_func uf, void* ud, const orc_mat4* vstart, int nlayers, int nqubits,
                                const int* perms, const orc_rtr_params* params, int niter,
                                double* f_iter, orc_mat4* vopt, int* accepted, int* on_boundary);
void orc_optimize_circuit_hvp(orc_linear_func uf, void* ud, const orc_mat4* gstart, int ngates, int nqubits,
                              const int* wires, const orc_rtr_params* params, int niter,
                              double* f_iter, orc_mat4* gopt, int* accepted, int* on_boundary);

/* ---- full-Hessian path (src/gate.c:195-460, src/brickwall_circuit.c:134-315,
 *      src/target.c:687-1035, src/trust_region.c:83-141, 230-293, src/brickwall_opt.c:85-186) ----
 * Arrays of ns states are interleaved: amplitude a of state s at data[a*ns + s].
 * Hessians are row-major (16 nlayers)^2, entry ((a*16 + x)*nlayers + b)*16 + y for
 * gate entry x of layer a and gate entry y of layer b. */
void orc_apply_gate_to_array(const orc_mat4* g, int i, int j, int nqubits, int ns, const orc_cplx* psi, orc_cplx* out);
void orc_apply_gate_backward_array(int i, int j, int nqubits, int ns, const orc_cplx* psi, const orc_cplx* dpsi_out,
                                   orc_mat4* dgates);
void orc_apply_gate_placeholder(int i, int j, int nqubits, const orc_cplx* psi, orc_cplx* out /* 16 states */);
int  orc_brickwall_backward_hessian(const orc_mat4* vlist, int nlayers, const int* perms, const orc_sv* cache,
                                    const orc_sv* dpsi_out, orc_sv* dpsi, orc_mat4* dvlist, orc_cplx* hess);
int  orc_apply_brickwall_placeholder(const orc_mat4* vlist, int nlayers, const int* perms, int l, const orc_sv* cache,
                                     orc_cplx* out /* 16 states */);
int  orc_brickwall_target_gradient_hessian(orc_linear_func uf, void* ud, const orc_mat4* vlist, int nlayers,
                                           int nqubits, const int* perms, orc_cplx* fval, orc_mat4* dvlist,
                                           orc_cplx* hess);
int  orc_brickwall_target_gradient_vector_hessian_matrix(orc_linear_func uf, void* ud, const orc_mat4* vlist,
                                                         int nlayers, int nqubits, const int* perms, orc_cplx* fval,
                                                         double* grad_vec, double* H);
bool orc_truncated_cg_hmat(const double* grad, const double* hess, int n, double radius,
                           const orc_tcg_params* params, double* z);
void orc_rtr_optimize_hmat(orc_target_func f, orc_target_grad_hess_func f_deriv_hess, void* fdata,
                           orc_retract_func retract, void* rdata, int n, const double* x_init, int m,
                           const orc_rtr_params* params, int niter, double* f_iter, double* x_final,
                           int* accepted, int* on_boundary);
void orc_optimize_brickwall_hmat(orc_linear_func uf, void* ud, const orc_mat4* vstart, int nlayers, int nqubits,
                                 const int* perms, const orc_rtr_params* params, int niter,
                                 double* f_iter, orc_mat4* vopt, int* accepted, int* on_boundary);

/* ---- sampling estimator (src/rng.c, src/pcg_basic.c, src/statevector.c:102-125,
 *      src/target.c:85-149, 491-505, 807-928, 1050-1088, src/brickwall_opt.c:189-267) ----
 * Layout-identical to the reference's struct pcg32_random / struct rng_state. */
typedef struct { uint64_t state, inc; } orc_pcg32;
typedef struct { orc_pcg32 gen[2]; } orc_rng;
void orc_seed_rng(uint64_t seed, orc_rng* rng);
void orc_haar_statevector(orc_sv* psi, orc_rng* rng);
/* real sample states (one real normal per amplitude), as in the reference's real build */
void orc_set_real_samples(int on);
int  orc_circuit_target_sampling(orc_linear_func uf, void* ud, const orc_mat4* gates, int ngates, const int* wires,
                                 int nqubits, long nsamples, orc_rng* rng, orc_cplx* fval);
int  orc_brickwall_target_sampling(orc_linear_func uf, void* ud, const orc_mat4* vlist, int nlayers, int nqubits,
                                   const int* perms, long nsamples, orc_rng* rng, orc_cplx* fval);
int  orc_brickwall_target_gradient_hessian_sampling(orc_linear_func uf, void* ud, const orc_mat4* vlist, int nlayers,
                                                    int nqubits, const int* perms, long nsamples, orc_rng* rng,
                                                    orc_cplx* fval, orc_mat4* dvlist, orc_cplx* hess);
int  orc_brickwall_target_gradient_vector_hessian_matrix_sampling(orc_linear_func uf, void* ud, const orc_mat4* vlist,
                                                                  int nlayers, int nqubits, const int* perms,
                                                                  long nsamples, orc_rng* rng, orc_cplx* fval,
                                                                  double* grad_vec, double* H);
void orc_optimize_brickwall_hmat_sampling(orc_linear_func uf, void* ud, const orc_mat4* vstart, int nlayers,
                                          int nqubits, const int* perms, long nsamples, orc_rng* rng,
                                          const orc_rtr_params* params, int niter, double* f_iter, orc_mat4* vopt,
                                          int* accepted, int* on_boundary);

/* ---- block-encoding target || P^dag W P - H ||_F^2 / 2 (src/target.c:1100-1720) ----
 * hfunc applies H to states of nqubits / 2 qubits. */
int  orc_blockenc_target(orc_linear_func hf, void* hd, const orc_mat4* vlist, int nlayers, int nqubits,
                         const int* perms, double* fval);
int  orc_blockenc_target_and_gradient(orc_linear_func hf, void* hd, const orc_mat4* vlist, int nlayers, int nqubits,
                                      const int* perms, double* fval, orc_mat4* dvlist);
int  orc_blockenc_target_and_gradient_vector(orc_linear_func hf, void* hd, const orc_mat4* vlist, int nlayers,
                                             int nqubits, const int* perms, double* fval, double* grad_vec);
int  orc_blockenc_target_gradient_hessian(orc_linear_func hf, void* hd, const orc_mat4* vlist, int nlayers,
                                          int nqubits, const int* perms, double* fval, orc_mat4* dvlist,
                                          orc_cplx* hess1, orc_cplx* hess2);
int  orc_blockenc_target_gradient_vector_hessian_matrix(orc_linear_func hf, void* hd, const orc_mat4* vlist,
                                                        int nlayers, int nqubits, const int* perms, double* fval,
                                                        double* grad_vec, double* H);

/* ---- targets used by tests and benchmarks ---- */
/* matrix-free brickwall target U: udata points to orc_brickwall_udata */
typedef struct { const orc_mat4* vlist; int nlayers; const int* perms; } orc_brickwall_udata;
int orc_brickwall_ufunc(const orc_sv* psi, void* udata, orc_sv* psi_out);
/* the synthetic four-term sparse map of the reference tests (test/test_target.c:16-34) */
int orc_fixture_ufunc(const orc_sv* psi, void* udata, orc_sv* psi_out);
/* dense row-major N x N target: udata points to the matrix */
int orc_dense_ufunc(const orc_sv* psi, void* udata, orc_sv* psi_out);
