// Exported 4x4 matrix helpers (src/matrix.h:16-70) and distance helpers
// (src/util.h:19-23).  They act on single host matrices, so they run on the
// host through the same __host__ __device__ code (manifold.cuh) that the
// on-device projection and retraction kernels use.
#include <math.h>
#include <string.h>

#include "manifold.cuh"
#include "rqcopt_gpu.h"

using namespace rqc;

namespace {
inline M4 ld(const struct mat4x4* a) { M4 m; memcpy(m.a, a->data, sizeof(m.a)); return m; }
inline void st(const M4& m, struct mat4x4* a) { memcpy(a->data, m.a, sizeof(m.a)); }
}  // namespace

extern "C" {

void zero_matrix(struct mat4x4* a) { memset(a->data, 0, sizeof(a->data)); }

void identity_matrix(struct mat4x4* a)
{
	zero_matrix(a);
	for (int r = 0; r < 4; r++) a->data[5 * r] = 1;
}

void scale_matrix(struct mat4x4* a, const double x)
{
	for (int k = 0; k < 16; k++) a->data[k] *= x;
}

void conjugate_matrix(struct mat4x4* a)
{
	for (int k = 0; k < 16; k++) a->data[k] = std::conj(a->data[k]);
}

void add_matrix(struct mat4x4* a, const struct mat4x4* b)
{
	for (int k = 0; k < 16; k++) a->data[k] += b->data[k];
}

void sub_matrix(struct mat4x4* a, const struct mat4x4* b)
{
	for (int k = 0; k < 16; k++) a->data[k] -= b->data[k];
}

void add_matrices(const struct mat4x4* a, const struct mat4x4* b, struct mat4x4* c)
{
	for (int k = 0; k < 16; k++) c->data[k] = a->data[k] + b->data[k];
}

void sub_matrices(const struct mat4x4* a, const struct mat4x4* b, struct mat4x4* c)
{
	for (int k = 0; k < 16; k++) c->data[k] = a->data[k] - b->data[k];
}

void transpose(const struct mat4x4* a, struct mat4x4* at) { M4 t; m4_transpose(ld(a), t); st(t, at); }
void adjoint(const struct mat4x4* a, struct mat4x4* ah) { M4 t; m4_adjoint(ld(a), t); st(t, ah); }
void symm(const struct mat4x4* w, struct mat4x4* z) { M4 t; m4_symm(ld(w), t); st(t, z); }
void antisymm(const struct mat4x4* w, struct mat4x4* z) { M4 t; m4_antisymm(ld(w), t); st(t, z); }
void real_to_antisymm(const double* r, struct mat4x4* w) { M4 t; m4_real_to_antisymm(r, t); st(t, w); }
void antisymm_to_real(const struct mat4x4* w, double* r) { m4_antisymm_to_real(ld(w), r); }
void real_to_tangent(const double* r, const struct mat4x4* v, struct mat4x4* z) { M4 t; m4_real_to_tangent(r, ld(v), t); st(t, z); }
void tangent_to_real(const struct mat4x4* v, const struct mat4x4* z, double* r) { m4_tangent_to_real(ld(v), ld(z), r); }
void project_tangent(const struct mat4x4* u, const struct mat4x4* z, struct mat4x4* p) { M4 t; m4_project_tangent(ld(u), ld(z), t); st(t, p); }
void multiply_matrices(const struct mat4x4* a, const struct mat4x4* b, struct mat4x4* c) { M4 t; m4_mul(ld(a), ld(b), t); st(t, c); }

void symmetric_triple_matrix_product(const struct mat4x4* a, const struct mat4x4* b, const struct mat4x4* c,
                                     struct mat4x4* ret)
{
	M4 t;
	m4_symmetric_triple(ld(a), ld(b), ld(c), t);
	st(t, ret);
}

int inverse_matrix(const struct mat4x4* a, struct mat4x4* ainv)
{
	M4 t;
	const int r = m4_inverse(ld(a), t);
	if (r == 0) st(t, ainv);
	return r;
}

void polar_factor(const struct mat4x4* a, struct mat4x4* u) { M4 t; m4_polar(ld(a), t); st(t, u); }
void retract(const struct mat4x4* u, const double* eta, struct mat4x4* v) { M4 t; m4_retract(ld(u), eta, t); st(t, v); }

double uniform_distance_real(long n, const double* x, const double* y)
{
	double d = 0;
	for (long i = 0; i < n; i++) d = fmax(d, fabs(x[i] - y[i]));
	return d;
}

double uniform_distance(long n, const numeric* x, const numeric* y)
{
	double d = 0;
	for (long i = 0; i < n; i++) d = fmax(d, std::abs(x[i] - y[i]));
	return d;
}

double relative_distance(long n, const numeric* x, const numeric* y, double eps)
{
	double d = 0;
	for (long i = 0; i < n; i++) d = fmax(d, std::abs(x[i] - y[i]) / fmax(std::abs(x[i]) + std::abs(y[i]), eps));
	return d;
}

}  // extern "C"
