// 4x4 complex matrix algebra of the unitary manifold, compiled for host and
// device.  One implementation serves the exported matrix helpers (host) and the
// on-device projection / retraction kernels of the optimiser.
//
// Matrices are 16 row-major double2 entries (layout of the reference's
// struct mat4x4, src/matrix.h:10-13).  Tangent vectors at a unitary V are
// represented by 16 reals: r = Re + Im of the anti-Hermitian part of V^H Z
// (src/matrix.c:279-286, 322-329).
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace rqc {

struct M4 { double2 a[16]; };

__host__ __device__ inline double2 c_(double re, double im) { double2 z; z.x = re; z.y = im; return z; }
__host__ __device__ inline double2 c_add(double2 a, double2 b) { return c_(a.x + b.x, a.y + b.y); }
__host__ __device__ inline double2 c_sub(double2 a, double2 b) { return c_(a.x - b.x, a.y - b.y); }
__host__ __device__ inline double2 c_mul(double2 a, double2 b) { return c_(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__host__ __device__ inline double2 c_conj(double2 a) { return c_(a.x, -a.y); }
__host__ __device__ inline double2 c_scale(double2 a, double s) { return c_(a.x * s, a.y * s); }
__host__ __device__ inline double c_abs(double2 a) { return hypot(a.x, a.y); }
__host__ __device__ inline double2 c_div(double2 a, double2 b)
{
	// Smith's algorithm for a / b
	if (fabs(b.x) >= fabs(b.y)) {
		const double r = b.y / b.x, d = b.x + b.y * r;
		return c_((a.x + a.y * r) / d, (a.y - a.x * r) / d);
	}
	const double r = b.x / b.y, d = b.x * r + b.y;
	return c_((a.x * r + a.y) / d, (a.y * r - a.x) / d);
}

// c = a b  (src/matrix.c:354-370)
__host__ __device__ inline void m4_mul(const M4& a, const M4& b, M4& c)
{
	M4 t;
	for (int r = 0; r < 4; r++)
		for (int k = 0; k < 4; k++) {
			double2 s = c_(0, 0);
			for (int m = 0; m < 4; m++) s = c_add(s, c_mul(a.a[4*r + m], b.a[4*m + k]));
			t.a[4*r + k] = s;
		}
	c = t;
}

// src/matrix.c:135-144
__host__ __device__ inline void m4_adjoint(const M4& a, M4& ah)
{
	M4 t;
	for (int r = 0; r < 4; r++)
		for (int c = 0; c < 4; c++) t.a[4*r + c] = c_conj(a.a[4*c + r]);
	ah = t;
}

// src/matrix.c:119-128
__host__ __device__ inline void m4_transpose(const M4& a, M4& at)
{
	M4 t;
	for (int r = 0; r < 4; r++)
		for (int c = 0; c < 4; c++) t.a[4*r + c] = a.a[4*c + r];
	at = t;
}

__host__ __device__ inline void m4_conj(M4& a)
{
	for (int k = 0; k < 16; k++) a.a[k] = c_conj(a.a[k]);
}

// Hermitian part (src/matrix.c:151-174)
__host__ __device__ inline void m4_symm(const M4& w, M4& z)
{
	M4 t;
	for (int r = 0; r < 4; r++) {
		t.a[5*r] = c_(w.a[5*r].x, 0);
		for (int c = r + 1; c < 4; c++) {
			t.a[4*r + c] = c_scale(c_add(w.a[4*r + c], c_conj(w.a[4*c + r])), 0.5);
			t.a[4*c + r] = c_conj(t.a[4*r + c]);
		}
	}
	z = t;
}

// anti-Hermitian part (src/matrix.c:181-211)
__host__ __device__ inline void m4_antisymm(const M4& w, M4& z)
{
	M4 t;
	for (int r = 0; r < 4; r++) {
		t.a[5*r] = c_(0, w.a[5*r].y);
		for (int c = r + 1; c < 4; c++) {
			t.a[4*r + c] = c_scale(c_sub(w.a[4*r + c], c_conj(w.a[4*c + r])), 0.5);
			const double2 u = t.a[4*r + c];
			t.a[4*c + r] = c_(-u.x, u.y);
		}
	}
	z = t;
}

// 16 reals -> anti-Hermitian matrix (src/matrix.c:218-243)
__host__ __device__ inline void m4_real_to_antisymm(const double* x, M4& w)
{
	for (int r = 0; r < 4; r++) {
		w.a[5*r] = c_(0, x[5*r]);
		for (int c = r + 1; c < 4; c++) {
			const double p = x[4*r + c], q = x[4*c + r];
			const double2 u = c_(0.5 * (p - q), 0.5 * (p + q));
			w.a[4*r + c] = u;
			w.a[4*c + r] = c_(-u.x, u.y);
		}
	}
}

// src/matrix.c:279-286
__host__ __device__ inline void m4_antisymm_to_real(const M4& w, double* x)
{
	for (int k = 0; k < 16; k++) x[k] = w.a[k].x + w.a[k].y;
}

// src/matrix.c:309-314
__host__ __device__ inline void m4_real_to_tangent(const double* x, const M4& v, M4& z)
{
	M4 a;
	m4_real_to_antisymm(x, a);
	m4_mul(v, a, z);
}

// src/matrix.c:322-329
__host__ __device__ inline void m4_tangent_to_real(const M4& v, const M4& z, double* x)
{
	M4 vh, t, a;
	m4_adjoint(v, vh);
	m4_mul(vh, z, t);
	m4_antisymm(t, a);
	m4_antisymm_to_real(a, x);
}

// src/matrix.c:336-347
__host__ __device__ inline void m4_project_tangent(const M4& u, const M4& z, M4& p)
{
	M4 uh, w, s;
	m4_adjoint(u, uh);
	m4_mul(uh, z, w);
	m4_symm(w, s);
	m4_mul(u, s, w);
	for (int k = 0; k < 16; k++) p.a[k] = c_sub(z.a[k], w.a[k]);
}

// (a b c + c b a) / 2  (src/matrix.c:376-389)
__host__ __device__ inline void m4_symmetric_triple(const M4& a, const M4& b, const M4& c, M4& ret)
{
	M4 ab, abc, cb, cba;
	m4_mul(a, b, ab);
	m4_mul(ab, c, abc);
	m4_mul(c, b, cb);
	m4_mul(cb, a, cba);
	for (int k = 0; k < 16; k++) ret.a[k] = c_scale(c_add(abc.a[k], cba.a[k]), 0.5);
}

// Gauss-Jordan elimination with partial pivoting; -1 if singular (src/matrix.c:410-475)
__host__ __device__ inline int m4_inverse(const M4& a, M4& ainv)
{
	M4 m = a, v;
	for (int r = 0; r < 4; r++)
		for (int c = 0; c < 4; c++) v.a[4*r + c] = c_(r == c ? 1.0 : 0.0, 0);
	for (int k = 0; k < 4; k++) {
		int piv = k;
		double best = c_abs(m.a[5*k]);
		for (int r = k + 1; r < 4; r++) {
			const double x = c_abs(m.a[4*r + k]);
			if (x > best) { best = x; piv = r; }
		}
		if (best == 0) return -1;
		if (piv != k)
			for (int c = 0; c < 4; c++) {
				double2 t = m.a[4*k + c]; m.a[4*k + c] = m.a[4*piv + c]; m.a[4*piv + c] = t;
				t = v.a[4*k + c]; v.a[4*k + c] = v.a[4*piv + c]; v.a[4*piv + c] = t;
			}
		const double2 d = m.a[5*k];
		for (int r = 0; r < 4; r++) {
			if (r == k) continue;
			const double2 s = c_div(m.a[4*r + k], d);
			for (int c = k + 1; c < 4; c++) m.a[4*r + c] = c_sub(m.a[4*r + c], c_mul(s, m.a[4*k + c]));
			m.a[4*r + k] = c_(0, 0);
			for (int c = 0; c < 4; c++) v.a[4*r + c] = c_sub(v.a[4*r + c], c_mul(s, v.a[4*k + c]));
		}
		for (int c = k + 1; c < 4; c++) m.a[4*k + c] = c_div(m.a[4*k + c], d);
		for (int c = 0; c < 4; c++) v.a[4*k + c] = c_div(v.a[4*k + c], d);
		m.a[5*k] = c_(1, 0);
	}
	ainv = v;
	return 0;
}

// Unitary polar factor by the Newton iteration X <- (X + X^{-H}) / 2, at most 14
// steps, stopping after step 4 once the largest entry change is below 1e-14
// (src/matrix.c:488-510, Higham 1986)
__host__ __device__ inline void m4_polar(const M4& a, M4& u)
{
	M4 x = a;
	for (int k = 0; k < 14; k++) {
		M4 xi, w;
		m4_inverse(x, xi);
		m4_adjoint(xi, w);
		double d = 0;
		for (int e = 0; e < 16; e++) {
			x.a[e] = c_scale(c_add(x.a[e], w.a[e]), 0.5);
			d = fmax(d, c_abs(c_sub(x.a[e], w.a[e])));
		}
		if (k >= 4 && d < 1e-14) break;
	}
	u = x;
}

// V = polar(U (I + A(eta)))  (src/matrix.c:517-531)
__host__ __device__ inline void m4_retract(const M4& u, const double* eta, M4& v)
{
	M4 z, w;
	m4_real_to_antisymm(eta, z);
	for (int r = 0; r < 4; r++) z.a[5*r].x += 1;
	m4_mul(u, z, w);
	m4_polar(w, v);
}

// Projection of gradient and Hessian-vector product of one gate
// (src/target.c:410-430): conj(dG) -> tangent_to_real; conj(HZ) minus
// symmetric_triple(Z, grad^H, G) -> tangent_to_real.
__host__ __device__ inline void m4_project_grad_hvp(const M4& g, const M4* z, M4 dg, M4* hg,
                                                    double* grad_vec, double* hvp_vec)
{
	m4_conj(dg);
	if (grad_vec) m4_tangent_to_real(g, dg, grad_vec);
	if (hg && z && hvp_vec) {
		M4 h = *hg, gradh, pd;
		m4_conj(h);
		m4_adjoint(dg, gradh);
		m4_symmetric_triple(*z, gradh, g, pd);
		for (int k = 0; k < 16; k++) h.a[k] = c_sub(h.a[k], pd.a[k]);
		m4_tangent_to_real(g, h, hvp_vec);
	}
}

}  // namespace rqc
