/*
 * CPU oracle: plain-C restatement of the rqcopt_hpc hot path.
 *
 * TEST INFRASTRUCTURE ONLY -- the checker for the GPU library, loaded by the
 * tests, the smoke check and the CPU-baseline leg of the benchmark.  It is
 * never linked into or called by the product library.
 *
 * Each function cites the reference file:line whose algorithm it restates
 * (paths relative to the cmendl/rqcopt_hpc project root).  The arithmetic is
 * the reference's: double complex, sequential basis-column sums.
 */
#include "rqc_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ utilities */

static orc_cplx* sv_alloc(int L)
{
	return (orc_cplx*)calloc((size_t)1 << L, sizeof(orc_cplx));
}

/* index of amplitude group member (bi, bj) for the rest index r; qubit q is bit L-1-q */
static inline long group_base(long r, int pa, int pb)
{
	/* insert zero bits at positions pa < pb */
	r = ((r >> pa) << (pa + 1)) | (r & ((1L << pa) - 1));
	r = ((r >> pb) << (pb + 1)) | (r & ((1L << pb) - 1));
	return r;
}

static inline void group_indices(long r, int L, int i, int j, long idx[4])
{
	const int pi = L - 1 - i, pj = L - 1 - j;
	const long base = group_base(r, pi < pj ? pi : pj, pi < pj ? pj : pi);
	const long si = 1L << pi, sj = 1L << pj;
	idx[0] = base;
	idx[1] = base + sj;
	idx[2] = base + si;
	idx[3] = base + si + sj;
}

/* ---------------------------------------------------------------- 4x4 algebra */

/* src/matrix.c:354-370 */
void orc_multiply(const orc_mat4* a, const orc_mat4* b, orc_mat4* c)
{
	orc_mat4 t;
	for (int r = 0; r < 4; r++)
		for (int k = 0; k < 4; k++) {
			orc_cplx s = 0;
			for (int m = 0; m < 4; m++) s += a->data[4*r + m] * b->data[4*m + k];
			t.data[4*r + k] = s;
		}
	*c = t;
}

/* src/matrix.c:135-144 */
void orc_adjoint(const orc_mat4* a, orc_mat4* ah)
{
	orc_mat4 t;
	for (int r = 0; r < 4; r++)
		for (int c = 0; c < 4; c++) t.data[4*r + c] = conj(a->data[4*c + r]);
	*ah = t;
}

/* src/matrix.c:119-128 */
void orc_transpose(const orc_mat4* a, orc_mat4* at)
{
	orc_mat4 t;
	for (int r = 0; r < 4; r++)
		for (int c = 0; c < 4; c++) t.data[4*r + c] = a->data[4*c + r];
	*at = t;
}

/* src/matrix.c:151-174 (Hermitian part) */
void orc_symm(const orc_mat4* w, orc_mat4* z)
{
	orc_mat4 t;
	for (int r = 0; r < 4; r++)
		for (int c = 0; c < 4; c++) {
			if (r == c) t.data[5*r] = creal(w->data[5*r]);
			else if (r < c) t.data[4*r + c] = 0.5 * (w->data[4*r + c] + conj(w->data[4*c + r]));
		}
	for (int r = 0; r < 4; r++)
		for (int c = 0; c < r; c++) t.data[4*r + c] = conj(t.data[4*c + r]);
	*z = t;
}

/* src/matrix.c:181-211 (anti-Hermitian part) */
void orc_antisymm(const orc_mat4* w, orc_mat4* z)
{
	orc_mat4 t;
	for (int r = 0; r < 4; r++)
		for (int c = 0; c < 4; c++) {
			if (r == c) t.data[5*r] = I * cimag(w->data[5*r]);
			else if (r < c) t.data[4*r + c] = 0.5 * (w->data[4*r + c] - conj(w->data[4*c + r]));
		}
	for (int r = 0; r < 4; r++)
		for (int c = 0; c < r; c++) t.data[4*r + c] = -conj(t.data[4*c + r]);
	*z = t;
}

/* src/matrix.c:218-243: 16 reals -> anti-Hermitian matrix */
void orc_real_to_antisymm(const double* x, orc_mat4* w)
{
	for (int r = 0; r < 4; r++) {
		w->data[5*r] = I * x[5*r];
		for (int c = r + 1; c < 4; c++) {
			const double p = x[4*r + c], q = x[4*c + r];
			w->data[4*r + c] = 0.5 * (p - q) + 0.5 * I * (p + q);
			w->data[4*c + r] = -conj(w->data[4*r + c]);
		}
	}
}

/* src/matrix.c:279-286 */
void orc_antisymm_to_real(const orc_mat4* w, double* x)
{
	for (int k = 0; k < 16; k++) x[k] = creal(w->data[k]) + cimag(w->data[k]);
}

/* src/matrix.c:309-314 */
void orc_real_to_tangent(const double* x, const orc_mat4* v, orc_mat4* z)
{
	orc_mat4 a;
	orc_real_to_antisymm(x, &a);
	orc_multiply(v, &a, z);
}

/* src/matrix.c:322-329 */
void orc_tangent_to_real(const orc_mat4* v, const orc_mat4* z, double* x)
{
	orc_mat4 vh, t, a;
	orc_adjoint(v, &vh);
	orc_multiply(&vh, z, &t);
	orc_antisymm(&t, &a);
	orc_antisymm_to_real(&a, x);
}

/* src/matrix.c:336-347 */
void orc_project_tangent(const orc_mat4* u, const orc_mat4* z, orc_mat4* p)
{
	orc_mat4 uh, w, s;
	orc_adjoint(u, &uh);
	orc_multiply(&uh, z, &w);
	orc_symm(&w, &s);
	orc_multiply(u, &s, &w);
	for (int k = 0; k < 16; k++) p->data[k] = z->data[k] - w.data[k];
}

/* src/matrix.c:376-389: (a b c + c b a) / 2 */
void orc_symmetric_triple_product(const orc_mat4* a, const orc_mat4* b, const orc_mat4* c, orc_mat4* ret)
{
	orc_mat4 ab, abc, cb, cba;
	orc_multiply(a, b, &ab);
	orc_multiply(&ab, c, &abc);
	orc_multiply(c, b, &cb);
	orc_multiply(&cb, a, &cba);
	for (int k = 0; k < 16; k++) ret->data[k] = 0.5 * (abc.data[k] + cba.data[k]);
}

/* src/matrix.c:410-475: Gauss-Jordan with partial pivoting */
int orc_inverse(const orc_mat4* a, orc_mat4* ainv)
{
	orc_cplx m[4][4], v[4][4];
	for (int r = 0; r < 4; r++)
		for (int c = 0; c < 4; c++) { m[r][c] = a->data[4*r + c]; v[r][c] = (r == c); }
	for (int k = 0; k < 4; k++) {
		int piv = k;
		double best = cabs(m[k][k]);
		for (int r = k + 1; r < 4; r++)
			if (cabs(m[r][k]) > best) { best = cabs(m[r][k]); piv = r; }
		if (best == 0) return -1;
		if (piv != k)
			for (int c = 0; c < 4; c++) {
				orc_cplx t = m[k][c]; m[k][c] = m[piv][c]; m[piv][c] = t;
				t = v[k][c]; v[k][c] = v[piv][c]; v[piv][c] = t;
			}
		for (int r = 0; r < 4; r++) {
			if (r == k) continue;
			const orc_cplx s = m[r][k] / m[k][k];
			for (int c = k + 1; c < 4; c++) m[r][c] -= s * m[k][c];
			m[r][k] = 0;
			for (int c = 0; c < 4; c++) v[r][c] -= s * v[k][c];
		}
		for (int c = k + 1; c < 4; c++) m[k][c] /= m[k][k];
		for (int c = 0; c < 4; c++) v[k][c] /= m[k][k];
		m[k][k] = 1;
	}
	for (int r = 0; r < 4; r++)
		for (int c = 0; c < 4; c++) ainv->data[4*r + c] = v[r][c];
	return 0;
}

/* src/matrix.c:488-510: Newton iteration u <- (u + u^{-H}) / 2, early stop after k >= 4 */
void orc_polar_factor(const orc_mat4* a, orc_mat4* u)
{
	orc_mat4 x = *a;
	for (int k = 0; k < 14; k++) {
		orc_mat4 xi, w;
		orc_inverse(&x, &xi);
		orc_adjoint(&xi, &w);
		double d = 0;
		for (int e = 0; e < 16; e++) {
			x.data[e] = 0.5 * (x.data[e] + w.data[e]);
			const double de = cabs(x.data[e] - w.data[e]);   /* src/util.c:24-33 */
			d = fmax(d, de);
		}
		if (k >= 4 && d < 1e-14) break;
	}
	*u = x;
}

/* src/matrix.c:517-531 */
void orc_retract(const orc_mat4* u, const double* eta, orc_mat4* v)
{
	orc_mat4 z, w;
	orc_real_to_antisymm(eta, &z);
	for (int r = 0; r < 4; r++) z.data[5*r] += 1;
	orc_multiply(u, &z, &w);
	orc_polar_factor(&w, v);
}

/* ------------------------------------------------------------------- statevectors */

/* src/statevector.c:132-142: psi_sum = psi1 + psi2, element by element */
void orc_add_statevectors(const orc_sv* psi1, const orc_sv* psi2, orc_sv* psi_sum)
{
	const long n = 1L << psi1->nqubits;
	for (long k = 0; k < n; k++) psi_sum->data[k] = psi1->data[k] + psi2->data[k];
}

/* ------------------------------------------------------------------- gates */

/* src/gate.c:10-76: psi_out = (gate on wires i, j) psi; row index of the gate is 2*b_i + b_j */
void orc_apply_gate(const orc_mat4* g, int i, int j, const orc_sv* psi, orc_sv* out)
{
	const int L = psi->nqubits;
	const long ngroups = 1L << (L - 2);
	for (long r = 0; r < ngroups; r++) {
		long idx[4];
		group_indices(r, L, i, j, idx);
		orc_cplx x[4];
		for (int c = 0; c < 4; c++) x[c] = psi->data[idx[c]];
		for (int k = 0; k < 4; k++) {
			orc_cplx s = 0;
			for (int c = 0; c < 4; c++) s += g->data[4*k + c] * x[c];
			out->data[idx[k]] = s;
		}
	}
}

/* src/gate.c:83-188: dpsi = gate^T dpsi_out; dgate = sum dpsi_out (x) psi (no conjugation) */
void orc_apply_gate_backward(const orc_mat4* g, int i, int j, const orc_sv* psi,
                             const orc_sv* dpsi_out, orc_sv* dpsi, orc_mat4* dg)
{
	const int L = psi->nqubits;
	const long ngroups = 1L << (L - 2);
	orc_mat4 acc;
	memset(&acc, 0, sizeof(acc));
	for (long r = 0; r < ngroups; r++) {
		long idx[4];
		group_indices(r, L, i, j, idx);
		orc_cplx x[4], d[4];
		for (int c = 0; c < 4; c++) { x[c] = psi->data[idx[c]]; d[c] = dpsi_out->data[idx[c]]; }
		for (int a = 0; a < 4; a++)
			for (int c = 0; c < 4; c++) acc.data[4*a + c] += d[a] * x[c];
		for (int c = 0; c < 4; c++) {
			orc_cplx s = 0;
			for (int a = 0; a < 4; a++) s += g->data[4*a + c] * d[a];
			dpsi->data[idx[c]] = s;
		}
	}
	*dg = acc;
}

/* ---------------------------------------------------------------- circuits */

/* src/quantum_circuit.c:13-35 */
int orc_apply_circuit(const orc_mat4* gates, int ngates, const int* wires, const orc_sv* psi, orc_sv* out)
{
	const int L = psi->nqubits;
	const size_t bytes = ((size_t)1 << L) * sizeof(orc_cplx);
	orc_sv a = { sv_alloc(L), L }, b = { sv_alloc(L), L };
	if (!a.data || !b.data) { free(a.data); free(b.data); return -1; }
	memcpy(a.data, psi->data, bytes);
	for (int k = 0; k < ngates; k++) {
		orc_apply_gate(&gates[k], wires[2*k], wires[2*k + 1], &a, &b);
		orc_cplx* t = a.data; a.data = b.data; b.data = t;
	}
	memcpy(out->data, a.data, bytes);
	free(a.data); free(b.data);
	return 0;
}

/* src/quantum_circuit.c:90-108: cache[k] = state entering gate k */
int orc_circuit_forward(const orc_mat4* gates, int ngates, const int* wires, const orc_sv* psi,
                        orc_sv* cache, orc_sv* out)
{
	const size_t bytes = ((size_t)1 << psi->nqubits) * sizeof(orc_cplx);
	memcpy(cache[0].data, psi->data, bytes);
	for (int k = 0; k < ngates; k++)
		orc_apply_gate(&gates[k], wires[2*k], wires[2*k + 1], &cache[k], k + 1 < ngates ? &cache[k + 1] : out);
	return 0;
}

/* src/quantum_circuit.c:115-140 */
int orc_circuit_backward(const orc_mat4* gates, int ngates, const int* wires, const orc_sv* cache,
                         const orc_sv* dpsi_out, orc_sv* dpsi, orc_mat4* dgates)
{
	const int L = dpsi->nqubits;
	const size_t bytes = ((size_t)1 << L) * sizeof(orc_cplx);
	orc_sv cur = { sv_alloc(L), L }, nxt = { sv_alloc(L), L };
	if (!cur.data || !nxt.data) { free(cur.data); free(nxt.data); return -1; }
	memcpy(cur.data, dpsi_out->data, bytes);
	for (int k = ngates - 1; k >= 0; k--) {
		orc_apply_gate_backward(&gates[k], wires[2*k], wires[2*k + 1], &cache[k], &cur, &nxt, &dgates[k]);
		orc_cplx* t = cur.data; cur.data = nxt.data; nxt.data = t;
	}
	memcpy(dpsi->data, cur.data, bytes);
	free(cur.data); free(nxt.data);
	return 0;
}

/* src/quantum_circuit.c:147-236: forward with cache, reverse pass from phi with cache,
 * then the ascending sweep (tangent of the forward states) and the descending sweep
 * (tangent of the reverse states). */
int orc_circuit_gates_hvp(const orc_mat4* gates, const orc_mat4* gatedirs, int ngates, const int* wires,
                          const orc_sv* psi, const orc_sv* phi, orc_sv* psi_out,
                          orc_mat4* dgates, orc_mat4* hess)
{
	const int L = psi->nqubits;
	const size_t bytes = ((size_t)1 << L) * sizeof(orc_cplx);
	orc_sv* fwd = (orc_sv*)calloc(ngates, sizeof(orc_sv));
	orc_sv* rev = (orc_sv*)calloc(ngates, sizeof(orc_sv));
	orc_sv t1 = { sv_alloc(L), L }, t2 = { sv_alloc(L), L }, d = { sv_alloc(L), L }, sink = { sv_alloc(L), L };
	int fail = !fwd || !rev || !t1.data || !t2.data || !d.data || !sink.data;
	for (int k = 0; k < ngates && !fail; k++) {
		fwd[k].nqubits = rev[k].nqubits = L;
		fwd[k].data = sv_alloc(L);
		rev[k].data = sv_alloc(L);
		fail = !fwd[k].data || !rev[k].data;
	}
	if (!fail) {
		orc_circuit_forward(gates, ngates, wires, psi, fwd, psi_out);
		/* reverse states: rev[k] = adjoint vector at the output of gate k */
		memcpy(rev[ngates - 1].data, phi->data, bytes);
		for (int k = ngates - 1; k >= 0; k--)
			orc_apply_gate_backward(&gates[k], wires[2*k], wires[2*k + 1], &fwd[k], &rev[k],
			                        k > 0 ? &rev[k - 1] : &sink, &dgates[k]);
		/* ascending sweep: d = tangent of the state entering gate k */
		memset(&hess[0], 0, sizeof(orc_mat4));
		orc_apply_gate(&gatedirs[0], wires[0], wires[1], &fwd[0], &d);
		for (int k = 1; k < ngates; k++) {
			orc_mat4 gt, dg;
			orc_transpose(&gates[k], &gt);
			orc_apply_gate_backward(&gt, wires[2*k], wires[2*k + 1], &rev[k], &d, &t1, &dg);
			orc_transpose(&dg, &hess[k]);
			orc_apply_gate(&gatedirs[k], wires[2*k], wires[2*k + 1], &fwd[k], &t2);
			for (long a = 0; a < (1L << L); a++) d.data[a] = t1.data[a] + t2.data[a];
		}
		/* descending sweep: d = tangent of the adjoint vector at the output of gate k */
		{
			orc_mat4 zt;
			orc_transpose(&gatedirs[ngates - 1], &zt);
			orc_apply_gate(&zt, wires[2*ngates - 2], wires[2*ngates - 1], &rev[ngates - 1], &d);
		}
		for (int k = ngates - 2; k >= 0; k--) {
			orc_mat4 dg, zt;
			orc_apply_gate_backward(&gates[k], wires[2*k], wires[2*k + 1], &fwd[k], &d, &t1, &dg);
			for (int e = 0; e < 16; e++) hess[k].data[e] += dg.data[e];
			orc_transpose(&gatedirs[k], &zt);
			orc_apply_gate(&zt, wires[2*k], wires[2*k + 1], &rev[k], &t2);
			for (long a = 0; a < (1L << L); a++) d.data[a] = t1.data[a] + t2.data[a];
		}
	}
	for (int k = 0; k < ngates && fwd && rev; k++) { free(fwd[k].data); free(rev[k].data); }
	free(fwd); free(rev); free(t1.data); free(t2.data); free(d.data); free(sink.data);
	return fail ? -1 : 0;
}

/* brickwall -> sequential gate list (src/target.c:443-458); perms is [nlayers][L] */
static void brickwall_expand(int L, int nlayers, const orc_mat4* vlist, const int* perms,
                             orc_mat4* gates, int* wires)
{
	const int per = L / 2;
	for (int l = 0; l < nlayers; l++)
		for (int p = 0; p < per; p++) {
			if (gates) gates[l*per + p] = vlist[l];
			wires[2*(l*per + p)]     = perms[l*L + 2*p];
			wires[2*(l*per + p) + 1] = perms[l*L + 2*p + 1];
		}
}

/* src/brickwall_circuit.c:14-43 */
int orc_apply_brickwall(const orc_mat4* vlist, int nlayers, const int* perms, const orc_sv* psi, orc_sv* out)
{
	const int L = psi->nqubits, G = nlayers * (L / 2);
	orc_mat4* gates = (orc_mat4*)malloc(G * sizeof(orc_mat4));
	int* wires = (int*)malloc(2 * G * sizeof(int));
	brickwall_expand(L, nlayers, vlist, perms, gates, wires);
	int ret = orc_apply_circuit(gates, G, wires, psi, out);
	free(gates); free(wires);
	return ret;
}

/* src/brickwall_circuit.c:51-77 */
int orc_brickwall_forward(const orc_mat4* vlist, int nlayers, const int* perms, const orc_sv* psi,
                          orc_sv* cache, orc_sv* out)
{
	const int L = psi->nqubits, G = nlayers * (L / 2);
	orc_mat4* gates = (orc_mat4*)malloc(G * sizeof(orc_mat4));
	int* wires = (int*)malloc(2 * G * sizeof(int));
	brickwall_expand(L, nlayers, vlist, perms, gates, wires);
	int ret = orc_circuit_forward(gates, G, wires, psi, cache, out);
	free(gates); free(wires);
	return ret;
}

/* src/brickwall_circuit.c:85-124: per-layer gradient = sum over the layer's gate copies */
int orc_brickwall_backward(const orc_mat4* vlist, int nlayers, const int* perms, const orc_sv* cache,
                           const orc_sv* dpsi_out, orc_sv* dpsi, orc_mat4* dvlist)
{
	const int L = dpsi->nqubits, per = L / 2, G = nlayers * per;
	orc_mat4* gates = (orc_mat4*)malloc(G * sizeof(orc_mat4));
	orc_mat4* dg = (orc_mat4*)malloc(G * sizeof(orc_mat4));
	int* wires = (int*)malloc(2 * G * sizeof(int));
	brickwall_expand(L, nlayers, vlist, perms, gates, wires);
	int ret = orc_circuit_backward(gates, G, wires, cache, dpsi_out, dpsi, dg);
	for (int l = 0; l < nlayers; l++) {
		memset(&dvlist[l], 0, sizeof(orc_mat4));
		for (int p = per - 1; p >= 0; p--)
			for (int e = 0; e < 16; e++) dvlist[l].data[e] += dg[l*per + p].data[e];
	}
	free(gates); free(dg); free(wires);
	return ret;
}

/* ------------------------------------------------------------------ targets */

/* one basis column of -conj(U): src/target.c:41-53 */
static int target_column(orc_linear_func uf, void* ud, long b, orc_sv* e, orc_sv* u)
{
	const long n = 1L << e->nqubits;
	memset(e->data, 0, n * sizeof(orc_cplx));
	e->data[b] = 1;
	int ret = uf(e, ud, u);
	if (ret < 0) return -2;
	for (long a = 0; a < n; a++) u->data[a] = -conj(u->data[a]);
	return 0;
}

/* src/target.c:15-75 */
int orc_circuit_target(orc_linear_func uf, void* ud, const orc_mat4* gates, int ngates, const int* wires,
                       int L, long b_begin, long b_end, orc_cplx* fval)
{
	const long n = 1L << L;
	orc_sv e = { sv_alloc(L), L }, u = { sv_alloc(L), L }, c = { sv_alloc(L), L };
	orc_cplx f = 0;
	int ret = 0;
	for (long b = b_begin; b < b_end && ret == 0; b++) {
		ret = target_column(uf, ud, b, &e, &u);
		if (ret) break;
		e.data[b] = 1;
		orc_apply_circuit(gates, ngates, wires, &e, &c);
		for (long a = 0; a < n; a++) f += u.data[a] * c.data[a];
	}
	free(e.data); free(u.data); free(c.data);
	*fval = f;
	return ret;
}

/* src/target.c:158-247 */
int orc_circuit_target_and_gradient(orc_linear_func uf, void* ud, const orc_mat4* gates, int ngates,
                                    const int* wires, int L, long b_begin, long b_end,
                                    orc_cplx* fval, orc_mat4* dgates)
{
	const long n = 1L << L;
	orc_sv e = { sv_alloc(L), L }, u = { sv_alloc(L), L }, c = { sv_alloc(L), L };
	orc_sv* cache = (orc_sv*)calloc(ngates, sizeof(orc_sv));
	orc_mat4* dg = (orc_mat4*)malloc(ngates * sizeof(orc_mat4));
	for (int k = 0; k < ngates; k++) { cache[k].nqubits = L; cache[k].data = sv_alloc(L); }
	memset(dgates, 0, ngates * sizeof(orc_mat4));
	orc_cplx f = 0;
	int ret = 0;
	for (long b = b_begin; b < b_end; b++) {
		ret = target_column(uf, ud, b, &e, &u);
		if (ret) break;
		e.data[b] = 1;
		orc_circuit_forward(gates, ngates, wires, &e, cache, &c);
		for (long a = 0; a < n; a++) f += u.data[a] * c.data[a];
		orc_circuit_backward(gates, ngates, wires, cache, &u, &e, dg);
		for (int k = 0; k < ngates; k++)
			for (int x = 0; x < 16; x++) dgates[k].data[x] += dg[k].data[x];
	}
	for (int k = 0; k < ngates; k++) free(cache[k].data);
	free(cache); free(dg); free(e.data); free(u.data); free(c.data);
	*fval = f;
	return ret;
}

/* src/target.c:289-380 */
int orc_circuit_target_hvp(orc_linear_func uf, void* ud, const orc_mat4* gates, const orc_mat4* gatedirs,
                           int ngates, const int* wires, int L, long b_begin, long b_end,
                           orc_cplx* fval, orc_mat4* dgates, orc_mat4* hess)
{
	const long n = 1L << L;
	orc_sv e = { sv_alloc(L), L }, u = { sv_alloc(L), L }, c = { sv_alloc(L), L };
	orc_mat4* dg = (orc_mat4*)malloc(ngates * sizeof(orc_mat4));
	orc_mat4* hg = (orc_mat4*)malloc(ngates * sizeof(orc_mat4));
	memset(dgates, 0, ngates * sizeof(orc_mat4));
	memset(hess, 0, ngates * sizeof(orc_mat4));
	orc_cplx f = 0;
	int ret = 0;
	for (long b = b_begin; b < b_end; b++) {
		ret = target_column(uf, ud, b, &e, &u);
		if (ret) break;
		e.data[b] = 1;
		if (orc_circuit_gates_hvp(gates, gatedirs, ngates, wires, &e, &u, &c, dg, hg) < 0) { ret = -3; break; }
		for (long a = 0; a < n; a++) f += u.data[a] * c.data[a];
		for (int k = 0; k < ngates; k++)
			for (int x = 0; x < 16; x++) { dgates[k].data[x] += dg[k].data[x]; hess[k].data[x] += hg[k].data[x]; }
	}
	free(dg); free(hg); free(e.data); free(u.data); free(c.data);
	*fval = f;
	return ret;
}

/* src/target.c:256-280 */
int orc_circuit_target_projected_gradient(orc_linear_func uf, void* ud, const orc_mat4* gates, int ngates,
                                          const int* wires, int L, orc_cplx* fval, double* grad_vec)
{
	orc_mat4* dg = (orc_mat4*)malloc(ngates * sizeof(orc_mat4));
	int ret = orc_circuit_target_and_gradient(uf, ud, gates, ngates, wires, L, 0, 1L << L, fval, dg);
	for (int k = 0; k < ngates && ret == 0; k++) {
		for (int x = 0; x < 16; x++) dg[k].data[x] = conj(dg[k].data[x]);
		orc_tangent_to_real(&gates[k], &dg[k], &grad_vec[16*k]);
	}
	free(dg);
	return ret;
}

/* projection of gradient and HVP for one gate: src/target.c:410-430 */
static void project_grad_hvp(const orc_mat4* g, const orc_mat4* z, orc_mat4* dg, orc_mat4* hg,
                             double* grad_vec, double* hvp_vec)
{
	for (int x = 0; x < 16; x++) { dg->data[x] = conj(dg->data[x]); hg->data[x] = conj(hg->data[x]); }
	orc_tangent_to_real(g, dg, grad_vec);
	orc_mat4 gradh, pd;
	orc_adjoint(dg, &gradh);
	orc_symmetric_triple_product(z, &gradh, g, &pd);
	for (int x = 0; x < 16; x++) hg->data[x] -= pd.data[x];
	orc_tangent_to_real(g, hg, hvp_vec);
}

/* src/target.c:389-436 */
int orc_circuit_target_projected_hvp(orc_linear_func uf, void* ud, const orc_mat4* gates, const orc_mat4* gatedirs,
                                     int ngates, const int* wires, int L,
                                     orc_cplx* fval, double* grad_vec, double* hvp_vec)
{
	orc_mat4* dg = (orc_mat4*)malloc(ngates * sizeof(orc_mat4));
	orc_mat4* hg = (orc_mat4*)malloc(ngates * sizeof(orc_mat4));
	int ret = orc_circuit_target_hvp(uf, ud, gates, gatedirs, ngates, wires, L, 0, 1L << L, fval, dg, hg);
	for (int k = 0; k < ngates && ret == 0; k++)
		project_grad_hvp(&gates[k], &gatedirs[k], &dg[k], &hg[k], &grad_vec[16*k], &hvp_vec[16*k]);
	free(dg); free(hg);
	return ret < 0 ? -2 : 0;
}

/* src/target.c:467-481 */
int orc_brickwall_target(orc_linear_func uf, void* ud, const orc_mat4* vlist, int nlayers, int L,
                         const int* perms, orc_cplx* fval)
{
	const int G = nlayers * (L / 2);
	orc_mat4* gates = (orc_mat4*)malloc(G * sizeof(orc_mat4));
	int* wires = (int*)malloc(2 * G * sizeof(int));
	brickwall_expand(L, nlayers, vlist, perms, gates, wires);
	int ret = orc_circuit_target(uf, ud, gates, G, wires, L, 0, 1L << L, fval);
	free(gates); free(wires);
	return ret;
}

/* src/target.c:514-542 */
int orc_brickwall_target_and_gradient(orc_linear_func uf, void* ud, const orc_mat4* vlist, int nlayers,
                                      int L, const int* perms, orc_cplx* fval, orc_mat4* dvlist)
{
	const int per = L / 2, G = nlayers * per;
	orc_mat4* gates = (orc_mat4*)malloc(G * sizeof(orc_mat4));
	orc_mat4* dg = (orc_mat4*)malloc(G * sizeof(orc_mat4));
	int* wires = (int*)malloc(2 * G * sizeof(int));
	brickwall_expand(L, nlayers, vlist, perms, gates, wires);
	int ret = orc_circuit_target_and_gradient(uf, ud, gates, G, wires, L, 0, 1L << L, fval, dg);
	for (int l = 0; l < nlayers; l++) {
		memset(&dvlist[l], 0, sizeof(orc_mat4));
		for (int p = 0; p < per; p++)
			for (int x = 0; x < 16; x++) dvlist[l].data[x] += dg[l*per + p].data[x];
	}
	free(gates); free(dg); free(wires);
	return ret;
}

/* src/target.c:551-575 */
int orc_brickwall_target_projected_gradient(orc_linear_func uf, void* ud, const orc_mat4* vlist, int nlayers,
                                            int L, const int* perms, orc_cplx* fval, double* grad_vec)
{
	orc_mat4* dv = (orc_mat4*)malloc(nlayers * sizeof(orc_mat4));
	int ret = orc_brickwall_target_and_gradient(uf, ud, vlist, nlayers, L, perms, fval, dv);
	for (int l = 0; l < nlayers && ret == 0; l++) {
		for (int x = 0; x < 16; x++) dv[l].data[x] = conj(dv[l].data[x]);
		orc_tangent_to_real(&vlist[l], &dv[l], &grad_vec[16*l]);
	}
	free(dv);
	return ret;
}

/* src/target.c:584-622 */
int orc_brickwall_target_hvp(orc_linear_func uf, void* ud, const orc_mat4* vlist, const orc_mat4* vdirs,
                             int nlayers, const int* perms, int L, long b_begin, long b_end,
                             orc_cplx* fval, orc_mat4* dvlist, orc_mat4* hess_vdirs)
{
	const int per = L / 2, G = nlayers * per;
	orc_mat4* gates = (orc_mat4*)malloc(G * sizeof(orc_mat4));
	orc_mat4* dirs = (orc_mat4*)malloc(G * sizeof(orc_mat4));
	orc_mat4* dg = (orc_mat4*)malloc(G * sizeof(orc_mat4));
	orc_mat4* hg = (orc_mat4*)malloc(G * sizeof(orc_mat4));
	int* wires = (int*)malloc(2 * G * sizeof(int));
	brickwall_expand(L, nlayers, vlist, perms, gates, wires);
	brickwall_expand(L, nlayers, vdirs, perms, dirs, wires);
	int ret = orc_circuit_target_hvp(uf, ud, gates, dirs, G, wires, L, b_begin, b_end, fval, dg, hg);
	for (int l = 0; l < nlayers; l++) {
		memset(&dvlist[l], 0, sizeof(orc_mat4));
		memset(&hess_vdirs[l], 0, sizeof(orc_mat4));
		for (int p = 0; p < per; p++)
			for (int x = 0; x < 16; x++) {
				dvlist[l].data[x] += dg[l*per + p].data[x];
				hess_vdirs[l].data[x] += hg[l*per + p].data[x];
			}
	}
	free(gates); free(dirs); free(dg); free(hg); free(wires);
	return ret;
}

/* src/target.c:631-678 */
int orc_brickwall_target_projected_hvp(orc_linear_func uf, void* ud, const orc_mat4* vlist, const orc_mat4* vdirs,
                                       int nlayers, const int* perms, int L,
                                       orc_cplx* fval, double* grad_vec, double* hvp_vec)
{
	orc_mat4* dv = (orc_mat4*)malloc(nlayers * sizeof(orc_mat4));
	orc_mat4* hv = (orc_mat4*)malloc(nlayers * sizeof(orc_mat4));
	int ret = orc_brickwall_target_hvp(uf, ud, vlist, vdirs, nlayers, perms, L, 0, 1L << L, fval, dv, hv);
	for (int l = 0; l < nlayers && ret == 0; l++)
		project_grad_hvp(&vlist[l], &vdirs[l], &dv[l], &hv[l], &grad_vec[16*l], &hvp_vec[16*l]);
	free(dv); free(hv);
	return ret < 0 ? -2 : 0;
}

/* ------------------------------------------------------------- trust region */

static double dot(int n, const double* a, const double* b)
{
	double s = 0;
	for (int k = 0; k < n; k++) s += a[k] * b[k];
	return s;
}

/* src/trust_region.c:14-40: roots of x^2 + 2 p x + q */
static void quadratic_roots(double p, double q, double x[2])
{
	if (p == 0) { const double a = sqrt(-q); x[0] = -a; x[1] = a; return; }
	const double a = -(p + copysign(1.0, p) * sqrt(p * p - q));
	const double b = q / a;
	if (a <= b) { x[0] = a; x[1] = b; } else { x[0] = b; x[1] = a; }
}

/* src/trust_region.c:49-65: positive t with ||b + t d|| = radius */
static double to_boundary(const double* b, const double* d, int n, double radius)
{
	const double dsq = dot(n, d, d);
	if (dsq == 0) return 0;
	const double p = dot(n, b, d) / dsq;
	const double q = (dot(n, b, b) - radius * radius) / dsq;
	double t[2];
	quadratic_roots(p, q, t);
	return t[1];
}

/* src/trust_region.c:159-217 (Steihaug-Toint truncated CG) */
bool orc_truncated_cg_hvp(const double* x, const double* grad, orc_hvp_func f_hvp, void* fdata, int n,
                          double radius, const orc_tcg_params* params, double* z)
{
	double* r = (double*)malloc(n * sizeof(double));
	double* d = (double*)malloc(n * sizeof(double));
	double* hd = (double*)malloc(n * sizeof(double));
	memcpy(r, grad, n * sizeof(double));
	double rsq = dot(n, r, r);
	const double stoptol = fmax(params->abstol, params->reltol * sqrt(rsq));
	memset(z, 0, n * sizeof(double));
	for (int k = 0; k < n; k++) d[k] = -r[k];
	bool boundary = false;
	for (int it = 0; it < params->maxiter; it++) {
		f_hvp(x, fdata, d, hd);
		const double dhd = dot(n, d, hd);
		const double t = to_boundary(z, d, n, radius);
		const double alpha = rsq / dhd;
		if (dhd <= 0 || alpha > t) {
			for (int k = 0; k < n; k++) z[k] += t * d[k];
			boundary = true;
			break;
		}
		for (int k = 0; k < n; k++) r[k] += alpha * hd[k];
		for (int k = 0; k < n; k++) z[k] += alpha * d[k];
		const double rsq_next = dot(n, r, r);
		if (sqrt(rsq_next) <= stoptol) break;
		const double beta = rsq_next / rsq;
		for (int k = 0; k < n; k++) d[k] = beta * d[k] - r[k];
		rsq = rsq_next;
	}
	free(r); free(d); free(hd);
	return boundary;
}

/* src/trust_region.c:306-368 (Riemannian trust region, Absil et al. Algorithm 10) */
void orc_rtr_optimize_hvp(orc_target_func f, orc_target_grad_func f_deriv, orc_hvp_func f_hvp, void* fdata,
                          orc_retract_func retract, void* rdata, int n, const double* x_init, int m,
                          const orc_rtr_params* params, int niter, double* f_iter, double* x_final,
                          int* accepted, int* on_boundary)
{
	double* x = (double*)malloc(m * sizeof(double));
	double* xn = (double*)malloc(m * sizeof(double));
	double* grad = (double*)malloc(n * sizeof(double));
	double* eta = (double*)malloc(n * sizeof(double));
	double* heta = (double*)malloc(n * sizeof(double));
	memcpy(x, x_init, m * sizeof(double));
	double radius = params->radius_init;
	for (int k = 0; k < niter; k++) {
		const double fx = f_deriv(x, fdata, grad);
		const bool bnd = orc_truncated_cg_hvp(x, grad, f_hvp, fdata, n, radius, &params->tcg, eta);
		retract(x, eta, rdata, xn);
		f_iter[k] = fx;
		f_hvp(x, fdata, eta, heta);
		const double rho = (f(xn, fdata) - fx) / (dot(n, grad, eta) + 0.5 * dot(n, eta, heta));
		if (rho < 0.25) radius *= 0.25;
		else if (rho > 0.75 && bnd) radius = fmin(2 * radius, params->maxradius);
		const int acc = rho > params->rho_trust;
		if (acc) { double* t = x; x = xn; xn = t; }
		if (accepted) accepted[k] = acc;
		if (on_boundary) on_boundary[k] = bnd;
	}
	memcpy(x_final, x, m * sizeof(double));
	f_iter[niter] = f(x_final, fdata);
	free(x); free(xn); free(grad); free(eta); free(heta);
}

/* ---------------------------------------------------------- optimiser glue */

typedef struct {
	orc_linear_func uf; void* ud; const int* perms_or_wires; int ngates_or_layers; int L; int brickwall;
} glue;

/* src/brickwall_opt.c:22-33, src/circuit_opt.c:22-33 */
static double glue_f(const double* x, void* fd)
{
	const glue* g = (const glue*)fd;
	orc_cplx f;
	int ret = g->brickwall
		? orc_brickwall_target(g->uf, g->ud, (const orc_mat4*)x, g->ngates_or_layers, g->L, g->perms_or_wires, &f)
		: orc_circuit_target(g->uf, g->ud, (const orc_mat4*)x, g->ngates_or_layers, g->perms_or_wires, g->L, 0, 1L << g->L, &f);
	return ret < 0 ? -1 : creal(f);
}

/* src/brickwall_opt.c:40-51, src/circuit_opt.c:40-51 */
static double glue_fd(const double* x, void* fd, double* grad)
{
	const glue* g = (const glue*)fd;
	orc_cplx f;
	int ret = g->brickwall
		? orc_brickwall_target_projected_gradient(g->uf, g->ud, (const orc_mat4*)x, g->ngates_or_layers, g->L, g->perms_or_wires, &f, grad)
		: orc_circuit_target_projected_gradient(g->uf, g->ud, (const orc_mat4*)x, g->ngates_or_layers, g->perms_or_wires, g->L, &f, grad);
	return ret < 0 ? -1 : creal(f);
}

/* src/brickwall_opt.c:58-78, src/circuit_opt.c:58-78 */
static void glue_hvp(const double* x, void* fd, double* vec, double* hvp)
{
	const glue* g = (const glue*)fd;
	const int k = g->ngates_or_layers;
	const orc_mat4* v = (const orc_mat4*)x;
	orc_mat4* dirs = (orc_mat4*)malloc(k * sizeof(orc_mat4));
	double* gv = (double*)malloc(16 * k * sizeof(double));
	for (int i = 0; i < k; i++) orc_real_to_tangent(&vec[16*i], &v[i], &dirs[i]);
	orc_cplx f;
	if (g->brickwall)
		orc_brickwall_target_projected_hvp(g->uf, g->ud, v, dirs, k, g->perms_or_wires, g->L, &f, gv, hvp);
	else
		orc_circuit_target_projected_hvp(g->uf, g->ud, v, dirs, k, g->perms_or_wires, g->L, &f, gv, hvp);
	free(dirs); free(gv);
}

/* src/brickwall_opt.c:107-119 */
static void glue_retract(const double* x, const double* eta, void* rdata, double* xs)
{
	const int k = *(const int*)rdata;
	for (int i = 0; i < k; i++) orc_retract(&((const orc_mat4*)x)[i], &eta[16*i], &((orc_mat4*)xs)[i]);
}

/* src/brickwall_opt.c:127-149 */
void orc_optimize_brickwall_hvp(orc_linear_func uf, void* ud, const orc_mat4* vstart, int nlayers, int L,
                                const int* perms, const orc_rtr_params* params, int niter,
                                double* f_iter, orc_mat4* vopt, int* accepted, int* on_boundary)
{
	glue g = { uf, ud, perms, nlayers, L, 1 };
	int k = nlayers;
	orc_rtr_optimize_hvp(glue_f, glue_fd, glue_hvp, &g, glue_retract, &k, 16 * nlayers,
	                     (const double*)vstart, 32 * nlayers, params, niter, f_iter, (double*)vopt,
	                     accepted, on_boundary);
}

/* src/circuit_opt.c:104-124 */
void orc_optimize_circuit_hvp(orc_linear_func uf, void* ud, const orc_mat4* gstart, int ngates, int L,
                              const int* wires, const orc_rtr_params* params, int niter,
                              double* f_iter, orc_mat4* gopt, int* accepted, int* on_boundary)
{
	glue g = { uf, ud, wires, ngates, L, 0 };
	int k = ngates;
	orc_rtr_optimize_hvp(glue_f, glue_fd, glue_hvp, &g, glue_retract, &k, 16 * ngates,
	                     (const double*)gstart, 32 * ngates, params, niter, f_iter, (double*)gopt,
	                     accepted, on_boundary);
}

/* ------------------------------------------------------------ target maps */

int orc_brickwall_ufunc(const orc_sv* psi, void* udata, orc_sv* psi_out)
{
	const orc_brickwall_udata* t = (const orc_brickwall_udata*)udata;
	return orc_apply_brickwall(t->vlist, t->nlayers, t->perms, psi, psi_out);
}

/* test/test_target.c:16-34 */
int orc_fixture_ufunc(const orc_sv* psi, void* udata, orc_sv* psi_out)
{
	(void)udata;
	const long n = 1L << psi->nqubits;
	for (long i = 0; i < n; i++)
		psi_out->data[i] = (-1.1 + 0.8*I) * psi->data[((i + 3) * 113) % n]
		                 + ( 0.4 - 0.7*I) * psi->data[((i + 9) * 173) % n]
		                 + ( 0.5 + 0.1*I) * psi->data[i]
		                 + (-0.3 + 0.2*I) * psi->data[((i + 4) * 199) % n];
	return 0;
}

int orc_dense_ufunc(const orc_sv* psi, void* udata, orc_sv* psi_out)
{
	const orc_cplx* u = (const orc_cplx*)udata;
	const long n = 1L << psi->nqubits;
	for (long r = 0; r < n; r++) {
		orc_cplx s = 0;
		for (long c = 0; c < n; c++) s += u[r*n + c] * psi->data[c];
		psi_out->data[r] = s;
	}
	return 0;
}

/* ------------------------------------------------------------ full-Hessian path */

/* src/gate.c:195-262: the gate on wires (i, j) of each of the ns states of an
 * interleaved array, amplitude a of state s at data[a*ns + s] */
void orc_apply_gate_to_array(const orc_mat4* g, int i, int j, int L, int ns, const orc_cplx* psi, orc_cplx* out)
{
	const long ngroups = 1L << (L - 2);
	for (long r = 0; r < ngroups; r++) {
		long idx[4];
		group_indices(r, L, i, j, idx);
		for (int s = 0; s < ns; s++) {
			orc_cplx x[4];
			for (int c = 0; c < 4; c++) x[c] = psi[idx[c]*ns + s];
			for (int k = 0; k < 4; k++) {
				orc_cplx acc = 0;
				for (int c = 0; c < 4; c++) acc += g->data[4*k + c] * x[c];
				out[idx[k]*ns + s] = acc;
			}
		}
	}
}

/* src/gate.c:269-377: dgates[s] = sum over groups of dpsi_out (x) psi_s (no conjugation) */
void orc_apply_gate_backward_array(int i, int j, int L, int ns, const orc_cplx* psi, const orc_cplx* dpsi_out,
                                   orc_mat4* dgates)
{
	const long ngroups = 1L << (L - 2);
	memset(dgates, 0, ns * sizeof(orc_mat4));
	for (long r = 0; r < ngroups; r++) {
		long idx[4];
		group_indices(r, L, i, j, idx);
		orc_cplx d[4];
		for (int c = 0; c < 4; c++) d[c] = dpsi_out[idx[c]];
		for (int s = 0; s < ns; s++)
			for (int a = 0; a < 4; a++)
				for (int c = 0; c < 4; c++) dgates[s].data[4*a + c] += d[a] * psi[idx[c]*ns + s];
	}
}

/* src/gate.c:386-460: 16 states, state e = 4 r + c is E_rc psi (the unit gate with
 * entry (r, c)): at group member r it holds psi's member c, zero elsewhere */
void orc_apply_gate_placeholder(int i, int j, int L, const orc_cplx* psi, orc_cplx* out)
{
	const long ngroups = 1L << (L - 2);
	memset(out, 0, ((size_t)16 << L) * sizeof(orc_cplx));
	for (long r = 0; r < ngroups; r++) {
		long idx[4];
		group_indices(r, L, i, j, idx);
		for (int row = 0; row < 4; row++)
			for (int c = 0; c < 4; c++) out[idx[row]*16 + 4*row + c] = psi[idx[c]];
	}
}

/* flat row-major (m x m) index of Hessian entry (layer a, entry x), (layer b, entry y) */
static inline long hidx(int nlayers, int a, int x, int b, int y)
{
	return ((long)(a*16 + x)*nlayers + b)*16 + y;
}

/* src/brickwall_circuit.c:134-255.  cache[k] is the input state of sequential gate
 * k (layer-major order); returns dpsi, the per-layer gradients and the symmetric
 * (16 nlayers)^2 complex Hessian of psi_out . dpsi_out in the gate entries. */
int orc_brickwall_backward_hessian(const orc_mat4* vlist, int nlayers, const int* perms, const orc_sv* cache,
                                   const orc_sv* dpsi_out, orc_sv* dpsi, orc_mat4* dvlist, orc_cplx* hess)
{
	const int L = dpsi->nqubits, per = L / 2, G = nlayers * per, m = 16 * nlayers;
	const long N = 1L << L;
	int* wires = (int*)malloc(2 * G * sizeof(int));
	brickwall_expand(L, nlayers, NULL, perms, NULL, wires);
	/* adjoint states at each gate output: phi[k] for gate k */
	orc_cplx* phi = (orc_cplx*)malloc((size_t)G * N * sizeof(orc_cplx));
	memcpy(phi + (size_t)(G - 1) * N, dpsi_out->data, N * sizeof(orc_cplx));
	for (int l = 0; l < nlayers; l++) memset(&dvlist[l], 0, sizeof(orc_mat4));
	for (int k = G - 1; k >= 0; k--) {
		orc_sv in = { phi + (size_t)k * N, L };
		orc_sv o = { k > 0 ? phi + (size_t)(k - 1) * N : dpsi->data, L };
		orc_mat4 dv;
		orc_apply_gate_backward(&vlist[k / per], wires[2*k], wires[2*k + 1], &cache[k], &in, &o, &dv);
		for (int e = 0; e < 16; e++) dvlist[k / per].data[e] += dv.data[e];
	}
	memset(hess, 0, (size_t)m * m * sizeof(orc_cplx));
	orc_cplx* t[2];
	t[0] = (orc_cplx*)malloc((size_t)16 * N * sizeof(orc_cplx));
	t[1] = (orc_cplx*)malloc((size_t)16 * N * sizeof(orc_cplx));
	orc_mat4 h[16];
	for (int k = 0; k < G; k++) {
		const int a = k / per;
		orc_apply_gate_placeholder(wires[2*k], wires[2*k + 1], L, cache[k].data, t[0]);
		int cur = 0;
		for (int q = k + 1; q < G; q++) {
			const int b = q / per;
			orc_apply_gate_backward_array(wires[2*q], wires[2*q + 1], L, 16, t[cur], phi + (size_t)q * N, h);
			for (int x = 0; x < 16; x++)
				for (int y = 0; y < 16; y++) hess[hidx(nlayers, a, x, b, y)] += h[x].data[y];
			if (q < G - 1) {
				orc_apply_gate_to_array(&vlist[b], wires[2*q], wires[2*q + 1], L, 16, t[cur], t[1 - cur]);
				cur = 1 - cur;
			}
		}
	}
	/* diagonal blocks: both orders of a pair of gates of the same layer */
	for (int a = 0; a < nlayers; a++)
		for (int x = 0; x < 16; x++)
			for (int y = 0; y <= x; y++) {
				const orc_cplx s = hess[hidx(nlayers, a, x, a, y)] + hess[hidx(nlayers, a, y, a, x)];
				hess[hidx(nlayers, a, x, a, y)] = s;
				hess[hidx(nlayers, a, y, a, x)] = s;
			}
	/* blocks below the diagonal from the ones above */
	for (int a = 0; a < nlayers; a++)
		for (int b = 0; b < a; b++)
			for (int x = 0; x < 16; x++)
				for (int y = 0; y < 16; y++) hess[hidx(nlayers, a, x, b, y)] = hess[hidx(nlayers, b, y, a, x)];
	free(t[0]); free(t[1]); free(phi); free(wires);
	return 0;
}

/* src/brickwall_circuit.c:264-315: sum over the gate positions s of layer l of the
 * circuit with the gate at (l, s) replaced by the 16 unit placeholders */
int orc_apply_brickwall_placeholder(const orc_mat4* vlist, int nlayers, const int* perms, int l, const orc_sv* cache,
                                    orc_cplx* out)
{
	const int L = cache[0].nqubits, per = L / 2, G = nlayers * per;
	const long N = 1L << L;
	if (l < 0 || l >= nlayers) return -1;
	int* wires = (int*)malloc(2 * G * sizeof(int));
	brickwall_expand(L, nlayers, NULL, perms, NULL, wires);
	orc_cplx* t[2];
	t[0] = (orc_cplx*)malloc((size_t)16 * N * sizeof(orc_cplx));
	t[1] = (orc_cplx*)malloc((size_t)16 * N * sizeof(orc_cplx));
	memset(out, 0, (size_t)16 * N * sizeof(orc_cplx));
	for (int p = 0; p < per; p++) {
		const int k = l * per + p;
		orc_apply_gate_placeholder(wires[2*k], wires[2*k + 1], L, cache[k].data, t[0]);
		int cur = 0;
		for (int q = k + 1; q < G; q++) {
			orc_apply_gate_to_array(&vlist[q / per], wires[2*q], wires[2*q + 1], L, 16, t[cur], t[1 - cur]);
			cur = 1 - cur;
		}
		for (long e = 0; e < 16 * N; e++) out[e] += t[cur][e];
	}
	free(t[0]); free(t[1]); free(wires);
	return 0;
}

/* src/target.c:687-806: f, per-layer gradients and the complex Hessian summed over
 * all basis columns (one forward pass and one backward_hessian per column) */
int orc_brickwall_target_gradient_hessian(orc_linear_func uf, void* ud, const orc_mat4* vlist, int nlayers, int L,
                                          const int* perms, orc_cplx* fval, orc_mat4* dvlist, orc_cplx* hess)
{
	const int per = L / 2, G = nlayers * per, m = 16 * nlayers;
	const long N = 1L << L;
	orc_sv psi = { sv_alloc(L), L }, upsi = { sv_alloc(L), L }, wpsi = { sv_alloc(L), L };
	orc_sv* cache = (orc_sv*)malloc(G * sizeof(orc_sv));
	for (int k = 0; k < G; k++) { cache[k].data = sv_alloc(L); cache[k].nqubits = L; }
	orc_mat4* dv = (orc_mat4*)malloc(nlayers * sizeof(orc_mat4));
	orc_cplx* hu = (orc_cplx*)malloc((size_t)m * m * sizeof(orc_cplx));
	for (int l = 0; l < nlayers; l++) memset(&dvlist[l], 0, sizeof(orc_mat4));
	memset(hess, 0, (size_t)m * m * sizeof(orc_cplx));
	orc_cplx f = 0;
	int ret = 0;
	for (long b = 0; b < N && !ret; b++) {
		if (target_column(uf, ud, b, &psi, &upsi) < 0) { ret = -2; break; }
		memset(psi.data, 0, N * sizeof(orc_cplx));
		psi.data[b] = 1;
		orc_brickwall_forward(vlist, nlayers, perms, &psi, cache, &wpsi);
		for (long a = 0; a < N; a++) f += upsi.data[a] * wpsi.data[a];
		orc_brickwall_backward_hessian(vlist, nlayers, perms, cache, &upsi, &psi, dv, hu);
		for (int l = 0; l < nlayers; l++)
			for (int e = 0; e < 16; e++) dvlist[l].data[e] += dv[l].data[e];
		for (long e = 0; e < (long)m * m; e++) hess[e] += hu[e];
	}
	*fval = f;
	for (int k = 0; k < G; k++) free(cache[k].data);
	free(cache); free(dv); free(hu);
	free(psi.data); free(upsi.data); free(wpsi.data);
	return ret;
}

/* src/target.c:937-987: real (16 nlayers)^2 Riemannian Hessian from the complex one;
 * dvlist holds the conjugated gradients.  Column (b, k) is the Hessian applied to
 * the tangent direction real_to_tangent(e_k, V_b); rows of layers a <= b are
 * computed, the rest mirrored. */
static void project_hessian_matrix(int nlayers, const orc_mat4* vlist, const orc_mat4* dvlist, const orc_cplx* hess,
                                   double* H)
{
	const int m = 16 * nlayers;
	for (int a = 0; a < nlayers; a++)
		for (int b = a; b < nlayers; b++)
			for (int k = 0; k < 16; k++) {
				double r[16] = { 0 };
				r[k] = 1;
				orc_mat4 z, g;
				orc_real_to_tangent(r, &vlist[b], &z);
				for (int x = 0; x < 16; x++) {
					orc_cplx s = 0;
					for (int y = 0; y < 16; y++) s += hess[hidx(nlayers, a, x, b, y)] * z.data[y];
					g.data[x] = conj(s);
				}
				if (a == b) {
					orc_mat4 p, gh, t;
					orc_project_tangent(&vlist[a], &g, &p);
					orc_adjoint(&dvlist[a], &gh);
					orc_symmetric_triple_product(&z, &gh, &vlist[a], &t);
					for (int e = 0; e < 16; e++) g.data[e] = p.data[e] - t.data[e];
				}
				orc_tangent_to_real(&vlist[a], &g, r);
				for (int x = 0; x < 16; x++) H[hidx(nlayers, a, x, b, k)] = r[x];
			}
	for (int row = 0; row < m; row++)
		for (int col = 0; col < row; col++) H[(long)row * m + col] = H[(long)col * m + row];
}

/* src/target.c:996-1035 */
int orc_brickwall_target_gradient_vector_hessian_matrix(orc_linear_func uf, void* ud, const orc_mat4* vlist,
                                                        int nlayers, int L, const int* perms, orc_cplx* fval,
                                                        double* grad_vec, double* H)
{
	const int m = 16 * nlayers;
	orc_mat4* dv = (orc_mat4*)malloc(nlayers * sizeof(orc_mat4));
	orc_cplx* hess = (orc_cplx*)malloc((size_t)m * m * sizeof(orc_cplx));
	int ret = orc_brickwall_target_gradient_hessian(uf, ud, vlist, nlayers, L, perms, fval, dv, hess);
	if (!ret) {
		for (int l = 0; l < nlayers; l++) {
			for (int e = 0; e < 16; e++) dv[l].data[e] = conj(dv[l].data[e]);
			orc_tangent_to_real(&vlist[l], &dv[l], &grad_vec[16*l]);
		}
		project_hessian_matrix(nlayers, vlist, dv, hess, H);
	}
	free(dv); free(hess);
	return ret;
}

/* row-major y = A x with sequential row sums (cblas_dgemv, alpha 1, beta 0) */
static void gemv_rows(int n, const double* a, const double* x, double* y)
{
	for (int r = 0; r < n; r++) y[r] = dot(n, a + (long)r * n, x);
}

/* src/trust_region.c:83-141 */
bool orc_truncated_cg_hmat(const double* grad, const double* hess, int n, double radius,
                           const orc_tcg_params* params, double* z)
{
	double* r = (double*)malloc(n * sizeof(double));
	double* d = (double*)malloc(n * sizeof(double));
	double* hd = (double*)malloc(n * sizeof(double));
	memcpy(r, grad, n * sizeof(double));
	double rsq = dot(n, r, r);
	const double stoptol = fmax(params->abstol, params->reltol * sqrt(rsq));
	memset(z, 0, n * sizeof(double));
	for (int k = 0; k < n; k++) d[k] = -r[k];
	bool boundary = false;
	for (int it = 0; it < params->maxiter; it++) {
		gemv_rows(n, hess, d, hd);
		const double dhd = dot(n, d, hd);
		const double t = to_boundary(z, d, n, radius);
		const double alpha = rsq / dhd;
		if (dhd <= 0 || alpha > t) {
			for (int k = 0; k < n; k++) z[k] += t * d[k];
			boundary = true;
			break;
		}
		for (int k = 0; k < n; k++) r[k] += alpha * hd[k];
		for (int k = 0; k < n; k++) z[k] += alpha * d[k];
		const double rsq_next = dot(n, r, r);
		if (sqrt(rsq_next) <= stoptol) break;
		const double beta = rsq_next / rsq;
		for (int k = 0; k < n; k++) d[k] = beta * d[k] - r[k];
		rsq = rsq_next;
	}
	free(r); free(d); free(hd);
	return boundary;
}

/* src/trust_region.c:230-293 */
void orc_rtr_optimize_hmat(orc_target_func f, orc_target_grad_hess_func f_deriv_hess, void* fdata,
                           orc_retract_func retract, void* rdata, int n, const double* x_init, int m,
                           const orc_rtr_params* params, int niter, double* f_iter, double* x_final,
                           int* accepted, int* on_boundary)
{
	double* x = (double*)malloc(m * sizeof(double));
	double* xn = (double*)malloc(m * sizeof(double));
	double* grad = (double*)malloc(n * sizeof(double));
	double* hess = (double*)malloc((size_t)n * n * sizeof(double));
	double* eta = (double*)malloc(n * sizeof(double));
	double* heta = (double*)malloc(n * sizeof(double));
	memcpy(x, x_init, m * sizeof(double));
	double radius = params->radius_init;
	for (int k = 0; k < niter; k++) {
		const double fx = f_deriv_hess(x, fdata, grad, hess);
		const bool bnd = orc_truncated_cg_hmat(grad, hess, n, radius, &params->tcg, eta);
		retract(x, eta, rdata, xn);
		f_iter[k] = fx;
		gemv_rows(n, hess, eta, heta);
		const double rho = (f(xn, fdata) - fx) / (dot(n, grad, eta) + 0.5 * dot(n, eta, heta));
		if (rho < 0.25) radius *= 0.25;
		else if (rho > 0.75 && bnd) radius = fmin(2 * radius, params->maxradius);
		const int acc = rho > params->rho_trust;
		if (acc) { double* t = x; x = xn; xn = t; }
		if (accepted) accepted[k] = acc;
		if (on_boundary) on_boundary[k] = bnd;
	}
	memcpy(x_final, x, m * sizeof(double));
	f_iter[niter] = f(x_final, fdata);
	free(x); free(xn); free(grad); free(hess); free(eta); free(heta);
}

/* src/brickwall_opt.c:85-100 */
static double glue_fdh(const double* x, void* fd, double* grad, double* hess)
{
	const glue* g = (const glue*)fd;
	orc_cplx f;
	int ret = orc_brickwall_target_gradient_vector_hessian_matrix(g->uf, g->ud, (const orc_mat4*)x,
		g->ngates_or_layers, g->L, g->perms_or_wires, &f, grad, hess);
	return ret < 0 ? -1 : creal(f);
}

/* src/brickwall_opt.c:159-186 */
void orc_optimize_brickwall_hmat(orc_linear_func uf, void* ud, const orc_mat4* vstart, int nlayers, int L,
                                 const int* perms, const orc_rtr_params* params, int niter,
                                 double* f_iter, orc_mat4* vopt, int* accepted, int* on_boundary)
{
	glue g = { uf, ud, perms, nlayers, L, 1 };
	int k = nlayers;
	orc_rtr_optimize_hmat(glue_f, glue_fdh, &g, glue_retract, &k, 16 * nlayers, (const double*)vstart,
	                      32 * nlayers, params, niter, f_iter, (double*)vopt, accepted, on_boundary);
}

/* ------------------------------------------------------------ sampling estimator */

/* PCG32 (O'Neill 2014, the XSH-RR output of a 64-bit LCG; the reference vendors it as
 * src/pcg_basic.c): one step, returning the output of the old state */
static uint32_t pcg32_step(orc_pcg32* g)
{
	const uint64_t old = g->state;
	g->state = old * 6364136223846793005ULL + g->inc;
	const uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
	const uint32_t rot = (uint32_t)(old >> 59u);
	return (xs >> rot) | (xs << ((32u - rot) & 31u));
}

/* src/pcg_basic.c:31-38 */
static void pcg32_seed(orc_pcg32* g, uint64_t initstate, uint64_t initseq)
{
	g->state = 0;
	g->inc = (initseq << 1u) | 1u;
	pcg32_step(g);
	g->state += initstate;
	pcg32_step(g);
}

/* src/rng.c:13-25 with src/pcg_basic.c:112-121 */
void orc_seed_rng(uint64_t seed, orc_rng* rng)
{
	orc_pcg32 s;
	pcg32_seed(&s, seed, 6364136223846793005ULL * seed + 1442695040888963407ULL);
	uint64_t v[4];
	for (int k = 0; k < 4; k++) {
		const uint64_t hi = pcg32_step(&s);
		v[k] = (hi << 32) | pcg32_step(&s);
	}
	uint64_t seq2 = v[3];
	const uint64_t mask = ~0ull >> 1;
	if ((v[2] & mask) == (seq2 & mask)) seq2 = ~seq2;
	pcg32_seed(&rng->gen[0], v[0], v[2]);
	pcg32_seed(&rng->gen[1], v[1], seq2);
}

/* src/pcg_basic.c:128-132 */
static uint64_t rng_u64(orc_rng* rng)
{
	const uint64_t hi = pcg32_step(&rng->gen[0]);
	return (hi << 32) | pcg32_step(&rng->gen[1]);
}

/* src/rng.c:100-123, 146-157: Box-Muller normals, complex normal / sqrt(2) */
static double rng_randn(orc_rng* rng)
{
	double u1 = ldexp((double)rng_u64(rng), -64);
	const double u2 = ldexp((double)rng_u64(rng), -64);
	if (u1 == 0) u1 = 1;
	return sqrt(-2 * log(u1)) * sin(6.2831853071795864769 * u2);
}

static orc_cplx rng_crandn(orc_rng* rng)
{
	const double x = rng_randn(rng);
	const double y = rng_randn(rng);
	return x / sqrt(2.0) + I * (y / sqrt(2.0));
}

/* the reference's real build draws one real normal per amplitude (src/statevector.c:115-121) */
static int orc_real_samples = 0;

void orc_set_real_samples(int on) { orc_real_samples = on ? 1 : 0; }

/* src/statevector.c:47-66, 102-125 */
void orc_haar_statevector(orc_sv* psi, orc_rng* rng)
{
	const long n = 1L << psi->nqubits;
	if (orc_real_samples) {
		for (long j = 0; j < n; j++) psi->data[j] = rng_randn(rng);
	} else {
		for (long j = 0; j < n; j++) psi->data[j] = rng_crandn(rng);
	}
	double s = 0;
	for (long j = 0; j < n; j++) s += creal(psi->data[j]) * creal(psi->data[j]) + cimag(psi->data[j]) * cimag(psi->data[j]);
	const double nrm = sqrt(s);
	if (nrm > 0) {
		const double a = 1. / nrm;
		for (long j = 0; j < n; j++) psi->data[j] *= a;
	}
}

/* src/target.c:85-149 */
int orc_circuit_target_sampling(orc_linear_func uf, void* ud, const orc_mat4* gates, int ngates, const int* wires,
                                int L, long nsamples, orc_rng* rng, orc_cplx* fval)
{
	const long n = 1L << L;
	orc_sv psi = { sv_alloc(L), L }, upsi = { sv_alloc(L), L }, cpsi = { sv_alloc(L), L };
	orc_cplx f = 0;
	int ret = 0;
	for (long b = 0; b < nsamples && !ret; b++) {
		orc_haar_statevector(&psi, rng);
		if (uf(&psi, ud, &upsi) < 0) { ret = -2; break; }
		for (long a = 0; a < n; a++) upsi.data[a] = -conj(upsi.data[a]);
		orc_apply_circuit(gates, ngates, wires, &psi, &cpsi);
		for (long a = 0; a < n; a++) f += upsi.data[a] * cpsi.data[a];
	}
	*fval = f * ((double)n / nsamples);
	free(psi.data); free(upsi.data); free(cpsi.data);
	return ret;
}

/* src/target.c:491-505 */
int orc_brickwall_target_sampling(orc_linear_func uf, void* ud, const orc_mat4* vlist, int nlayers, int L,
                                  const int* perms, long nsamples, orc_rng* rng, orc_cplx* fval)
{
	const int G = nlayers * (L / 2);
	orc_mat4* gates = (orc_mat4*)malloc(G * sizeof(orc_mat4));
	int* wires = (int*)malloc(2 * G * sizeof(int));
	brickwall_expand(L, nlayers, vlist, perms, gates, wires);
	int ret = orc_circuit_target_sampling(uf, ud, gates, G, wires, L, nsamples, rng, fval);
	free(gates); free(wires);
	return ret;
}

/* src/target.c:807-928 */
int orc_brickwall_target_gradient_hessian_sampling(orc_linear_func uf, void* ud, const orc_mat4* vlist, int nlayers,
                                                   int L, const int* perms, long nsamples, orc_rng* rng,
                                                   orc_cplx* fval, orc_mat4* dvlist, orc_cplx* hess)
{
	const int per = L / 2, G = nlayers * per, m = 16 * nlayers;
	const long N = 1L << L;
	orc_sv psi = { sv_alloc(L), L }, upsi = { sv_alloc(L), L }, wpsi = { sv_alloc(L), L };
	orc_sv* cache = (orc_sv*)malloc(G * sizeof(orc_sv));
	for (int k = 0; k < G; k++) { cache[k].data = sv_alloc(L); cache[k].nqubits = L; }
	orc_mat4* dv = (orc_mat4*)malloc(nlayers * sizeof(orc_mat4));
	orc_cplx* hu = (orc_cplx*)malloc((size_t)m * m * sizeof(orc_cplx));
	for (int l = 0; l < nlayers; l++) memset(&dvlist[l], 0, sizeof(orc_mat4));
	memset(hess, 0, (size_t)m * m * sizeof(orc_cplx));
	orc_cplx f = 0;
	int ret = 0;
	for (long b = 0; b < nsamples && !ret; b++) {
		orc_haar_statevector(&psi, rng);
		if (uf(&psi, ud, &upsi) < 0) { ret = -2; break; }
		for (long a = 0; a < N; a++) upsi.data[a] = -conj(upsi.data[a]);
		orc_brickwall_forward(vlist, nlayers, perms, &psi, cache, &wpsi);
		for (long a = 0; a < N; a++) f += upsi.data[a] * wpsi.data[a];
		orc_brickwall_backward_hessian(vlist, nlayers, perms, cache, &upsi, &psi, dv, hu);
		for (int l = 0; l < nlayers; l++)
			for (int e = 0; e < 16; e++) dvlist[l].data[e] += dv[l].data[e];
		for (long e = 0; e < (long)m * m; e++) hess[e] += hu[e];
	}
	const double scale = (double)N / nsamples;
	*fval = f * scale;
	for (int l = 0; l < nlayers; l++)
		for (int e = 0; e < 16; e++) dvlist[l].data[e] *= scale;
	for (long e = 0; e < (long)m * m; e++) hess[e] *= scale;
	for (int k = 0; k < G; k++) free(cache[k].data);
	free(cache); free(dv); free(hu);
	free(psi.data); free(upsi.data); free(wpsi.data);
	return ret;
}

/* src/target.c:1050-1088 */
int orc_brickwall_target_gradient_vector_hessian_matrix_sampling(orc_linear_func uf, void* ud, const orc_mat4* vlist,
                                                                 int nlayers, int L, const int* perms, long nsamples,
                                                                 orc_rng* rng, orc_cplx* fval, double* grad_vec,
                                                                 double* H)
{
	const int m = 16 * nlayers;
	orc_mat4* dv = (orc_mat4*)malloc(nlayers * sizeof(orc_mat4));
	orc_cplx* hess = (orc_cplx*)malloc((size_t)m * m * sizeof(orc_cplx));
	int ret = orc_brickwall_target_gradient_hessian_sampling(uf, ud, vlist, nlayers, L, perms, nsamples, rng, fval, dv,
	                                                         hess);
	if (!ret) {
		for (int l = 0; l < nlayers; l++) {
			for (int e = 0; e < 16; e++) dv[l].data[e] = conj(dv[l].data[e]);
			orc_tangent_to_real(&vlist[l], &dv[l], &grad_vec[16*l]);
		}
		project_hessian_matrix(nlayers, vlist, dv, hess, H);
	}
	free(dv); free(hess);
	return ret;
}

typedef struct { glue g; long nsamples; orc_rng* rng; } glue_sampling;

/* src/brickwall_opt.c:205-217 */
static double glue_f_sampling(const double* x, void* fd)
{
	const glue_sampling* s = (const glue_sampling*)fd;
	orc_cplx f;
	int ret = orc_brickwall_target_sampling(s->g.uf, s->g.ud, (const orc_mat4*)x, s->g.ngates_or_layers, s->g.L,
	                                        s->g.perms_or_wires, s->nsamples, s->rng, &f);
	return ret < 0 ? -1 : creal(f);
}

/* src/brickwall_opt.c:224-236 */
static double glue_fdh_sampling(const double* x, void* fd, double* grad, double* hess)
{
	const glue_sampling* s = (const glue_sampling*)fd;
	orc_cplx f;
	int ret = orc_brickwall_target_gradient_vector_hessian_matrix_sampling(s->g.uf, s->g.ud, (const orc_mat4*)x,
		s->g.ngates_or_layers, s->g.L, s->g.perms_or_wires, s->nsamples, s->rng, &f, grad, hess);
	return ret < 0 ? -1 : creal(f);
}

/* src/brickwall_opt.c:244-265 */
void orc_optimize_brickwall_hmat_sampling(orc_linear_func uf, void* ud, const orc_mat4* vstart, int nlayers, int L,
                                          const int* perms, long nsamples, orc_rng* rng, const orc_rtr_params* params,
                                          int niter, double* f_iter, orc_mat4* vopt, int* accepted, int* on_boundary)
{
	glue_sampling s = { { uf, ud, perms, nlayers, L, 1 }, nsamples, rng };
	int k = nlayers;
	orc_rtr_optimize_hmat(glue_f_sampling, glue_fdh_sampling, &s, glue_retract, &k, 16 * nlayers,
	                      (const double*)vstart, 32 * nlayers, params, niter, f_iter, (double*)vopt, accepted,
	                      on_boundary);
}

/* ------------------------------------------------------------ block-encoding target */

/* index of a half-register basis state b in the full register: bit i of b becomes bit
 * 2 i + 1 (the even-numbered qubits; the odd ones stay |0>), src/target.c:1148-1157 */
static long blockenc_index(long b, int half)
{
	long c = 0;
	for (int i = 0; i < half; i++) c |= ((b >> i) & 1L) << (2 * i + 1);
	return c;
}

/* src/target.c:1100-1193 (f), 1202-1333 (f and gradient), 1380-1623 (f, gradient and the
 * two complex Hessians); what: 0 f, 1 f and gradient, 2 everything */
static int blockenc_sums(int what, orc_linear_func hf, void* hd, const orc_mat4* vlist, int nlayers, int L,
                         const int* perms, double* fval, orc_mat4* dvlist, orc_cplx* hess1, orc_cplx* hess2)
{
	const int half = L / 2, per = L / 2, G = nlayers * per, m = 16 * nlayers;
	const long s = 1L << half, N = 1L << L;
	orc_sv psi = { sv_alloc(half), half }, hpsi = { sv_alloc(half), half };
	orc_sv chi = { sv_alloc(L), L }, wchi = { sv_alloc(L), L };
	orc_sv* cache = (orc_sv*)malloc(G * sizeof(orc_sv));
	for (int k = 0; k < G; k++) { cache[k].data = sv_alloc(L); cache[k].nqubits = L; }
	orc_mat4* dv = (orc_mat4*)malloc(nlayers * sizeof(orc_mat4));
	orc_cplx* hu = what == 2 ? (orc_cplx*)malloc((size_t)m * m * sizeof(orc_cplx)) : NULL;
	orc_cplx* phi = what == 2 ? (orc_cplx*)malloc((size_t)nlayers * s * 16 * sizeof(orc_cplx)) : NULL;
	orc_cplx* tmp = what == 2 ? (orc_cplx*)malloc((size_t)N * 16 * sizeof(orc_cplx)) : NULL;
	if (what >= 1) for (int l = 0; l < nlayers; l++) memset(&dvlist[l], 0, sizeof(orc_mat4));
	if (what == 2) {
		memset(hess1, 0, (size_t)m * m * sizeof(orc_cplx));
		memset(hess2, 0, (size_t)m * m * sizeof(orc_cplx));
	}
	double f = 0;
	int ret = 0;
	for (long b = 0; b < s && !ret; b++) {
		memset(psi.data, 0, s * sizeof(orc_cplx));
		psi.data[b] = 1;
		if (hf(&psi, hd, &hpsi) < 0) { ret = -2; break; }
		memset(chi.data, 0, N * sizeof(orc_cplx));
		chi.data[blockenc_index(b, half)] = 1;
		orc_brickwall_forward(vlist, nlayers, perms, &chi, cache, &wchi);
		memset(chi.data, 0, N * sizeof(orc_cplx));
		for (long a = 0; a < s; a++) {
			const long c = blockenc_index(a, half);
			const orc_cplx d = wchi.data[c] - hpsi.data[a];
			f += 0.5 * (creal(d) * creal(d) + cimag(d) * cimag(d));
			chi.data[c] = conj(d);
		}
		if (what == 0) continue;
		if (what == 1) {
			orc_brickwall_backward(vlist, nlayers, perms, cache, &chi, &wchi, dv);
		} else {
			orc_brickwall_backward_hessian(vlist, nlayers, perms, cache, &chi, &wchi, dv, hu);
			for (long e = 0; e < (long)m * m; e++) hess1[e] += hu[e];
			/* Jacobian of P^dag W P e_b in the gate entries of each layer */
			for (int l = 0; l < nlayers; l++) {
				orc_apply_brickwall_placeholder(vlist, nlayers, perms, l, cache, tmp);
				for (long a = 0; a < s; a++)
					for (int j = 0; j < 16; j++)
						phi[((size_t)l * s + a) * 16 + j] = tmp[blockenc_index(a, half) * 16 + j];
			}
			/* Gauss-Newton part: lower blocks, then the upper ones by conjugate symmetry */
			memset(hu, 0, (size_t)m * m * sizeof(orc_cplx));
			for (int l = 0; l < nlayers; l++)
				for (int k = 0; k <= l; k++)
					for (long a = 0; a < s; a++)
						for (int i = 0; i < 16; i++)
							for (int j = 0; j < 16; j++)
								hu[hidx(nlayers, l, i, k, j)] += conj(phi[((size_t)l * s + a) * 16 + i])
								                                * phi[((size_t)k * s + a) * 16 + j];
			for (int l = 0; l < nlayers; l++)
				for (int k = l + 1; k < nlayers; k++)
					for (int i = 0; i < 16; i++)
						for (int j = 0; j < 16; j++) hu[hidx(nlayers, l, i, k, j)] = conj(hu[hidx(nlayers, k, j, l, i)]);
			for (long e = 0; e < (long)m * m; e++) hess2[e] += hu[e];
		}
		for (int l = 0; l < nlayers; l++)
			for (int e = 0; e < 16; e++) dvlist[l].data[e] += dv[l].data[e];
	}
	*fval = f;
	for (int k = 0; k < G; k++) free(cache[k].data);
	free(cache); free(dv); free(hu); free(phi); free(tmp);
	free(psi.data); free(hpsi.data); free(chi.data); free(wchi.data);
	return ret;
}

int orc_blockenc_target(orc_linear_func hf, void* hd, const orc_mat4* vlist, int nlayers, int L, const int* perms,
                        double* fval)
{
	return blockenc_sums(0, hf, hd, vlist, nlayers, L, perms, fval, NULL, NULL, NULL);
}

int orc_blockenc_target_and_gradient(orc_linear_func hf, void* hd, const orc_mat4* vlist, int nlayers, int L,
                                     const int* perms, double* fval, orc_mat4* dvlist)
{
	return blockenc_sums(1, hf, hd, vlist, nlayers, L, perms, fval, dvlist, NULL, NULL);
}

/* src/target.c:1341-1370 */
int orc_blockenc_target_and_gradient_vector(orc_linear_func hf, void* hd, const orc_mat4* vlist, int nlayers, int L,
                                            const int* perms, double* fval, double* grad_vec)
{
	orc_mat4* dv = (orc_mat4*)malloc(nlayers * sizeof(orc_mat4));
	int ret = blockenc_sums(1, hf, hd, vlist, nlayers, L, perms, fval, dv, NULL, NULL);
	if (!ret)
		for (int l = 0; l < nlayers; l++) {
			for (int e = 0; e < 16; e++) dv[l].data[e] = conj(dv[l].data[e]);
			orc_tangent_to_real(&vlist[l], &dv[l], &grad_vec[16*l]);
		}
	free(dv);
	return ret;
}

int orc_blockenc_target_gradient_hessian(orc_linear_func hf, void* hd, const orc_mat4* vlist, int nlayers, int L,
                                         const int* perms, double* fval, orc_mat4* dvlist, orc_cplx* hess1,
                                         orc_cplx* hess2)
{
	return blockenc_sums(2, hf, hd, vlist, nlayers, L, perms, fval, dvlist, hess1, hess2);
}

/* src/target.c:1631-1720: H column (j, k) from conj(hess1 Z) + hess2 Z */
int orc_blockenc_target_gradient_vector_hessian_matrix(orc_linear_func hf, void* hd, const orc_mat4* vlist,
                                                       int nlayers, int L, const int* perms, double* fval,
                                                       double* grad_vec, double* H)
{
	const int m = 16 * nlayers;
	orc_mat4* dv = (orc_mat4*)malloc(nlayers * sizeof(orc_mat4));
	orc_cplx* h1 = (orc_cplx*)malloc((size_t)m * m * sizeof(orc_cplx));
	orc_cplx* h2 = (orc_cplx*)malloc((size_t)m * m * sizeof(orc_cplx));
	int ret = blockenc_sums(2, hf, hd, vlist, nlayers, L, perms, fval, dv, h1, h2);
	if (!ret) {
		for (int l = 0; l < nlayers; l++) {
			for (int e = 0; e < 16; e++) dv[l].data[e] = conj(dv[l].data[e]);
			orc_tangent_to_real(&vlist[l], &dv[l], &grad_vec[16*l]);
		}
		for (int a = 0; a < nlayers; a++)
			for (int b = a; b < nlayers; b++)
				for (int k = 0; k < 16; k++) {
					double r[16] = { 0 };
					r[k] = 1;
					orc_mat4 z, g;
					orc_real_to_tangent(r, &vlist[b], &z);
					for (int x = 0; x < 16; x++) {
						orc_cplx s1 = 0, s2 = 0;
						for (int y = 0; y < 16; y++) {
							s1 += h1[hidx(nlayers, a, x, b, y)] * z.data[y];
							s2 += h2[hidx(nlayers, a, x, b, y)] * z.data[y];
						}
						g.data[x] = conj(s1) + s2;
					}
					if (a == b) {
						orc_mat4 p, gh, t;
						orc_project_tangent(&vlist[a], &g, &p);
						orc_adjoint(&dv[a], &gh);
						orc_symmetric_triple_product(&z, &gh, &vlist[a], &t);
						for (int e = 0; e < 16; e++) g.data[e] = p.data[e] - t.data[e];
					}
					orc_tangent_to_real(&vlist[a], &g, r);
					for (int x = 0; x < 16; x++) H[hidx(nlayers, a, x, b, k)] = r[x];
				}
		for (int row = 0; row < m; row++)
			for (int col = 0; col < row; col++) H[(long)row * m + col] = H[(long)col * m + row];
	}
	free(dv); free(h1); free(h2);
	return ret;
}
