// librqcopt_gpu_real.so: the reference's real-orthogonal build (compiled without
// COMPLEX_CIRCUIT; declarations in include/rqcopt_gpu_real.h) on the GPU engine of
// librqcopt_gpu.so.
//
// Every quantity the real build forms -- states, gate products, the basis-column
// sums of f, gradient, HVP and Hessian, the trust-region steps -- is what the
// complex build forms on the same real inputs: with zero imaginary parts, every
// complex product and sum the complex engine evaluates has a zero imaginary part
// and the real build's value as real part, and the complex build's conjugations
// are the identity.  So each function here embeds its real arguments as complex
// ones, calls the complex library (loaded from the same directory with
// RTLD_LOCAL, so its symbols do not clash with these), and returns the real
// parts.  What the builds do differently is restated here:
//   - a tangent direction of a real gate has 6 parameters, the upper triangle of
//     an antisymmetric matrix scaled by sqrt(2) (src/matrix.c:245-271, 288-300); the
//     complex build's 16 parameters of the same real antisymmetric w are its 16
//     entries, so the 6 are sqrt(2) * w[1, 2, 3, 6, 7, 11];
//   - Haar-random sample states have one real normal per amplitude
//     (src/statevector.c:115-121), drawn on the GPU by the complex library in its
//     real-sample mode;
//   - the f / gradient / HVP sums run over half the columns: the complex engine takes
//     the paired basis columns e_b + i e_{b + N/2} (rqcopt_gpu_set_real_pairs); every
//     sum pairs an adjoint-type state, -conj(U psi) = -(U e_b) + i (U e_{b+N/2}), with a
//     forward-type state, both propagated by real matrices, so its real part is the
//     sum of the two real columns' terms;
//   - the block-encoding Hessian is one matrix, the sum of the two terms
//     (src/target.c:1595-1597);
//   - the optimisers run the generic trust region over 6 nlayers (or 6 ngates)
//     parameters with the real retraction (src/brickwall_opt.c:22-149,
//     src/circuit_opt.c).
// Device-native targets (rqcopt_brickwall_ufunc, rqcopt_circuit_ufunc,
// rqcopt_dense_ufunc with real gates or matrix) map to the complex library's, so
// the target stays on the GPU; any other linear_func is called on the real and
// imaginary parts of each column the engine hands out (once for basis columns).
#pragma GCC visibility push(default)
#include "rqcopt_gpu_real.h"
#pragma GCC visibility pop

#include <dlfcn.h>
#include <libgen.h>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

namespace {

using cd = std::complex<double>;

// the complex build's types (rqcopt_gpu.h), under other names
namespace cx {
struct mat4x4 { cd data[16]; };
struct statevector { cd* data; int nqubits; };
struct statevector_array { cd* data; int nqubits; int nstates; };
struct quantum_circuit_cache { statevector* psi_list; int nqubits; int ngates; };
typedef int (*linear_func)(const statevector* psi, void* fdata, statevector* psi_out);
struct brickwall_target { const mat4x4* vlist; int nlayers; const int* const* perms; };
struct circuit_target { const mat4x4* gates; int ngates; const int* wires; };
struct dense_target { const cd* u; int nqubits; };
}  // namespace cx

constexpr int E_ALLOC = -1, E_CUDA = -5, E_ARG = -6;
constexpr int UPPER[6] = { 1, 2, 3, 6, 7, 11 };

int g_error = 0;   // adapter-level error of the last void call

void* complex_library()
{
	static void* handle = [] {
		Dl_info info;
		std::string dir = ".";
		if (dladdr(reinterpret_cast<void*>(&complex_library), &info) && info.dli_fname) {
			std::vector<char> path(info.dli_fname, info.dli_fname + std::strlen(info.dli_fname) + 1);
			dir = dirname(path.data());
		}
		const std::string lib = dir + "/librqcopt_gpu.so";
		void* h = dlopen(lib.c_str(), RTLD_NOW | RTLD_LOCAL);
		if (!h) fprintf(stderr, "librqcopt_gpu_real: cannot load %s: %s\n", lib.c_str(), dlerror());
		return h;
	}();
	return handle;
}

template <class F>
F sym(const char* name)
{
	void* h = complex_library();
	void* p = h ? dlsym(h, name) : nullptr;
	if (!p) fprintf(stderr, "librqcopt_gpu_real: symbol %s missing from librqcopt_gpu.so\n", name);
	return reinterpret_cast<F>(p);
}

// resolve complex-library function `name` once, with the given signature
#define CX(name, ret, ...)                                                      \
	static const auto cx_##name = sym<ret (*)(__VA_ARGS__)>(#name);             \
	if (!cx_##name) return fail_missing<ret>();

template <class R>
R fail_missing()
{
	g_error = E_CUDA;
	if constexpr (std::is_same_v<R, void>) return;
	else if constexpr (std::is_same_v<R, bool>) return false;
	else return static_cast<R>(E_CUDA);
}

// ---------------------------------------------------------------- conversions

std::vector<cd> cvec(const double* x, size_t n)
{
	std::vector<cd> z(n);
	for (size_t k = 0; k < n; k++) z[k] = cd(x[k], 0.0);
	return z;
}

void rvec(const cd* z, size_t n, double* x)
{
	for (size_t k = 0; k < n; k++) x[k] = z[k].real();
}

std::vector<cx::mat4x4> cmats(const mat4x4* a, int n)
{
	std::vector<cx::mat4x4> z(n > 0 ? n : 0);
	for (int k = 0; k < n; k++)
		for (int e = 0; e < 16; e++) z[k].data[e] = cd(a[k].data[e], 0.0);
	return z;
}

cx::mat4x4 cmat(const mat4x4* a) { return cmats(a, 1)[0]; }

void rmats(const cx::mat4x4* z, int n, mat4x4* a)
{
	for (int k = 0; k < n; k++)
		for (int e = 0; e < 16; e++) a[k].data[e] = z[k].data[e].real();
}

size_t dim(int nqubits) { return (size_t)1 << nqubits; }

// complex copy of a real statevector
struct CState
{
	std::vector<cd> buf;
	cx::statevector sv{};
	CState() = default;
	explicit CState(int nqubits) : buf(dim(nqubits)) { sv = { buf.data(), nqubits }; }
	explicit CState(const statevector* psi) : buf(cvec(psi->data, dim(psi->nqubits))) { sv = { buf.data(), psi->nqubits }; }
	void to(statevector* psi) const { rvec(buf.data(), buf.size(), psi->data); }
};

struct CArray
{
	std::vector<cd> buf;
	cx::statevector_array a{};
	CArray(int nqubits, int nstates) : buf(dim(nqubits) * nstates) { a = { buf.data(), nqubits, nstates }; }
	explicit CArray(const statevector_array* psi) : buf(cvec(psi->data, dim(psi->nqubits) * psi->nstates))
	{
		a = { buf.data(), psi->nqubits, psi->nstates };
	}
	void to(statevector_array* psi) const { rvec(buf.data(), buf.size(), psi->data); }
};

// complex copy of a real quantum_circuit_cache (or an empty one of its shape)
struct CCache
{
	std::vector<std::vector<cd>> states;
	std::vector<cx::statevector> list;
	cx::quantum_circuit_cache c{};
	CCache(int nqubits, int ngates) : states(ngates, std::vector<cd>(dim(nqubits))), list(ngates)
	{
		for (int k = 0; k < ngates; k++) list[k] = { states[k].data(), nqubits };
		c = { list.data(), nqubits, ngates };
	}
	explicit CCache(const quantum_circuit_cache* r) : CCache(r->nqubits, r->ngates)
	{
		for (int k = 0; k < r->ngates; k++)
			for (size_t a = 0; a < dim(r->nqubits); a++) states[k][a] = cd(r->psi_list[k].data[a], 0.0);
	}
	void to(quantum_circuit_cache* r) const
	{
		for (int k = 0; k < r->ngates && k < c.ngates; k++) rvec(states[k].data(), states[k].size(), r->psi_list[k].data);
	}
};

// complex build's 16 tangent parameters -> real build's 6
void tangent16_to_6(const double* r16, int ngates, double* r6)
{
	const double s2 = std::sqrt(2.0);
	for (int g = 0; g < ngates; g++)
		for (int k = 0; k < 6; k++) r6[6 * g + k] = s2 * r16[16 * g + UPPER[k]];
}

// ---------------------------------------------------------------- targets

struct HostCallback
{
	linear_func f;
	void* data;
	std::vector<double> re, im, ore, oim;   // column buffers, reused across calls
};

// a real linear_func applied to the complex column psi: its real and imaginary parts
int host_callback(const cx::statevector* psi, void* udata, cx::statevector* out)
{
	HostCallback* cb = static_cast<HostCallback*>(udata);
	const size_t n = dim(psi->nqubits);
	std::vector<double>& re = cb->re;
	std::vector<double>& im = cb->im;
	std::vector<double>& ore = cb->ore;
	std::vector<double>& oim = cb->oim;
	re.resize(n);
	im.resize(n);
	ore.resize(n);
	oim.assign(n, 0.0);
	bool has_im = false;
	for (size_t k = 0; k < n; k++) {
		re[k] = psi->data[k].real();
		im[k] = psi->data[k].imag();
		has_im |= im[k] != 0.0;
	}
	statevector in = { re.data(), psi->nqubits }, o = { ore.data(), psi->nqubits };
	int ret = cb->f(&in, cb->data, &o);
	if (ret < 0) return ret;
	if (has_im) {
		statevector in2 = { im.data(), psi->nqubits }, o2 = { oim.data(), psi->nqubits };
		if ((ret = cb->f(&in2, cb->data, &o2)) < 0) return ret;
	}
	for (size_t k = 0; k < n; k++) out->data[k] = cd(ore[k], oim[k]);
	return 0;
}

// the complex form of a target (ufunc, udata); keeps the converted data alive
struct Target
{
	cx::linear_func f = nullptr;
	void* data = nullptr;
	HostCallback cb{};
	std::vector<cx::mat4x4> gates;
	cx::brickwall_target bw{};
	cx::circuit_target ct{};
	std::vector<cd> u;
	cx::dense_target dt{};

	Target(linear_func ufunc, void* udata)
	{
		if (ufunc == rqcopt_brickwall_ufunc && udata) {
			const auto* t = static_cast<const rqcopt_brickwall_target*>(udata);
			gates = cmats(t->vlist, t->nlayers);
			bw = { gates.data(), t->nlayers, t->perms };
			f = sym<cx::linear_func>("rqcopt_brickwall_ufunc");
			data = &bw;
		} else if (ufunc == rqcopt_circuit_ufunc && udata) {
			const auto* t = static_cast<const rqcopt_circuit_target*>(udata);
			gates = cmats(t->gates, t->ngates);
			ct = { gates.data(), t->ngates, t->wires };
			f = sym<cx::linear_func>("rqcopt_circuit_ufunc");
			data = &ct;
		} else if (ufunc == rqcopt_dense_ufunc && udata) {
			const auto* t = static_cast<const rqcopt_dense_target*>(udata);
			u = cvec(t->u, dim(t->nqubits) * dim(t->nqubits));
			dt = { u.data(), t->nqubits };
			f = sym<cx::linear_func>("rqcopt_dense_ufunc");
			data = &dt;
		} else {
			cb.f = ufunc;
			cb.data = udata;
			f = host_callback;
			data = &cb;
		}
	}
};

// real sample states for the duration of a call
struct RealSamples
{
	void (*set)(int);
	RealSamples() : set(sym<void (*)(int)>("rqcopt_gpu_set_real_samples")) { if (set) set(1); }
	~RealSamples() { if (set) set(0); }
};

// paired basis columns in the complex engine for the duration of a call: the sums of
// the f / gradient / HVP functions run over 2^(n-1) columns e_b + i e_{b + 2^(n-1)}
// and keep real parts, which are the sums over the 2^n real columns
struct RealPairs
{
	void (*set)(int);
	RealPairs() : set(sym<void (*)(int)>("rqcopt_gpu_set_real_pairs")) { if (set) set(1); }
	~RealPairs() { if (set) set(0); }
};

typedef const int* const* cperms;

// ---------------------------------------------------------------- small real matrix algebra

void mat_mul(const mat4x4* a, const mat4x4* b, mat4x4* c)
{
	for (int i = 0; i < 4; i++)
		for (int j = 0; j < 4; j++) {
			double s = 0;
			for (int k = 0; k < 4; k++) s += a->data[4 * i + k] * b->data[4 * k + j];
			c->data[4 * i + j] = s;
		}
}

}  // namespace

extern "C" {

// ================================================================ statevector.h

int allocate_statevector(int nqubits, struct statevector* psi)
{
	const size_t bytes = (dim(nqubits) * sizeof(double) + 63) & ~(size_t)63;
	psi->data = static_cast<double*>(aligned_alloc(64, bytes));
	if (!psi->data) return E_ALLOC;
	psi->nqubits = nqubits;
	return 0;
}

void free_statevector(struct statevector* psi)
{
	free(psi->data);
	psi->data = nullptr;
	psi->nqubits = 0;
}

void add_statevectors(const struct statevector* psi1, const struct statevector* psi2, struct statevector* psi_sum)
{
	g_error = 0;
	if (psi1->nqubits != psi2->nqubits || psi1->nqubits != psi_sum->nqubits) { g_error = E_ARG; return; }
	for (size_t k = 0; k < dim(psi1->nqubits); k++) psi_sum->data[k] = psi1->data[k] + psi2->data[k];
}

// psi_trans[j] = psi[k], k the index j with qubit i moved to qubit perm[i] (src/statevector.c:72-98)
void transpose_statevector(const struct statevector* psi, const int* perm, struct statevector* psi_trans)
{
	g_error = 0;
	if (!psi || !psi_trans || !perm || psi->nqubits != psi_trans->nqubits || psi->nqubits < 0 || psi->nqubits > 40) {
		g_error = E_ARG;
		return;
	}
	const int L = psi->nqubits;
	std::vector<long> strides(L > 0 ? L : 1);
	std::vector<char> seen(L > 0 ? L : 1, 0);
	for (int i = 0; i < L; i++) {
		if (perm[i] < 0 || perm[i] >= L || seen[perm[i]]) {
			g_error = E_ARG;
			return;
		}
		seen[perm[i]] = 1;
		strides[L - 1 - i] = 1L << (L - 1 - perm[i]);
	}
	for (long j = 0; j < (1L << L); j++) {
		long k = 0;
		for (int i = 0; i < L; i++) k += ((j >> i) & 1) * strides[i];
		psi_trans->data[j] = psi->data[k];
	}
}

// the host random numbers need no real form: forwarded (src/pcg_basic.c, src/rng.c)
void pcg32_srandom_r(const uint64_t initstate, const uint64_t initseq, struct pcg32_random* rng)
{
	CX(pcg32_srandom_r, void, uint64_t, uint64_t, struct pcg32_random*);
	cx_pcg32_srandom_r(initstate, initseq, rng);
}

uint32_t pcg32_random_r(struct pcg32_random* rng)
{
	CX(pcg32_random_r, uint32_t, struct pcg32_random*);
	return cx_pcg32_random_r(rng);
}

uint32_t pcg32_boundedrand_r(const uint32_t bound, struct pcg32_random* rng)
{
	CX(pcg32_boundedrand_r, uint32_t, uint32_t, struct pcg32_random*);
	return cx_pcg32_boundedrand_r(bound, rng);
}

void pcg32x2_srandom_r(uint64_t seed1, uint64_t seed2, uint64_t seq1, uint64_t seq2, struct pcg32x2_random* rng)
{
	CX(pcg32x2_srandom_r, void, uint64_t, uint64_t, uint64_t, uint64_t, struct pcg32x2_random*);
	cx_pcg32x2_srandom_r(seed1, seed2, seq1, seq2, rng);
}

uint64_t pcg32x2_random_r(struct pcg32x2_random* rng)
{
	CX(pcg32x2_random_r, uint64_t, struct pcg32x2_random*);
	return cx_pcg32x2_random_r(rng);
}

uint64_t pcg32x2_boundedrand_r(const uint64_t bound, struct pcg32x2_random* rng)
{
	CX(pcg32x2_boundedrand_r, uint64_t, uint64_t, struct pcg32x2_random*);
	return cx_pcg32x2_boundedrand_r(bound, rng);
}

uint32_t rand_uint32(struct rng_state* state)
{
	CX(rand_uint32, uint32_t, struct rng_state*);
	return cx_rand_uint32(state);
}

uint64_t rand_uint64(struct rng_state* state)
{
	CX(rand_uint64, uint64_t, struct rng_state*);
	return cx_rand_uint64(state);
}

uint64_t rand_interval(const uint64_t bound, struct rng_state* state)
{
	CX(rand_interval, uint64_t, uint64_t, struct rng_state*);
	return cx_rand_interval(bound, state);
}

void rand_choice(const uint64_t bound, const uint64_t num_samples, struct rng_state* state, uint64_t* ret)
{
	g_error = 0;
	CX(rand_choice, void, uint64_t, uint64_t, struct rng_state*, uint64_t*);
	cx_rand_choice(bound, num_samples, state, ret);
}

double randu(struct rng_state* state)
{
	CX(randu, double, struct rng_state*);
	return cx_randu(state);
}

float randuf(struct rng_state* state)
{
	CX(randuf, float, struct rng_state*);
	return cx_randuf(state);
}

double randn(struct rng_state* state)
{
	CX(randn, double, struct rng_state*);
	return cx_randn(state);
}

float randnf(struct rng_state* state)
{
	CX(randnf, float, struct rng_state*);
	return cx_randnf(state);
}

// src/statevector.c:47-66 (real build): divide by the 2-norm unless it is zero
void normalize_statevector(struct statevector* psi)
{
	g_error = 0;
	if (!psi || !psi->data || psi->nqubits < 0 || psi->nqubits > 40) {
		g_error = E_ARG;
		return;
	}
	const size_t n = dim(psi->nqubits);
	double scale = 0, ssq = 1;   // scaled sum of squares
	for (size_t k = 0; k < n; k++) {
		const double av = std::fabs(psi->data[k]);
		if (av == 0) continue;
		if (scale < av) {
			ssq = 1 + ssq * (scale / av) * (scale / av);
			scale = av;
		} else {
			ssq += (av / scale) * (av / scale);
		}
	}
	const double nrm = scale * std::sqrt(ssq);
	if (nrm > 0)
		for (size_t k = 0; k < n; k++) psi->data[k] *= 1. / nrm;
}

void seed_rng_state(const uint64_t seed, struct rng_state* state)
{
	g_error = 0;
	CX(seed_rng_state, void, uint64_t, struct rng_state*);
	cx_seed_rng_state(seed, state);
}

void haar_random_statevector(struct statevector* psi, struct rng_state* rng)
{
	g_error = 0;
	CX(haar_random_statevector, void, cx::statevector*, struct rng_state*);
	RealSamples real;
	CState c(psi->nqubits);
	cx_haar_random_statevector(&c.sv, rng);
	c.to(psi);
}

int allocate_statevector_array(int nqubits, int nstates, struct statevector_array* psi_list)
{
	const size_t bytes = (dim(nqubits) * nstates * sizeof(double) + 63) & ~(size_t)63;
	psi_list->data = static_cast<double*>(aligned_alloc(64, bytes));
	if (!psi_list->data) return E_ALLOC;
	psi_list->nqubits = nqubits;
	psi_list->nstates = nstates;
	return 0;
}

void free_statevector_array(struct statevector_array* psi_list)
{
	free(psi_list->data);
	psi_list->data = nullptr;
}

// ================================================================ gate.h

void apply_gate(const struct mat4x4* gate, const int i, const int j, const struct statevector* psi,
                struct statevector* psi_out)
{
	g_error = 0;
	CX(apply_gate, void, const cx::mat4x4*, int, int, const cx::statevector*, cx::statevector*);
	const cx::mat4x4 g = cmat(gate);
	CState in(psi), out(psi_out->nqubits);
	cx_apply_gate(&g, i, j, &in.sv, &out.sv);
	out.to(psi_out);
}

void apply_gate_backward(const struct mat4x4* gate, const int i, const int j, const struct statevector* psi,
                         const struct statevector* dpsi_out, struct statevector* dpsi, struct mat4x4* dgate)
{
	g_error = 0;
	CX(apply_gate_backward, void, const cx::mat4x4*, int, int, const cx::statevector*, const cx::statevector*,
	   cx::statevector*, cx::mat4x4*);
	const cx::mat4x4 g = cmat(gate);
	CState in(psi), dout(dpsi_out), d(dpsi->nqubits);
	cx::mat4x4 dg;
	cx_apply_gate_backward(&g, i, j, &in.sv, &dout.sv, &d.sv, &dg);
	d.to(dpsi);
	rmats(&dg, 1, dgate);
}

void apply_gate_to_array(const struct mat4x4* gate, const int i, const int j, const struct statevector_array* psi,
                         struct statevector_array* psi_out)
{
	g_error = 0;
	CX(apply_gate_to_array, void, const cx::mat4x4*, int, int, const cx::statevector_array*, cx::statevector_array*);
	const cx::mat4x4 g = cmat(gate);
	CArray in(psi), out(psi_out->nqubits, psi_out->nstates);
	cx_apply_gate_to_array(&g, i, j, &in.a, &out.a);
	out.to(psi_out);
}

void apply_gate_backward_array(const struct mat4x4* gate, const int i, const int j, const struct statevector_array* psi,
                               const struct statevector* dpsi_out, struct mat4x4* dgates)
{
	g_error = 0;
	CX(apply_gate_backward_array, void, const cx::mat4x4*, int, int, const cx::statevector_array*,
	   const cx::statevector*, cx::mat4x4*);
	const cx::mat4x4 g = cmat(gate);
	CArray in(psi);
	CState dout(dpsi_out);
	std::vector<cx::mat4x4> dg(psi->nstates);
	cx_apply_gate_backward_array(&g, i, j, &in.a, &dout.sv, dg.data());
	rmats(dg.data(), psi->nstates, dgates);
}

void apply_gate_placeholder(const int i, const int j, const struct statevector* psi, struct statevector_array* psi_out)
{
	g_error = 0;
	CX(apply_gate_placeholder, void, int, int, const cx::statevector*, cx::statevector_array*);
	CState in(psi);
	CArray out(psi_out->nqubits, psi_out->nstates);
	cx_apply_gate_placeholder(i, j, &in.sv, &out.a);
	out.to(psi_out);
}

// ================================================================ quantum_circuit.h

int apply_quantum_circuit(const struct mat4x4 gates[], const int ngates, const int wires[],
                          const struct statevector* psi, struct statevector* psi_out)
{
	CX(apply_quantum_circuit, int, const cx::mat4x4*, int, const int*, const cx::statevector*, cx::statevector*);
	const auto g = cmats(gates, ngates);
	CState in(psi), out(psi_out->nqubits);
	const int ret = cx_apply_quantum_circuit(g.data(), ngates, wires, &in.sv, &out.sv);
	if (!ret) out.to(psi_out);
	return ret;
}

int allocate_quantum_circuit_cache(const int nqubits, const int ngates, struct quantum_circuit_cache* cache)
{
	cache->nqubits = nqubits;
	cache->ngates = ngates;
	cache->psi_list = static_cast<statevector*>(calloc(ngates > 0 ? ngates : 1, sizeof(statevector)));
	if (!cache->psi_list) return E_ALLOC;
	for (int k = 0; k < ngates; k++)
		if (allocate_statevector(nqubits, &cache->psi_list[k]) < 0) return E_ALLOC;
	return 0;
}

void free_quantum_circuit_cache(struct quantum_circuit_cache* cache)
{
	if (!cache->psi_list) return;
	for (int k = 0; k < cache->ngates; k++) free_statevector(&cache->psi_list[k]);
	free(cache->psi_list);
	cache->psi_list = nullptr;
}

int quantum_circuit_forward(const struct mat4x4 gates[], const int ngates, const int wires[],
                            const struct statevector* psi, struct quantum_circuit_cache* cache, struct statevector* psi_out)
{
	CX(quantum_circuit_forward, int, const cx::mat4x4*, int, const int*, const cx::statevector*,
	   cx::quantum_circuit_cache*, cx::statevector*);
	if (cache->ngates != ngates || cache->nqubits != psi->nqubits) return E_ARG;
	const auto g = cmats(gates, ngates);
	CState in(psi), out(psi_out->nqubits);
	CCache cc(psi->nqubits, ngates);
	const int ret = cx_quantum_circuit_forward(g.data(), ngates, wires, &in.sv, &cc.c, &out.sv);
	if (!ret) {
		out.to(psi_out);
		cc.to(cache);
	}
	return ret;
}

int quantum_circuit_backward(const struct mat4x4 gates[], const int ngates, const int wires[],
                             const struct quantum_circuit_cache* cache, const struct statevector* dpsi_out,
                             struct statevector* dpsi, struct mat4x4 dgates[])
{
	CX(quantum_circuit_backward, int, const cx::mat4x4*, int, const int*, const cx::quantum_circuit_cache*,
	   const cx::statevector*, cx::statevector*, cx::mat4x4*);
	const auto g = cmats(gates, ngates);
	CCache cc(cache);
	CState dout(dpsi_out), d(dpsi->nqubits);
	std::vector<cx::mat4x4> dg(ngates);
	const int ret = cx_quantum_circuit_backward(g.data(), ngates, wires, &cc.c, &dout.sv, &d.sv, dg.data());
	if (!ret) {
		d.to(dpsi);
		rmats(dg.data(), ngates, dgates);
	}
	return ret;
}

int quantum_circuit_gates_hessian_vector_product(const struct mat4x4 gates[], const struct mat4x4 gatedirs[],
                                                 const int ngates, const int wires[], const struct statevector* psi,
                                                 const struct statevector* phi, struct statevector* psi_out,
                                                 struct mat4x4 dgates[], struct mat4x4 hess_gatedirs[])
{
	CX(quantum_circuit_gates_hessian_vector_product, int, const cx::mat4x4*, const cx::mat4x4*, int, const int*,
	   const cx::statevector*, const cx::statevector*, cx::statevector*, cx::mat4x4*, cx::mat4x4*);
	const auto g = cmats(gates, ngates), z = cmats(gatedirs, ngates);
	CState in(psi), ph(phi), out(psi_out->nqubits);
	std::vector<cx::mat4x4> dg(ngates), hg(ngates);
	const int ret = cx_quantum_circuit_gates_hessian_vector_product(g.data(), z.data(), ngates, wires, &in.sv, &ph.sv,
	                                                                &out.sv, dg.data(), hg.data());
	if (!ret) {
		out.to(psi_out);
		rmats(dg.data(), ngates, dgates);
		rmats(hg.data(), ngates, hess_gatedirs);
	}
	return ret;
}

// ================================================================ brickwall_circuit.h

int apply_brickwall_unitary(const struct mat4x4 vlist[], const int nlayers, const int* perms[],
                            const struct statevector* psi, struct statevector* psi_out)
{
	CX(apply_brickwall_unitary, int, const cx::mat4x4*, int, const int**, const cx::statevector*, cx::statevector*);
	const auto v = cmats(vlist, nlayers);
	CState in(psi), out(psi_out->nqubits);
	const int ret = cx_apply_brickwall_unitary(v.data(), nlayers, perms, &in.sv, &out.sv);
	if (!ret) out.to(psi_out);
	return ret;
}

int brickwall_unitary_forward(const struct mat4x4 vlist[], int nlayers, const int* perms[], const struct statevector* psi,
                              struct quantum_circuit_cache* cache, struct statevector* psi_out)
{
	CX(brickwall_unitary_forward, int, const cx::mat4x4*, int, const int**, const cx::statevector*,
	   cx::quantum_circuit_cache*, cx::statevector*);
	if (cache->ngates != nlayers * (psi->nqubits / 2) || cache->nqubits != psi->nqubits) return E_ARG;
	const auto v = cmats(vlist, nlayers);
	CState in(psi), out(psi_out->nqubits);
	CCache cc(psi->nqubits, cache->ngates);
	const int ret = cx_brickwall_unitary_forward(v.data(), nlayers, perms, &in.sv, &cc.c, &out.sv);
	if (!ret) {
		out.to(psi_out);
		cc.to(cache);
	}
	return ret;
}

int brickwall_unitary_backward(const struct mat4x4 vlist[], int nlayers, const int* perms[],
                               const struct quantum_circuit_cache* cache, const struct statevector* dpsi_out,
                               struct statevector* dpsi, struct mat4x4 dvlist[])
{
	CX(brickwall_unitary_backward, int, const cx::mat4x4*, int, const int**, const cx::quantum_circuit_cache*,
	   const cx::statevector*, cx::statevector*, cx::mat4x4*);
	const auto v = cmats(vlist, nlayers);
	CCache cc(cache);
	CState dout(dpsi_out), d(dpsi->nqubits);
	std::vector<cx::mat4x4> dv(nlayers);
	const int ret = cx_brickwall_unitary_backward(v.data(), nlayers, perms, &cc.c, &dout.sv, &d.sv, dv.data());
	if (!ret) {
		d.to(dpsi);
		rmats(dv.data(), nlayers, dvlist);
	}
	return ret;
}

int brickwall_unitary_backward_hessian(const struct mat4x4 vlist[], int nlayers, const int* perms[],
                                       const struct quantum_circuit_cache* cache, const struct statevector* dpsi_out,
                                       struct statevector* dpsi, struct mat4x4 dvlist[], numeric* hess)
{
	CX(brickwall_unitary_backward_hessian, int, const cx::mat4x4*, int, const int**, const cx::quantum_circuit_cache*,
	   const cx::statevector*, cx::statevector*, cx::mat4x4*, cd*);
	const auto v = cmats(vlist, nlayers);
	CCache cc(cache);
	CState dout(dpsi_out), d(dpsi->nqubits);
	std::vector<cx::mat4x4> dv(nlayers);
	const size_t m = 16 * (size_t)nlayers;
	std::vector<cd> h(m * m);
	const int ret = cx_brickwall_unitary_backward_hessian(v.data(), nlayers, perms, &cc.c, &dout.sv, &d.sv, dv.data(),
	                                                     h.data());
	if (!ret) {
		d.to(dpsi);
		rmats(dv.data(), nlayers, dvlist);
		rvec(h.data(), m * m, hess);
	}
	return ret;
}

int apply_brickwall_unitary_gate_placeholder(const struct mat4x4 vlist[], int nlayers, const int* perms[], int l,
                                             const struct quantum_circuit_cache* cache, struct statevector_array* psi_out)
{
	CX(apply_brickwall_unitary_gate_placeholder, int, const cx::mat4x4*, int, const int**, int,
	   const cx::quantum_circuit_cache*, cx::statevector_array*);
	const auto v = cmats(vlist, nlayers);
	CCache cc(cache);
	CArray out(psi_out->nqubits, psi_out->nstates);
	const int ret = cx_apply_brickwall_unitary_gate_placeholder(v.data(), nlayers, perms, l, &cc.c, &out.a);
	if (!ret) out.to(psi_out);
	return ret;
}

// ================================================================ target.h

int circuit_unitary_target(linear_func ufunc, void* udata, const struct mat4x4 gates[], const int ngates,
                           const int wires[], const int nqubits, numeric* fval)
{
	CX(circuit_unitary_target, int, cx::linear_func, void*, const cx::mat4x4*, int, const int*, int, cd*);
	Target t(ufunc, udata);
	RealPairs pairs;
	const auto g = cmats(gates, ngates);
	cd f;
	const int ret = cx_circuit_unitary_target(t.f, t.data, g.data(), ngates, wires, nqubits, &f);
	if (!ret) *fval = f.real();
	return ret;
}

int circuit_unitary_target_sampling(linear_func ufunc, void* udata, const struct mat4x4 gates[], const int ngates,
                                    const int wires[], const int nqubits, const long nsamples, struct rng_state* rng,
                                    numeric* fval)
{
	CX(circuit_unitary_target_sampling, int, cx::linear_func, void*, const cx::mat4x4*, int, const int*, int, long,
	   struct rng_state*, cd*);
	Target t(ufunc, udata);
	const auto g = cmats(gates, ngates);
	RealSamples real;
	cd f;
	const int ret = cx_circuit_unitary_target_sampling(t.f, t.data, g.data(), ngates, wires, nqubits, nsamples, rng, &f);
	if (!ret) *fval = f.real();
	return ret;
}

int circuit_unitary_target_and_gradient(linear_func ufunc, void* udata, const struct mat4x4 gates[], const int ngates,
                                        const int wires[], const int nqubits, numeric* fval, struct mat4x4 dgates[])
{
	CX(circuit_unitary_target_and_gradient, int, cx::linear_func, void*, const cx::mat4x4*, int, const int*, int, cd*,
	   cx::mat4x4*);
	Target t(ufunc, udata);
	RealPairs pairs;
	const auto g = cmats(gates, ngates);
	std::vector<cx::mat4x4> dg(ngates);
	cd f;
	const int ret = cx_circuit_unitary_target_and_gradient(t.f, t.data, g.data(), ngates, wires, nqubits, &f, dg.data());
	if (!ret) {
		*fval = f.real();
		rmats(dg.data(), ngates, dgates);
	}
	return ret;
}

int circuit_unitary_target_and_projected_gradient(linear_func ufunc, void* udata, const struct mat4x4 gates[],
                                                  const int ngates, const int wires[], const int nqubits, numeric* fval,
                                                  double* grad_vec)
{
	CX(circuit_unitary_target_and_projected_gradient, int, cx::linear_func, void*, const cx::mat4x4*, int, const int*,
	   int, cd*, double*);
	Target t(ufunc, udata);
	RealPairs pairs;
	const auto g = cmats(gates, ngates);
	std::vector<double> g16(16 * (size_t)ngates);
	cd f;
	const int ret = cx_circuit_unitary_target_and_projected_gradient(t.f, t.data, g.data(), ngates, wires, nqubits, &f,
	                                                                 g16.data());
	if (!ret) {
		*fval = f.real();
		tangent16_to_6(g16.data(), ngates, grad_vec);
	}
	return ret;
}

int circuit_unitary_target_hessian_vector_product(linear_func ufunc, void* udata, const struct mat4x4 gates[],
                                                  const struct mat4x4 gatedirs[], const int ngates, const int wires[],
                                                  const int nqubits, numeric* fval, struct mat4x4 dgates[],
                                                  struct mat4x4 hess_gatedirs[])
{
	CX(circuit_unitary_target_hessian_vector_product, int, cx::linear_func, void*, const cx::mat4x4*, const cx::mat4x4*,
	   int, const int*, int, cd*, cx::mat4x4*, cx::mat4x4*);
	Target t(ufunc, udata);
	RealPairs pairs;
	const auto g = cmats(gates, ngates), z = cmats(gatedirs, ngates);
	std::vector<cx::mat4x4> dg(ngates), hg(ngates);
	cd f;
	const int ret = cx_circuit_unitary_target_hessian_vector_product(t.f, t.data, g.data(), z.data(), ngates, wires,
	                                                                 nqubits, &f, dg.data(), hg.data());
	if (!ret) {
		*fval = f.real();
		rmats(dg.data(), ngates, dgates);
		rmats(hg.data(), ngates, hess_gatedirs);
	}
	return ret;
}

int circuit_unitary_target_projected_hessian_vector_product(linear_func ufunc, void* udata, const struct mat4x4 gates[],
                                                            const struct mat4x4 gatedirs[], const int ngates,
                                                            const int wires[], const int nqubits, numeric* fval,
                                                            double* grad_vec, double* hvp_vec)
{
	CX(circuit_unitary_target_projected_hessian_vector_product, int, cx::linear_func, void*, const cx::mat4x4*,
	   const cx::mat4x4*, int, const int*, int, cd*, double*, double*);
	Target t(ufunc, udata);
	RealPairs pairs;
	const auto g = cmats(gates, ngates), z = cmats(gatedirs, ngates);
	std::vector<double> g16(16 * (size_t)ngates), h16(16 * (size_t)ngates);
	cd f;
	const int ret = cx_circuit_unitary_target_projected_hessian_vector_product(t.f, t.data, g.data(), z.data(), ngates,
	                                                                           wires, nqubits, &f, g16.data(), h16.data());
	if (!ret) {
		*fval = f.real();
		tangent16_to_6(g16.data(), ngates, grad_vec);
		tangent16_to_6(h16.data(), ngates, hvp_vec);
	}
	return ret;
}

int brickwall_unitary_target(linear_func ufunc, void* udata, const struct mat4x4 vlist[], const int nlayers,
                             const int nqubits, const int* perms[], numeric* fval)
{
	CX(brickwall_unitary_target, int, cx::linear_func, void*, const cx::mat4x4*, int, int, const int**, cd*);
	Target t(ufunc, udata);
	RealPairs pairs;
	const auto v = cmats(vlist, nlayers);
	cd f;
	const int ret = cx_brickwall_unitary_target(t.f, t.data, v.data(), nlayers, nqubits, perms, &f);
	if (!ret) *fval = f.real();
	return ret;
}

int brickwall_unitary_target_sampling(linear_func ufunc, void* udata, const struct mat4x4 vlist[], const int nlayers,
                                      const int nqubits, const int* perms[], const long nsamples, struct rng_state* rng,
                                      numeric* fval)
{
	CX(brickwall_unitary_target_sampling, int, cx::linear_func, void*, const cx::mat4x4*, int, int, const int**, long,
	   struct rng_state*, cd*);
	Target t(ufunc, udata);
	const auto v = cmats(vlist, nlayers);
	RealSamples real;
	cd f;
	const int ret = cx_brickwall_unitary_target_sampling(t.f, t.data, v.data(), nlayers, nqubits, perms, nsamples, rng,
	                                                     &f);
	if (!ret) *fval = f.real();
	return ret;
}

int brickwall_unitary_target_and_gradient(linear_func ufunc, void* udata, const struct mat4x4 vlist[],
                                          const int nlayers, const int nqubits, const int* perms[], numeric* fval,
                                          struct mat4x4 dvlist[])
{
	CX(brickwall_unitary_target_and_gradient, int, cx::linear_func, void*, const cx::mat4x4*, int, int, const int**,
	   cd*, cx::mat4x4*);
	Target t(ufunc, udata);
	RealPairs pairs;
	const auto v = cmats(vlist, nlayers);
	std::vector<cx::mat4x4> dv(nlayers);
	cd f;
	const int ret = cx_brickwall_unitary_target_and_gradient(t.f, t.data, v.data(), nlayers, nqubits, perms, &f, dv.data());
	if (!ret) {
		*fval = f.real();
		rmats(dv.data(), nlayers, dvlist);
	}
	return ret;
}

int brickwall_unitary_target_and_projected_gradient(linear_func ufunc, void* udata, const struct mat4x4 vlist[],
                                                    const int nlayers, const int nqubits, const int* perms[],
                                                    numeric* fval, double* grad_vec)
{
	CX(brickwall_unitary_target_and_projected_gradient, int, cx::linear_func, void*, const cx::mat4x4*, int, int,
	   const int**, cd*, double*);
	Target t(ufunc, udata);
	RealPairs pairs;
	const auto v = cmats(vlist, nlayers);
	std::vector<double> g16(16 * (size_t)nlayers);
	cd f;
	const int ret = cx_brickwall_unitary_target_and_projected_gradient(t.f, t.data, v.data(), nlayers, nqubits, perms,
	                                                                   &f, g16.data());
	if (!ret) {
		*fval = f.real();
		tangent16_to_6(g16.data(), nlayers, grad_vec);
	}
	return ret;
}

int brickwall_unitary_target_hessian_vector_product(linear_func ufunc, void* udata, const struct mat4x4 vlist[],
                                                    const struct mat4x4 vdirs[], const int nlayers, const int* perms[],
                                                    const int nqubits, numeric* fval, struct mat4x4 dvlist[],
                                                    struct mat4x4 hess_vdirs[])
{
	CX(brickwall_unitary_target_hessian_vector_product, int, cx::linear_func, void*, const cx::mat4x4*,
	   const cx::mat4x4*, int, const int**, int, cd*, cx::mat4x4*, cx::mat4x4*);
	Target t(ufunc, udata);
	RealPairs pairs;
	const auto v = cmats(vlist, nlayers), z = cmats(vdirs, nlayers);
	std::vector<cx::mat4x4> dv(nlayers), hv(nlayers);
	cd f;
	const int ret = cx_brickwall_unitary_target_hessian_vector_product(t.f, t.data, v.data(), z.data(), nlayers, perms,
	                                                                   nqubits, &f, dv.data(), hv.data());
	if (!ret) {
		*fval = f.real();
		rmats(dv.data(), nlayers, dvlist);
		rmats(hv.data(), nlayers, hess_vdirs);
	}
	return ret;
}

int brickwall_unitary_target_projected_hessian_vector_product(linear_func ufunc, void* udata,
                                                              const struct mat4x4 vlist[], const struct mat4x4 vdirs[],
                                                              const int nlayers, const int* perms[], const int nqubits,
                                                              numeric* fval, double* grad_vec, double* hvp_vec)
{
	CX(brickwall_unitary_target_projected_hessian_vector_product, int, cx::linear_func, void*, const cx::mat4x4*,
	   const cx::mat4x4*, int, const int**, int, cd*, double*, double*);
	Target t(ufunc, udata);
	RealPairs pairs;
	const auto v = cmats(vlist, nlayers), z = cmats(vdirs, nlayers);
	std::vector<double> g16(16 * (size_t)nlayers), h16(16 * (size_t)nlayers);
	cd f;
	const int ret = cx_brickwall_unitary_target_projected_hessian_vector_product(t.f, t.data, v.data(), z.data(), nlayers,
	                                                                             perms, nqubits, &f, g16.data(),
	                                                                             h16.data());
	if (!ret) {
		*fval = f.real();
		tangent16_to_6(g16.data(), nlayers, grad_vec);
		tangent16_to_6(h16.data(), nlayers, hvp_vec);
	}
	return ret;
}

int brickwall_unitary_target_gradient_hessian(linear_func ufunc, void* udata, const struct mat4x4 vlist[],
                                              const int nlayers, const int nqubits, const int* perms[], numeric* fval,
                                              struct mat4x4 dvlist[], numeric* hess)
{
	CX(brickwall_unitary_target_gradient_hessian, int, cx::linear_func, void*, const cx::mat4x4*, int, int, const int**,
	   cd*, cx::mat4x4*, cd*);
	Target t(ufunc, udata);
	const auto v = cmats(vlist, nlayers);
	std::vector<cx::mat4x4> dv(nlayers);
	const size_t m = 16 * (size_t)nlayers;
	std::vector<cd> h(m * m);
	cd f;
	const int ret = cx_brickwall_unitary_target_gradient_hessian(t.f, t.data, v.data(), nlayers, nqubits, perms, &f,
	                                                             dv.data(), h.data());
	if (!ret) {
		*fval = f.real();
		rmats(dv.data(), nlayers, dvlist);
		rvec(h.data(), m * m, hess);
	}
	return ret;
}

int brickwall_unitary_target_gradient_hessian_sampling(linear_func ufunc, void* udata, const struct mat4x4 vlist[],
                                                       const int nlayers, const int nqubits, const int* perms[],
                                                       const long nsamples, struct rng_state* rng, numeric* fval,
                                                       struct mat4x4 dvlist[], numeric* hess)
{
	CX(brickwall_unitary_target_gradient_hessian_sampling, int, cx::linear_func, void*, const cx::mat4x4*, int, int,
	   const int**, long, struct rng_state*, cd*, cx::mat4x4*, cd*);
	Target t(ufunc, udata);
	const auto v = cmats(vlist, nlayers);
	std::vector<cx::mat4x4> dv(nlayers);
	const size_t m = 16 * (size_t)nlayers;
	std::vector<cd> h(m * m);
	RealSamples real;
	cd f;
	const int ret = cx_brickwall_unitary_target_gradient_hessian_sampling(t.f, t.data, v.data(), nlayers, nqubits, perms,
	                                                                      nsamples, rng, &f, dv.data(), h.data());
	if (!ret) {
		*fval = f.real();
		rmats(dv.data(), nlayers, dvlist);
		rvec(h.data(), m * m, hess);
	}
	return ret;
}

int brickwall_blockenc_target(linear_func hfunc, void* hdata, const struct mat4x4 vlist[], const int nlayers,
                              const int nqubits, const int* perms[], double* fval)
{
	CX(brickwall_blockenc_target, int, cx::linear_func, void*, const cx::mat4x4*, int, int, const int**, double*);
	Target t(hfunc, hdata);
	const auto v = cmats(vlist, nlayers);
	return cx_brickwall_blockenc_target(t.f, t.data, v.data(), nlayers, nqubits, perms, fval);
}

int brickwall_blockenc_target_and_gradient(linear_func hfunc, void* hdata, const struct mat4x4 vlist[],
                                           const int nlayers, const int nqubits, const int* perms[], double* fval,
                                           struct mat4x4 dvlist[])
{
	CX(brickwall_blockenc_target_and_gradient, int, cx::linear_func, void*, const cx::mat4x4*, int, int, const int**,
	   double*, cx::mat4x4*);
	Target t(hfunc, hdata);
	const auto v = cmats(vlist, nlayers);
	std::vector<cx::mat4x4> dv(nlayers);
	const int ret = cx_brickwall_blockenc_target_and_gradient(t.f, t.data, v.data(), nlayers, nqubits, perms, fval,
	                                                          dv.data());
	if (!ret) rmats(dv.data(), nlayers, dvlist);
	return ret;
}

int brickwall_blockenc_target_gradient_hessian(linear_func hfunc, void* hdata, const struct mat4x4 vlist[],
                                               const int nlayers, const int nqubits, const int* perms[], double* fval,
                                               struct mat4x4 dvlist[], numeric* hess)
{
	CX(brickwall_blockenc_target_gradient_hessian, int, cx::linear_func, void*, const cx::mat4x4*, int, int,
	   const int**, double*, cx::mat4x4*, cd*, cd*);
	Target t(hfunc, hdata);
	const auto v = cmats(vlist, nlayers);
	std::vector<cx::mat4x4> dv(nlayers);
	const size_t m = 16 * (size_t)nlayers;
	std::vector<cd> h1(m * m), h2(m * m);
	const int ret = cx_brickwall_blockenc_target_gradient_hessian(t.f, t.data, v.data(), nlayers, nqubits, perms, fval,
	                                                              dv.data(), h1.data(), h2.data());
	if (!ret) {
		rmats(dv.data(), nlayers, dvlist);
		for (size_t k = 0; k < m * m; k++) hess[k] = h1[k].real() + h2[k].real();
	}
	return ret;
}

// ================================================================ trust_region.h (no numeric types: forwarded)

bool truncated_cg_hmat(const double* grad, const double* hess, int n, double radius,
                       const struct truncated_cg_params* params, double* z)
{
	CX(truncated_cg_hmat, bool, const double*, const double*, int, double, const struct truncated_cg_params*, double*);
	return cx_truncated_cg_hmat(grad, hess, n, radius, params, z);
}

bool truncated_cg_hvp(const double* x, const double* grad, const hessian_vector_product_func f_hvp, void* fdata,
                      const int n, const double radius, const struct truncated_cg_params* params, double* z)
{
	CX(truncated_cg_hvp, bool, const double*, const double*, hessian_vector_product_func, void*, int, double,
	   const struct truncated_cg_params*, double*);
	return cx_truncated_cg_hvp(x, grad, f_hvp, fdata, n, radius, params, z);
}

void riemannian_trust_region_optimize_hmat(target_func f, target_gradient_hessian_func f_deriv_hess, void* fdata,
                                           retract_func retract, void* rdata, const int n, const double* x_init,
                                           const int m, const struct rtr_params* params, const int niter,
                                           double* f_iter, double* x_final)
{
	g_error = 0;
	CX(riemannian_trust_region_optimize_hmat, void, target_func, target_gradient_hessian_func, void*, retract_func,
	   void*, int, const double*, int, const struct rtr_params*, int, double*, double*);
	cx_riemannian_trust_region_optimize_hmat(f, f_deriv_hess, fdata, retract, rdata, n, x_init, m, params, niter, f_iter,
	                                         x_final);
}

void riemannian_trust_region_optimize_hvp(const target_func f, const target_gradient_func f_deriv,
                                          const hessian_vector_product_func f_hvp, void* fdata, retract_func retract,
                                          void* rdata, const int n, const double* x_init, const int m,
                                          const struct rtr_params* params, const int niter, double* f_iter,
                                          double* x_final)
{
	g_error = 0;
	CX(riemannian_trust_region_optimize_hvp, void, target_func, target_gradient_func, hessian_vector_product_func,
	   void*, retract_func, void*, int, const double*, int, const struct rtr_params*, int, double*, double*);
	cx_riemannian_trust_region_optimize_hvp(f, f_deriv, f_hvp, fdata, retract, rdata, n, x_init, m, params, niter,
	                                        f_iter, x_final);
}

// ================================================================ brickwall_opt.h, circuit_opt.h

}  // extern "C"

namespace {

// the optimiser wrappers of src/brickwall_opt.c:22-119 and src/circuit_opt.c, real build
struct OptData
{
	linear_func ufunc;
	void* udata;
	const int** perms;    // brickwall
	const int* wires;     // circuit
	int n;                // nlayers or ngates
	int nqubits;
	int failed;
};

double bw_f(const double* x, void* d)
{
	auto* o = static_cast<OptData*>(d);
	numeric f;
	if (brickwall_unitary_target(o->ufunc, o->udata, reinterpret_cast<const mat4x4*>(x), o->n, o->nqubits, o->perms, &f) < 0) {
		fprintf(stderr, "target function evaluation failed internally\n");
		o->failed = 1;
		return -1;
	}
	return f;
}

double bw_fd(const double* x, void* d, double* grad)
{
	auto* o = static_cast<OptData*>(d);
	numeric f;
	if (brickwall_unitary_target_and_projected_gradient(o->ufunc, o->udata, reinterpret_cast<const mat4x4*>(x), o->n,
	                                                    o->nqubits, o->perms, &f, grad) < 0) {
		fprintf(stderr, "target function and derivative evaluation failed internally\n");
		o->failed = 1;
		return -1;
	}
	return f;
}

void bw_hvp(const double* x, void* d, double* vec, double* hvp)
{
	auto* o = static_cast<OptData*>(d);
	const mat4x4* vlist = reinterpret_cast<const mat4x4*>(x);
	std::vector<mat4x4> vdirs(o->n);
	for (int i = 0; i < o->n; i++) real_to_tangent(&vec[6 * i], &vlist[i], &vdirs[i]);
	std::vector<double> grad(6 * (size_t)o->n);
	numeric f;
	if (brickwall_unitary_target_projected_hessian_vector_product(o->ufunc, o->udata, vlist, vdirs.data(), o->n, o->perms,
	                                                              o->nqubits, &f, grad.data(), hvp) < 0)
		o->failed = 1;
}

double qc_f(const double* x, void* d)
{
	auto* o = static_cast<OptData*>(d);
	numeric f;
	if (circuit_unitary_target(o->ufunc, o->udata, reinterpret_cast<const mat4x4*>(x), o->n, o->wires, o->nqubits, &f) < 0) {
		fprintf(stderr, "target function evaluation failed internally\n");
		o->failed = 1;
		return -1;
	}
	return f;
}

double qc_fd(const double* x, void* d, double* grad)
{
	auto* o = static_cast<OptData*>(d);
	numeric f;
	if (circuit_unitary_target_and_projected_gradient(o->ufunc, o->udata, reinterpret_cast<const mat4x4*>(x), o->n,
	                                                  o->wires, o->nqubits, &f, grad) < 0) {
		fprintf(stderr, "target function and derivative evaluation failed internally\n");
		o->failed = 1;
		return -1;
	}
	return f;
}

void qc_hvp(const double* x, void* d, double* vec, double* hvp)
{
	auto* o = static_cast<OptData*>(d);
	const mat4x4* gates = reinterpret_cast<const mat4x4*>(x);
	std::vector<mat4x4> dirs(o->n);
	for (int i = 0; i < o->n; i++) real_to_tangent(&vec[6 * i], &gates[i], &dirs[i]);
	std::vector<double> grad(6 * (size_t)o->n);
	numeric f;
	if (circuit_unitary_target_projected_hessian_vector_product(o->ufunc, o->udata, gates, dirs.data(), o->n, o->wires,
	                                                            o->nqubits, &f, grad.data(), hvp) < 0)
		o->failed = 1;
}

void retract_list(const double* x, const double* eta, void* rdata, double* xs)
{
	const int n = *static_cast<int*>(rdata);
	const mat4x4* v = reinterpret_cast<const mat4x4*>(x);
	mat4x4* w = reinterpret_cast<mat4x4*>(xs);
	for (int i = 0; i < n; i++) retract(&v[i], &eta[6 * i], &w[i]);
}

}  // namespace

extern "C" {

void optimize_brickwall_circuit_hvp(linear_func ufunc, void* udata, const struct mat4x4 vlist_start[], const int nlayers,
                                    const int nqubits, const int* perms[], struct rtr_params* params, const int niter,
                                    double* f_iter, struct mat4x4 vlist_opt[])
{
	g_error = 0;
	OptData d{ ufunc, udata, perms, nullptr, nlayers, nqubits, 0 };
	params->g_func = nullptr;
	params->g_data = nullptr;
	params->g_iter = nullptr;
	int rdata = nlayers;
	riemannian_trust_region_optimize_hvp(bw_f, bw_fd, bw_hvp, &d, retract_list, &rdata, 6 * nlayers,
	                                     reinterpret_cast<const double*>(vlist_start), 16 * nlayers, params, niter, f_iter,
	                                     reinterpret_cast<double*>(vlist_opt));
	if (d.failed && !g_error) g_error = -3;
}

void optimize_quantum_circuit(linear_func ufunc, void* udata, const struct mat4x4 gates_start[], const int ngates,
                              const int nqubits, const int wires[], struct rtr_params* params, const int niter,
                              double* f_iter, struct mat4x4 gates_opt[])
{
	g_error = 0;
	OptData d{ ufunc, udata, nullptr, wires, ngates, nqubits, 0 };
	params->g_func = nullptr;
	params->g_data = nullptr;
	params->g_iter = nullptr;
	int rdata = ngates;
	riemannian_trust_region_optimize_hvp(qc_f, qc_fd, qc_hvp, &d, retract_list, &rdata, 6 * ngates,
	                                     reinterpret_cast<const double*>(gates_start), 16 * ngates, params, niter, f_iter,
	                                     reinterpret_cast<double*>(gates_opt));
	if (d.failed && !g_error) g_error = -3;
}

// ================================================================ matrix.h (real build)

void zero_matrix(struct mat4x4* a) { std::memset(a->data, 0, sizeof(a->data)); }

void identity_matrix(struct mat4x4* a)
{
	zero_matrix(a);
	for (int i = 0; i < 4; i++) a->data[5 * i] = 1;
}

void scale_matrix(struct mat4x4* a, const double x)
{
	for (int i = 0; i < 16; i++) a->data[i] *= x;
}

void conjugate_matrix(struct mat4x4* a) { (void)a; }

void add_matrix(struct mat4x4* a, const struct mat4x4* b)
{
	for (int i = 0; i < 16; i++) a->data[i] += b->data[i];
}

void sub_matrix(struct mat4x4* a, const struct mat4x4* b)
{
	for (int i = 0; i < 16; i++) a->data[i] -= b->data[i];
}

void add_matrices(const struct mat4x4* a, const struct mat4x4* b, struct mat4x4* c)
{
	for (int i = 0; i < 16; i++) c->data[i] = a->data[i] + b->data[i];
}

void sub_matrices(const struct mat4x4* a, const struct mat4x4* b, struct mat4x4* c)
{
	for (int i = 0; i < 16; i++) c->data[i] = a->data[i] - b->data[i];
}

void transpose(const struct mat4x4* a, struct mat4x4* at)
{
	for (int i = 0; i < 4; i++)
		for (int j = 0; j < 4; j++) at->data[4 * j + i] = a->data[4 * i + j];
}

void adjoint(const struct mat4x4* a, struct mat4x4* ah) { transpose(a, ah); }

void symm(const struct mat4x4* w, struct mat4x4* z)
{
	for (int i = 0; i < 4; i++)
		for (int j = 0; j < 4; j++) z->data[4 * i + j] = 0.5 * (w->data[4 * i + j] + w->data[4 * j + i]);
}

void antisymm(const struct mat4x4* w, struct mat4x4* z)
{
	for (int i = 0; i < 4; i++)
		for (int j = 0; j < 4; j++) z->data[4 * i + j] = i == j ? 0.0 : 0.5 * (w->data[4 * i + j] - w->data[4 * j + i]);
}

// 6 parameters <-> real antisymmetric matrix, isometric (src/matrix.c:245-271, 288-300)
void real_to_antisymm(const double* r, struct mat4x4* w)
{
	const double s = 1.0 / std::sqrt(2.0);
	zero_matrix(w);
	for (int k = 0; k < 6; k++) {
		const int e = UPPER[k], i = e / 4, j = e % 4;
		w->data[e] = s * r[k];
		w->data[4 * j + i] = -w->data[e];
	}
}

void antisymm_to_real(const struct mat4x4* w, double* r)
{
	const double s = std::sqrt(2.0);
	for (int k = 0; k < 6; k++) r[k] = s * w->data[UPPER[k]];
}

void multiply_matrices(const struct mat4x4* a, const struct mat4x4* b, struct mat4x4* c) { mat_mul(a, b, c); }

void real_to_tangent(const double* r, const struct mat4x4* v, struct mat4x4* z)
{
	mat4x4 a;
	real_to_antisymm(r, &a);
	mat_mul(v, &a, z);
}

void tangent_to_real(const struct mat4x4* v, const struct mat4x4* z, double* r)
{
	mat4x4 w, t;
	transpose(v, &w);
	mat_mul(&w, z, &t);
	antisymm(&t, &w);
	antisymm_to_real(&w, r);
}

void project_tangent(const struct mat4x4* u, const struct mat4x4* z, struct mat4x4* p)
{
	mat4x4 v, w;
	transpose(u, &v);
	mat_mul(&v, z, &w);
	symm(&w, &v);
	mat_mul(u, &v, &w);
	sub_matrices(z, &w, p);
}

void symmetric_triple_matrix_product(const struct mat4x4* a, const struct mat4x4* b, const struct mat4x4* c,
                                     struct mat4x4* ret)
{
	g_error = 0;
	CX(symmetric_triple_matrix_product, void, const cx::mat4x4*, const cx::mat4x4*, const cx::mat4x4*, cx::mat4x4*);
	const cx::mat4x4 ca = cmat(a), cb = cmat(b), cc = cmat(c);
	cx::mat4x4 r;
	cx_symmetric_triple_matrix_product(&ca, &cb, &cc, &r);
	rmats(&r, 1, ret);
}

int inverse_matrix(const struct mat4x4* a, struct mat4x4* ainv)
{
	CX(inverse_matrix, int, const cx::mat4x4*, cx::mat4x4*);
	const cx::mat4x4 ca = cmat(a);
	cx::mat4x4 r;
	const int ret = cx_inverse_matrix(&ca, &r);
	rmats(&r, 1, ainv);
	return ret;
}

void polar_factor(const struct mat4x4* a, struct mat4x4* u)
{
	g_error = 0;
	CX(polar_factor, void, const cx::mat4x4*, cx::mat4x4*);
	const cx::mat4x4 ca = cmat(a);
	cx::mat4x4 r;
	cx_polar_factor(&ca, &r);
	rmats(&r, 1, u);
}

void retract(const struct mat4x4* u, const double* eta, struct mat4x4* v)
{
	mat4x4 z, w;
	real_to_antisymm(eta, &z);
	for (int i = 0; i < 4; i++) z.data[5 * i] += 1;
	mat_mul(u, &z, &w);
	polar_factor(&w, v);
}

// ================================================================ util.h

double uniform_distance_real(long n, const double* x, const double* y)
{
	double d = 0;
	for (long i = 0; i < n; i++) d = std::fmax(d, std::fabs(x[i] - y[i]));
	return d;
}

double uniform_distance(long n, const numeric* x, const numeric* y) { return uniform_distance_real(n, x, y); }

// maximum element-wise |x - y| / max(|x| + |y|, eps) (src/util.h:12-15, src/util.c:40-49)
double relative_distance(long n, const numeric* x, const numeric* y, double eps)
{
	double d = 0;
	for (long i = 0; i < n; i++) d = std::fmax(d, std::fabs(x[i] - y[i]) / std::fmax(std::fabs(x[i]) + std::fabs(y[i]), eps));
	return d;
}

// ================================================================ additions

int rqcopt_brickwall_ufunc(const struct statevector* psi, void* udata, struct statevector* psi_out)
{
	const auto* t = static_cast<const rqcopt_brickwall_target*>(udata);
	return apply_brickwall_unitary(t->vlist, t->nlayers, const_cast<const int**>(t->perms), psi, psi_out);
}

int rqcopt_circuit_ufunc(const struct statevector* psi, void* udata, struct statevector* psi_out)
{
	const auto* t = static_cast<const rqcopt_circuit_target*>(udata);
	return apply_quantum_circuit(t->gates, t->ngates, t->wires, psi, psi_out);
}

int rqcopt_dense_ufunc(const struct statevector* psi, void* udata, struct statevector* psi_out)
{
	const auto* t = static_cast<const rqcopt_dense_target*>(udata);
	if (psi->nqubits != t->nqubits || psi_out->nqubits != t->nqubits) return E_ARG;
	const size_t n = dim(t->nqubits);
	for (size_t i = 0; i < n; i++) {
		double s = 0;
		for (size_t j = 0; j < n; j++) s += t->u[i * n + j] * psi->data[j];
		psi_out->data[i] = s;
	}
	return 0;
}

int rqcopt_gpu_set_precision(int precision)
{
	CX(rqcopt_gpu_set_precision, int, int);
	return cx_rqcopt_gpu_set_precision(precision);
}

int rqcopt_gpu_last_error(void)
{
	const int local = g_error;
	g_error = 0;
	static const auto cx_last = sym<int (*)(void)>("rqcopt_gpu_last_error");
	const int remote = cx_last ? cx_last() : E_CUDA;
	return local ? local : remote;
}

unsigned long long rqcopt_gpu_launch_count(void)
{
	static const auto f = sym<unsigned long long (*)(void)>("rqcopt_gpu_launch_count");
	return f ? f() : 0;
}

void rqcopt_gpu_reset_launch_count(void)
{
	static const auto f = sym<void (*)(void)>("rqcopt_gpu_reset_launch_count");
	if (f) f();
}

}  // extern "C"
