"""Benchmark: grad+HVP evaluations per second of the matrix-free brickwall objective.

Workload (default): L=16 qubits, periodic brickwall of depth 9 (Haar gates,
seed 10) against a matrix-free depth-5 brickwall target (seed 11); one step is
one f + projected gradient + projected Hessian-vector product evaluation summed
over all 65,536 basis columns (random tangent direction, seed 12).  Inputs are
seeded synthetic data; the working set is many GB, far larger than L2.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision mixed|c64|c128] [--L 16 --depth 9 --tdepth 5]

The default arm is the mixed-precision evaluation (complex64 passes on the tensor
cores with FP64 sums); the same run times the plain complex128 evaluation, reports
the error of one against the other, and runs a short trust-region optimisation in
both modes to compare time at equal final error.

One JSON line on rank 0.  `value` is device-timed throughput with the inputs
resident in HBM (CUDA events on the library stream); `e2e` is the same metric
through the C ABI with host buffers (gates in, gradient and HVP out).  With
N > 1 (torchrun) every rank evaluates its own replica (no collective on the
data path); throughput is the sum over ranks divided by the slowest rank's time.
`--impl reference` times the reference's C implementation (oracle/_ref) on the
host cores on a bounded column sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

# DRAM traffic / algorithmic bytes of the reverse-pass kernel, from ncu
# (complex64 k5_rev: 541.2 + 312.7 MB measured for 805.3 MB algorithmic at L=12)
TRAFFIC_RATIO = {8: 1.060}

METRIC = "grad+HVP evals/s (f + projected gradient + projected HVP, all basis columns; mixed vs FP64)"


from rqcopt_hpc_b200.workloads import haar, perms_for  # noqa: E402


def antisymm(r):
    w = np.zeros((4, 4), np.complex128)
    for a in range(4):
        w[a, a] = 1j * r[5 * a]
        for c in range(a + 1, 4):
            p, q = r[4 * a + c], r[4 * c + a]
            w[a, c] = 0.5 * (p - q) + 0.5j * (p + q)
            w[c, a] = -np.conj(w[a, c])
    return w


def workload(L, depth, tdepth, seed=10, tseed=11, dseed=12):
    rng = np.random.default_rng(seed)
    vlist = np.stack([haar(rng) for _ in range(depth)])
    trng = np.random.default_rng(tseed)
    tvlist = np.stack([haar(trng) for _ in range(tdepth)])
    r = np.random.default_rng(dseed).standard_normal((depth, 16))
    vdirs = np.stack([vlist[k] @ antisymm(r[k]) for k in range(depth)])
    return vlist, perms_for(L, depth), tvlist, perms_for(L, tdepth), vdirs


def flops_per_eval(L, G, Gt):
    """Algorithmic flops of one evaluation as the reference executes it:
    N^2 (32 G_t + 292 G - 124) (N = 2^L basis columns of 2^L amplitudes)."""
    N = 1 << L
    return float(N) * N * (32 * Gt + 292 * G - 124)


def reverse_flops_per_eval(L, G):
    """Algorithmic flops of the reverse (gradient/HVP) passes of one evaluation as the
    reference executes them: per gate and amplitude of each of the N = 2^L columns, the
    outer sums dG += phi (x) psi and HZ += phi (x) dpsi + dphi (x) psi and the adjoint
    updates phi' = G^T phi, dphi' = G^T dphi + Z^T phi: six 4x4 complex products of an
    amplitude group, 6 x 32 = 192 flop per amplitude (states rebuilt inside a fused pass
    are not counted)."""
    N = 1 << L
    return 192.0 * G * N * N


def reverse_bytes_per_eval(L, P, itemsize):
    """Algorithmic HBM bytes of the reverse (gradient/HVP) passes of one evaluation with P
    passes (one per gate, or one per group of fused gates): per column 6P - 5 statevector
    passes (reads of phi, dphi, psi, dpsi and writes of phi', dphi' per pass; the pass at the
    circuit output has no dphi to read, the pass at its input no psi / outputs)."""
    N = 1 << L
    return float(6 * P - 5) * N * N * itemsize


# ----------------------------------------------------------------------------- clocks

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


# ----------------------------------------------------------------------------- arithmetic peaks

def measure_fp_peaks(torch, n=8192, reps=5):
    """Dense FP64 and FP32 throughput of this GPU, measured here the way the bf16 figure of
    MEASURED_PEAKS.json is measured: cuBLAS GEMMs (torch.matmul) of n x n x n, float64 and
    float32 with TF32 off, best of `reps` (2 n^3 flop each), CUDA events."""
    out = {}
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        for name, dt in (("fp64_tflops", torch.float64), ("fp32_tflops", torch.float32)):
            a = torch.randn(n, n, dtype=dt, device="cuda")
            b = torch.randn(n, n, dtype=dt, device="cuda")
            c = torch.matmul(a, b)
            best = None
            for _ in range(reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                torch.matmul(a, b, out=c)
                e1.record()
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1)
                best = ms if best is None else min(best, ms)
            out[name] = 2.0 * n ** 3 / (best * 1e-3) / 1e12
            del a, b, c
        torch.cuda.empty_cache()
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    out["how"] = (f"torch.matmul {n}^3 (cuBLAS DGEMM / SGEMM with TF32 off), best of {reps}, 2 n^3 flop, CUDA events, "
                  "measured in this run")
    return out


# ----------------------------------------------------------------------------- CPU baseline

def _ref_columns_worker(args):
    L, depth, tdepth, b0, b1 = args
    from oracle.oracle import Reference
    vlist, perms, tvlist, tperms, vdirs = workload(L, depth, tdepth)
    t0 = time.perf_counter()
    Reference().brickwall_hvp_columns(vlist, vdirs, perms, L, tvlist, tperms, b0, b1)
    return time.perf_counter() - t0


def cpu_baseline(L, depth, tdepth, seconds=15.0, cores=None):
    """Reference C implementation (oracle/_ref, per-column grad+HVP function of the
    column loop) on a bounded contiguous column sample, one process per core (spawn)."""
    import multiprocessing as mp
    from oracle.oracle import Reference
    if not Reference.available():
        return None
    cores = cores or os.cpu_count() or 1
    N = 1 << L
    # calibrate: time one column on this process
    vlist, perms, tvlist, tperms, vdirs = workload(L, depth, tdepth)
    t0 = time.perf_counter()
    Reference().brickwall_hvp_columns(vlist, vdirs, perms, L, tvlist, tperms, 0, 1)
    per_col = max(time.perf_counter() - t0, 1e-6)
    cols_per_core = max(1, min(N // cores, int(seconds / per_col)))
    jobs = [(L, depth, tdepth, k * cols_per_core, (k + 1) * cols_per_core) for k in range(cores)]
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(cores) as pool:
        pool.map(_ref_columns_worker, jobs)
    wall = time.perf_counter() - t0
    cols = cols_per_core * cores
    return {"value": (cols / N) / wall, "unit": "evals/s", "cores": cores, "kind": "reference",
            "sample": f"{cols} of {N} basis columns ({cols_per_core} per core) through the reference's "
                      f"quantum_circuit_gates_hessian_vector_product with its brickwall target, "
                      f"{wall:.1f} s wall; evals/s = sampled fraction / wall time"}


# ----------------------------------------------------------------------------- gate throughput

def gate_throughput(gpu, torch, L=28, G=256, seed=20):
    """Forward through G Haar gates on uniformly random distinct qubit pairs, then the
    adjoint gates in reverse order, on one L-qubit state resident in HBM (complex128,
    then complex64), with 1 and with 4 gates per HBM round trip; DRAM GB/s counts one
    read and one write of the state per round trip."""
    import ctypes
    from rqcopt_hpc_b200.abi import Statevector
    rng = np.random.default_rng(seed)
    gates = np.stack([haar(rng) for _ in range(G)])
    wires = np.array([rng.choice(L, 2, replace=False) for _ in range(G)], np.int32)
    adj = np.ascontiguousarray(np.conj(np.transpose(gates[::-1], (0, 2, 1))))
    wires_rev = np.ascontiguousarray(wires[::-1])
    lib = gpu.lib()
    stream = torch.cuda.ExternalStream(lib.rqcopt_gpu_stream())
    res = {"workload": f"one L={L} state, {G} Haar gates on random distinct pairs, forward then adjoint backward"}
    for dtype, name, tol in ((torch.complex128, "c128", 1e-12), (torch.complex64, "c64", 1e-5)):
        gen = torch.Generator(device="cuda").manual_seed(seed)
        psi = torch.randn(1 << L, dtype=dtype, device="cuda", generator=gen)
        psi /= torch.linalg.vector_norm(psi)
        out, back = torch.empty_like(psi), torch.empty_like(psi)
        state_bytes = (1 << L) * psi.element_size()
        if name == "c128":
            sv = lambda t: ctypes.byref(Statevector(t.data_ptr(), L))
            run = lambda g, w, a, b: lib.apply_quantum_circuit(g.ctypes.data, G, w.ctypes.data, sv(a), sv(b))
        else:
            run = lambda g, w, a, b: lib.rqcopt_apply_quantum_circuit_c64(g.ctypes.data, G, w.ctypes.data, a.data_ptr(),
                                                                          b.data_ptr(), L)
        r = {"state_gib": state_bytes / 2 ** 30, "recovery_tolerance": tol}
        for gpp in (1, 4):
            gpu.set_gates_per_pass(gpp)
            run(gates, wires, psi, out)   # warm-up
            torch.cuda.synchronize()
            e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            e[0].record(stream)
            run(gates, wires, psi, out)
            e[1].record(stream)
            run(adj, wires_rev, out, back)
            e[2].record(stream)
            torch.cuda.synchronize()
            t_f, t_b = e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2])
            trips = G if gpp == 1 else -(-G // gpp)
            err = float(torch.max(torch.abs(back - psi)))
            r[f"gates_per_round_trip_{gpp}"] = {
                "forward_ms": t_f, "backward_ms": t_b, "round_trips": trips,
                "dram_gbs": 2 * trips * 2 * state_bytes / ((t_f + t_b) * 1e-3) / 1e9,
                "gate_equivalent_gbs": 2 * G * 2 * state_bytes / ((t_f + t_b) * 1e-3) / 1e9,
                "recovery_max_abs_err": err, "recovered": err <= tol}
        res[name] = r
        del psi, out, back
        torch.cuda.empty_cache()
    gpu.set_autotune(True)
    return res


# ----------------------------------------------------------------------------- full-Hessian path

def hess_model(L, nlayers, single):
    """Algorithmic HBM transfers (state-sized reads + writes) and complex multiply-adds
    per basis column of the full-Hessian sweep kernels of one evaluation.

    L <= 12 runs k_hlayer, one launch per layer with the tangents' column tiles in
    shared memory: per layer a the tangents of the earlier layers (16 a) are read once
    and all 16 (a + 1) written once (not after the last layer), phi_q and psi_q of the
    layer's gates are read once (psi_0 of a basis column is generated).  Larger L runs
    k_hsweep, one launch per gate: per gate q of layer a, phi_q is read, the tangents of
    the earlier layers are read and written, the 16 tangents of layer a are read (not
    at the layer's first gate) and written (not at the last gate), and psi_q is read
    (and, in target sums, the next psi written).  Complex multiply-adds: 16 for the
    contraction with phi_q and 16 for G_q per group of 4 amplitudes and active state."""
    per = L // 2
    G = nlayers * per
    layered = L <= 12
    transfers = 0
    cmacs = 0
    for q in range(G):
        a, pos = divmod(q, per)
        last = q == G - 1
        # multiply-adds: psi (contraction, G at the last gate), earlier layers, own layer
        cmacs += 16 + (16 if last else 0)
        cmacs += 16 * a * (16 + (0 if last else 16))
        cmacs += 0 if pos == 0 else 16 * (16 + (0 if last else 16))
        if layered:
            continue
        t_read = 16 * a + (0 if pos == 0 else 16)
        t_write = 0 if last else 16 * (a + 1)
        psi = 1 if single else (1 if q > 0 else 0) + (0 if last else 1)
        transfers += 1 + psi + t_read + t_write
    if layered:
        for a in range(nlayers):
            transfers += 16 * a + (16 * (a + 1) if a < nlayers - 1 else 0) + per + per
        if not single:
            transfers -= 1          # psi_0 is the basis column
    groups = (1 << L) // 4
    return {"kernel": ("k_hlayer (one brickwall layer of the full-Hessian tangent sweep, column tiles in shared memory)"
                       if layered else "k_hsweep (one gate of the full-Hessian tangent sweep)"),
            "launches": nlayers if layered else G, "transfers": transfers, "cmacs": cmacs * groups}


def _ref_hessian_worker(args):
    L, depth, tdepth, b0, b1 = args
    from oracle.oracle import Reference
    vlist, perms, tvlist, tperms, _ = workload(L, depth, tdepth)
    t0 = time.perf_counter()
    Reference().hessian_columns(vlist, perms, L, tvlist, tperms, b0, b1)
    return time.perf_counter() - t0


def _ref_sampling_worker(args):
    L, depth, tdepth, seed = args
    from oracle.oracle import Reference
    r = Reference()
    vlist, perms, tvlist, tperms, _ = workload(L, depth, tdepth)
    rng = r.seed_rng_state(seed)
    t0 = time.perf_counter()
    r.sampling(2, vlist, perms, L, (tvlist, tperms), 1, rng)
    return time.perf_counter() - t0


def _benc_case(L, depth, hdepth):
    """Block-encoding workload: brickwall gates seed 10, H a brickwall of depth hdepth on L/2
    qubits (seed 11)."""
    vlist, perms, _, _, _ = workload(L, depth, 1)
    hv, hp, _, _, _ = workload(L // 2, hdepth, 1, seed=11)
    return vlist, perms, hv, hp


def _ref_blockenc_worker(args):
    L, depth, hdepth, b0, b1 = args
    from oracle.oracle import Reference
    vlist, perms, hv, hp = _benc_case(L, depth, hdepth)
    t0 = time.perf_counter()
    Reference().blockenc_hessian_columns(vlist, perms, L, hv, hp, b0, b1)
    return time.perf_counter() - t0


def hmat_path(gpu, torch, stream, hbm_peak, with_reference=True, steps=3, fp64_peak=None):
    """Full-Hessian ("hmat") path.  (1) The reference's own Hessian benchmark
    (examples/benchmark/benchmark_16_qubits.c): brickwall_unitary_forward plus
    brickwall_unitary_backward_hessian of one L=16 state through 8 layers.
    (2) f + gradient vector + real Hessian matrix of the brickwall target summed over
    all basis columns (brickwall_unitary_target_gradient_vector_hessian_matrix) at
    L=8 depth 5 and L=12 depth 9.  (3) optimize_brickwall_circuit_hmat at L=8 depth 5.
    GPU numbers go through the C ABI with host buffers (e2e) and, per kernel, CUDA
    events on the library stream; the reference's C code runs on the host cores."""
    import multiprocessing as mp
    from rqcopt_hpc_b200.workloads import perms_for as pf
    from oracle.oracle import Reference
    have_ref = with_reference and Reference.available()
    out = {}

    def timed(fn, n):
        gpu.enable_kernel_timing(True)
        gpu.reset_launch_count()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(stream)
        for _ in range(n):
            r = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        wall = (time.perf_counter() - t0) / n
        hs_ms, hs_n = gpu.kernel_time(gpu.KC_HESS)
        gpu.enable_kernel_timing(False)
        return r, wall, e0.elapsed_time(e1) / n, hs_ms / n, hs_n // n, gpu.launch_count() // n

    def roofline(model, columns, L, ms, launches):
        """HBM roofline for the per-gate sweep; the layer kernel moves ~L/2 times fewer
        bytes and is bound by FP64 arithmetic instead, against the FP64 peak measured in
        this run (cuBLAS DGEMM), or the nominal 37 TFLOP/s of B200 where none was measured."""
        state_bytes = columns * (16 << L)
        per_launch = model["transfers"] * state_bytes / launches
        gbs = per_launch / (ms / launches * 1e-3) / 1e9
        tflops = 8.0 * model["cmacs"] * columns / (ms * 1e-3) / 1e12
        out = {"kernel": model["kernel"], "avg_launch_ms": ms / launches, "launches": launches,
               "bytes_per_launch": per_launch,
               "bytes_model": "algorithmic state transfers of the sweep (bench.hess_model) x columns x 2^L x 16 B",
               "hbm_gbs": gbs, "hbm_frac": gbs / hbm_peak, "fp64_tflops": tflops}
        if "k_hlayer" in model["kernel"]:
            pk = fp64_peak or 37.0
            out.update({"bound": "tensor", "achieved": tflops, "peak": pk, "unit": "TFLOP/s", "frac": tflops / pk,
                        "peak_source": "FP64 peak measured in this run (cuBLAS DGEMM 8192^3)" if fp64_peak
                        else "nominal B200 FP64"})
        else:
            out.update({"bound": "hbm", "achieved": gbs, "peak": hbm_peak, "unit": "GB/s", "frac": gbs / hbm_peak,
                        "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)"})
        return out

    # GPU legs first, the reference's CPU legs after them (no CPU load during GPU timing)
    # (1) single state, L = 16, 8 layers
    L, nl = 16, 8
    rng = np.random.default_rng(16)
    vlist = np.stack([haar(rng) for _ in range(nl)])
    perms = pf(L, nl)
    psi = (rng.standard_normal(1 << L) + 1j * rng.standard_normal(1 << L)) / np.sqrt(2 << L)
    dout = (rng.standard_normal(1 << L) + 1j * rng.standard_normal(1 << L)) / np.sqrt(2 << L)
    cache = gpu.Cache(L, nl * (L // 2))

    def single():
        gpu.brickwall_unitary_forward(vlist, perms, psi, cache)
        return gpu.brickwall_unitary_backward_hessian(vlist, perms, cache, dout)

    for _ in range(2):
        single()
    (dpsi, dv, hess), wall, dev_ms, hs_ms, hs_n, launches = timed(single, steps)
    r1 = {"workload": "brickwall_unitary_forward + brickwall_unitary_backward_hessian, one L=16 state, 8 layers "
                      "(examples/benchmark/benchmark_16_qubits.c)",
          "e2e_ms": wall * 1e3, "device_ms": dev_ms, "sweep_ms": hs_ms, "gpu_launches": launches,
          "roofline": roofline(hess_model(L, nl, True), 1, L, hs_ms, hs_n)}
    single_case = (vlist, perms, psi, dout, dpsi, dv, hess, wall)
    out["single_state_L16"] = r1
    del cache

    # (2) target sums
    target_cases = []
    for L, depth, tdepth, seed, tseed in [(8, 5, 3, 0, 1), (12, 9, 5, 10, 11)]:
        vlist, perms, tvlist, tperms, _ = workload(L, depth, tdepth, seed, tseed)
        tg = gpu.Target(brickwall=(tvlist, tperms))

        def target():
            return gpu.brickwall_unitary_target_gradient_vector_hessian_matrix(tg, vlist, perms, L)

        target()
        (f, g, H), wall, dev_ms, hs_ms, hs_n, launches = timed(target, steps)
        N = 1 << L
        r2 = {"workload": f"f + gradient vector + Hessian matrix, brickwall L={L} depth {depth} vs brickwall target "
                          f"depth {tdepth}, all {N} basis columns", "evals_per_s_e2e": 1.0 / wall,
              "evals_per_s_device": 1e3 / dev_ms, "sweep_ms": hs_ms, "gpu_launches": launches,
              "roofline": roofline(hess_model(L, depth, False), N, L, hs_ms, hs_n)}
        out[f"target_L{L}_depth{depth}"] = r2
        target_cases.append((r2, L, depth, tdepth, vlist, perms, tvlist, tperms, g, H, wall))

    # (3) optimiser
    L, depth, tdepth, niter = 8, 5, 3, 10
    vlist, perms, tvlist, tperms, _ = workload(L, depth, tdepth, 0, 1)
    tg = gpu.Target(brickwall=(tvlist, tperms))
    gpu.optimize_brickwall_circuit_hmat(tg, vlist, perms, L, 1)
    t0 = time.perf_counter()
    f_iter, _ = gpu.optimize_brickwall_circuit_hmat(tg, vlist, perms, L, niter)
    tg_s = time.perf_counter() - t0
    r3 = {"workload": f"optimize_brickwall_circuit_hmat, L={L} depth {depth}, target depth {tdepth}, {niter} iterations",
          "seconds": tg_s, "seconds_per_iteration": tg_s / niter, "f_first": float(f_iter[0]),
          "f_final": float(f_iter[-1])}
    out["optimize_hmat_L8"] = r3

    # (4) sampling estimator: gradient vector and Hessian matrix from Haar-random states
    L, depth, tdepth, ns = 14, 8, 4, 64
    vlist, perms, tvlist, tperms, _ = workload(L, depth, tdepth)
    tg = gpu.Target(brickwall=(tvlist, tperms))
    rng = gpu.seed_rng_state(2024)

    def sampled():
        return gpu.brickwall_unitary_target_gradient_vector_hessian_matrix_sampling(tg, vlist, perms, L, ns, rng)

    sampled()
    _, wall, dev_ms, hs_ms, hs_n, launches = timed(sampled, steps)
    r4 = {"workload": f"f + gradient vector + Hessian matrix estimated from {ns} Haar-random states, brickwall L={L} "
                      f"depth {depth} vs brickwall target depth {tdepth} (per-gate sweep)",
          "samples_per_s_e2e": ns / wall, "ms_per_call": wall * 1e3, "sweep_ms": hs_ms, "gpu_launches": launches,
          "roofline": roofline(hess_model(L, depth, False), ns, L, hs_ms, hs_n)}
    out["sampling_L14"] = r4

    # (5) block-encoding target: gradient vector and Hessian matrix
    L, depth, hdepth = 12, 9, 3
    vlist, perms, hv, hp = _benc_case(L, depth, hdepth)
    th = gpu.Target(brickwall=(hv, hp))

    def benc():
        return gpu.brickwall_blockenc_target_gradient_vector_hessian_matrix(th, vlist, perms, L)

    benc()
    _, wall, dev_ms, hs_ms, hs_n, launches = timed(benc, steps)
    r5 = {"workload": f"block encoding || P^dag W P - H ||_F^2 / 2: f + gradient vector + Hessian matrix, brickwall "
                      f"L={L} depth {depth}, H a brickwall of depth {hdepth} on {L // 2} qubits, all {1 << (L // 2)} "
                      f"columns", "evals_per_s_e2e": 1.0 / wall, "ms_per_call": wall * 1e3, "sweep_ms": hs_ms,
          "gpu_launches": launches,
          "roofline": roofline(hess_model(L, depth, False), 1 << (L // 2), L, hs_ms, hs_n)}
    r5["roofline"]["bytes_model"] += (" (the 2^(L/2) block-encoding columns; the tangents the sweep also carries "
                                      "through the last gate are not counted)")
    out["blockenc_L12"] = r5
    if not have_ref:
        return out
    cores = os.cpu_count() or 1
    s_cols = 1 << (L // 2)
    with mp.get_context("spawn").Pool(cores) as pool:
        t0 = time.perf_counter()
        pool.map(_ref_blockenc_worker, [(L, depth, hdepth, k, k + 1) for k in range(min(cores, s_cols))])
        tref = time.perf_counter() - t0
    v = (min(cores, s_cols) / s_cols) / tref
    r5["cpu_baseline"] = {"value": v, "unit": "evals/s", "cores": min(cores, s_cols), "kind": "reference",
                          "sample": f"{min(cores, s_cols)} of {s_cols} columns (one per core) through the reference's "
                                    f"block-encoding Hessian column loop, {tref:.1f} s wall; evals/s = sampled "
                                    f"fraction / wall time"}
    r5["speedup_e2e"] = (1.0 / wall) / v

    cores = os.cpu_count() or 1
    with mp.get_context("spawn").Pool(cores) as pool:
        t0 = time.perf_counter()
        pool.map(_ref_sampling_worker, [(L, depth, tdepth, 100 + k) for k in range(cores)])
        tref = time.perf_counter() - t0
    r4["cpu_baseline"] = {"value": cores / tref, "unit": "samples/s", "cores": cores, "kind": "reference",
                          "sample": f"{cores} single-sample calls of the reference's "
                                    f"brickwall_unitary_target_gradient_vector_hessian_matrix_sampling, one per core, "
                                    f"{tref:.1f} s wall"}
    r4["speedup_e2e"] = (ns / wall) / (cores / tref)

    # reference legs
    vlist, perms, psi, dout, dpsi, dv, hess, wall = single_case
    t0 = time.perf_counter()
    _, dpr, dvr, hr = Reference().forward_backward_hessian(vlist, perms, psi, dout)
    tref = time.perf_counter() - t0
    r1["cpu_baseline"] = {"value": tref * 1e3, "unit": "ms per call", "cores": 1, "kind": "reference",
                          "sample": "one full call of the reference (single-threaded C)"}
    r1["speedup_e2e"] = tref / wall
    r1["max_rel_diff_vs_reference"] = {
        "hess": float(np.max(np.abs(hess - hr)) / np.max(np.abs(hr))),
        "dvlist": float(np.max(np.abs(dv - dvr)) / np.max(np.abs(dvr))),
        "dpsi": float(np.max(np.abs(dpsi - dpr)) / np.max(np.abs(dpr)))}
    for r2, L, depth, tdepth, vlist, perms, tvlist, tperms, g, H, wall in target_cases:
        N = 1 << L
        if L <= 8:
            t0 = time.perf_counter()
            fr, gr, Hr = Reference().gradient_vector_hessian_matrix(vlist, perms, L, tvlist, tperms)
            tref = time.perf_counter() - t0
            r2["cpu_baseline"] = {"value": 1.0 / tref, "unit": "evals/s", "cores": 1, "kind": "reference",
                                  "sample": "one full evaluation of the reference (single-threaded C)"}
            r2["speedup_e2e"] = tref / wall
            r2["max_rel_diff_vs_reference"] = {"H": float(np.max(np.abs(H - Hr)) / np.max(np.abs(Hr))),
                                               "grad": float(np.max(np.abs(g - gr)) / np.max(np.abs(gr)))}
        else:
            cores = os.cpu_count() or 1
            jobs = [(L, depth, tdepth, k, k + 1) for k in range(cores)]
            with mp.get_context("spawn").Pool(cores) as pool:
                t0 = time.perf_counter()
                pool.map(_ref_hessian_worker, jobs)
                tref = time.perf_counter() - t0
            v = (cores / N) / tref
            r2["cpu_baseline"] = {"value": v, "unit": "evals/s", "cores": cores, "kind": "reference",
                                  "sample": f"{cores} of {N} basis columns (one per core) through the reference's "
                                            f"forward + backward_hessian column loop, {tref:.1f} s wall; "
                                            f"evals/s = sampled fraction / wall time"}
            r2["speedup_e2e"] = (1.0 / wall) / v
    L, depth, tdepth = 8, 5, 3
    vlist, perms, tvlist, tperms, _ = workload(L, depth, tdepth, 0, 1)
    nref = 2
    t0 = time.perf_counter()
    fr, _ = Reference().optimize_brickwall_hmat(vlist, perms, L, tvlist, tperms, nref)
    tref = time.perf_counter() - t0
    r3["cpu_baseline"] = {"value": tref / nref, "unit": "s per iteration", "cores": 1, "kind": "reference",
                          "sample": f"{nref} iterations of the reference driver"}
    r3["speedup_per_iteration"] = (tref / nref) / r3["seconds_per_iteration"]
    r3["f_iter_max_rel_diff_vs_reference"] = float(np.max(np.abs(f_iter[:nref] - fr[:nref]) / np.abs(fr[:nref])))
    return out


# ----------------------------------------------------------------------------- batched and serving

def _real_workload(L, depth, tdepth, seed=30):
    """Real orthogonal brickwall (QR of Gaussian matrices, sign-fixed) against a real
    brickwall target, with a 6-parameter tangent direction per gate."""
    def orth(rng):
        q, r = np.linalg.qr(rng.standard_normal((4, 4)))
        return q * np.sign(np.diagonal(r))

    from rqcopt_hpc_b200 import real
    rng, trng, drng = (np.random.default_rng(seed + k) for k in range(3))
    vlist = np.stack([orth(rng) for _ in range(depth)])
    tvlist = np.stack([orth(trng) for _ in range(tdepth)])
    vdirs = np.stack([real.real_to_tangent(drng.standard_normal(6), vlist[k]) for k in range(depth)])
    return vlist, perms_for(L, depth), tvlist, perms_for(L, tdepth), vdirs


def _ref_real_columns_worker(args):
    L, depth, tdepth, b0, b1 = args
    from oracle.oracle import RealReference
    vlist, perms, tvlist, tperms, vdirs = _real_workload(L, depth, tdepth)
    t0 = time.perf_counter()
    RealReference().brickwall_hvp_columns(vlist, vdirs, perms, L, tvlist, tperms, b0, b1)
    return time.perf_counter() - t0


def real_build_path(gpu, steps=3, L=14, depth=9, tdepth=5, seconds=8.0, with_reference=True):
    """The reference's real-orthogonal build (librqcopt_gpu_real.so): one f + projected
    gradient + projected HVP evaluation over all basis columns through the real C ABI
    (host gates, complex128 engine), against the reference's real build compiled in
    oracle/_ref on a per-core column sample."""
    import multiprocessing as mp
    from rqcopt_hpc_b200 import real
    vlist, perms, tvlist, tperms, vdirs = _real_workload(L, depth, tdepth)
    gpu.set_precision(gpu.PRECISION_C128)
    t = real.Target(brickwall=(tvlist, tperms))

    def ev():
        return real.brickwall_unitary_target_projected_hessian_vector_product(t, vlist, vdirs, perms, L)

    ev()
    real.reset_launch_count()
    t0 = time.perf_counter()
    for _ in range(steps):
        f, g, h = ev()
    wall = (time.perf_counter() - t0) / steps
    launches = real.launch_count() // steps
    # reverse-pass kernel time of one more evaluation (CUDA events around each launch)
    gpu.enable_kernel_timing(True)
    gpu.kernel_time(gpu.KC_REVERSE)
    ev()
    rev_ms, rev_n = gpu.kernel_time(gpu.KC_REVERSE)
    gpu.enable_kernel_timing(False)
    N = 1 << L
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    cfg = gpu.last_config()
    G = depth * (L // 2)
    npass = G if cfg["gates_per_pass"] == 1 else -(-G // cfg["gates_per_pass"])
    rbytes = float(6 * npass - 5) * N * (N // 2) * 16   # npass reverse passes per column over N/2 paired columns
    achieved = rbytes / (rev_ms * 1e-3) / 1e9 if rev_ms > 0 else None
    out = {"workload": f"real build: f + projected gradient (6 per gate) + projected HVP, real orthogonal brickwall "
                       f"L={L} depth {depth} vs real brickwall target depth {tdepth}, all {N} basis columns as "
                       f"{N // 2} paired columns, complex128 engine", "evals_per_s_e2e": 1.0 / wall,
           "ms_per_eval": wall * 1e3, "gpu_launches": launches, "f": float(f),
           "roofline": {"kernel": ("k6_rev" if cfg["reconstruct"] else "k3_rev") + " (complex128 FP64-MMA "
                                  "gradient/HVP pass)", "bound": "hbm",
                        "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                        "frac": achieved / hbm_peak if achieved else None,
                        "bytes_model": "(6P-5) x 2^L x 2^(L-1) x 16 B per evaluation (P reverse passes over the "
                                       "paired columns)", "passes_per_column": npass, "launches": rev_n,
                        "reverse_ms": rev_ms,
                        "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in peaks
                        else "fallback 6650 GB/s"}}
    from oracle.oracle import RealReference
    if not with_reference or not RealReference.available():
        return out
    N = 1 << L
    t0 = time.perf_counter()
    RealReference().brickwall_hvp_columns(vlist, vdirs, perms, L, tvlist, tperms, 0, 2)
    per_col = max((time.perf_counter() - t0) / 2, 1e-6)
    cores = os.cpu_count() or 1
    cols = max(1, min(N // cores, int(seconds / per_col)))
    with mp.get_context("spawn").Pool(cores) as pool:
        t0 = time.perf_counter()
        pool.map(_ref_real_columns_worker, [(L, depth, tdepth, k * cols, (k + 1) * cols) for k in range(cores)])
        tref = time.perf_counter() - t0
    v = (cores * cols / N) / tref
    out["cpu_baseline"] = {"value": v, "unit": "evals/s", "cores": cores, "kind": "reference",
                           "sample": f"{cores * cols} of {N} basis columns ({cols} per core) through the real build's "
                                     f"quantum_circuit_gates_hessian_vector_product with its brickwall target, "
                                     f"{tref:.1f} s wall; evals/s = sampled fraction / wall time"}
    out["speedup_e2e"] = (1.0 / wall) / v
    return out


def front_end_path(L=8, depth=5, niter=10, ref_niter=2, seed=50, with_reference=True):
    """The reference's Python module API (pymodule/rqcopt_module.c): optimize_brickwall_circuit
    with a dense Haar-random 2^L x 2^L target U, through rqcopt_hpc_b200.rqcopt_hpc (the GPU
    library) and through the reference module compiled in oracle/_ref (single-threaded C);
    seconds per trust-region iteration."""
    from rqcopt_hpc_b200 import rqcopt_hpc
    rng = np.random.default_rng(seed)
    z = (rng.standard_normal((1 << L, 1 << L)) + 1j * rng.standard_normal((1 << L, 1 << L))) / np.sqrt(2)
    q, r = np.linalg.qr(z)
    U = np.ascontiguousarray(q * (np.diagonal(r) / np.abs(np.diagonal(r))))
    vlist, perms, _, _, _ = workload(L, depth, 1)
    vl, pm = list(vlist), [list(map(int, p)) for p in perms]
    rqcopt_hpc.optimize_brickwall_circuit(L, U, vl, pm, 1)
    t0 = time.perf_counter()
    _, f_iter = rqcopt_hpc.optimize_brickwall_circuit(L, U, vl, pm, niter)
    wall = (time.perf_counter() - t0) / niter
    out = {"workload": f"rqcopt_hpc.optimize_brickwall_circuit (the reference's Python module API), L={L} depth {depth}, "
                       f"dense Haar-random target U, {niter} iterations", "seconds_per_iteration": wall,
           "f_first": float(f_iter[0]), "f_final": float(f_iter[-1])}
    if not with_reference:
        return out
    from oracle.oracle import reference_module
    ref = reference_module()
    if ref is None:
        return out
    t0 = time.perf_counter()
    _, fr = ref.optimize_brickwall_circuit(L, U, vl, pm, ref_niter)
    tref = (time.perf_counter() - t0) / ref_niter
    out["cpu_baseline"] = {"value": tref, "unit": "s per iteration", "cores": 1, "kind": "reference",
                           "sample": f"{ref_niter} iterations of the reference module's optimize_brickwall_circuit "
                                     f"(single-threaded C)"}
    out["speedup_per_iteration"] = tref / wall
    out["f_iter_max_rel_diff_vs_reference"] = float(np.max(np.abs(f_iter[:ref_niter + 1] - fr)) / np.max(np.abs(fr)))
    return out


def batched_c4(gpu, torch, count=512, niter=30, sample_every=8):
    """C4: 512 independent brickwall instances (even L uniform over 6..12, depth over
    {3,5,7,9}, target depth 3, seeds 30+i / 10000+i), 30 trust-region iterations each.
    The batched complex64 path (complex64 passes with FP64 sums; one persistent kernel
    per round on a device work queue, CUDA-graph rounds) runs all instances.  The plain per-instance complex128 loop
    (optimize_brickwall_circuit_hvp one instance after another) runs on every
    `sample_every`-th instance, and so does the batched path once more, so the speed-up
    compares the two on identical work; the full loop's time is that sample's time scaled
    by count / sample size."""
    from rqcopt_hpc_b200 import batch
    from rqcopt_hpc_b200.workloads import batched_instances
    probs = batched_instances(count)
    sample = probs[::sample_every]
    out = {"workload": f"{count} brickwall instances, L in {{6,8,10,12}}, depth in {{3,5,7,9}}, target depth 3, "
                       f"{niter} RTR iterations each"}
    warm = batch.Batch(16, 2)   # kernel and graph set-up outside the timed runs
    for p in probs[:16]:
        warm.add(p, 2, gpu.PRECISION_C64)
    while warm.run(32) > 0:
        pass
    warm.close()

    def run_batched(ps):
        b = batch.Batch(len(ps), niter)
        for p in ps:
            b.add(p, niter, gpu.PRECISION_C64)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        while b.run(32) > 0:
            pass
        torch.cuda.synchronize()
        sec = time.perf_counter() - t0
        ev, hv = b.evaluations()
        f = np.array([b.result(k)[0][-1] for k in range(len(ps))])
        b.close()
        return sec, ev, hv, f

    tb, ev, hv, fb = run_batched(probs)
    tbs, evs, _, fbs = run_batched(sample)
    gpu.set_precision(gpu.PRECISION_C128)
    seen = set()
    for (L, vl, pm, tv, tp) in sample:
        if (L, len(vl)) not in seen:
            seen.add((L, len(vl)))
            gpu.optimize_brickwall_circuit_hvp(gpu.Target(brickwall=(tv, tp)), vl, pm, L, 2)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    fp = []
    for (L, vl, pm, tv, tp) in sample:
        f, _ = gpu.optimize_brickwall_circuit_hvp(gpu.Target(brickwall=(tv, tp)), vl, pm, L, niter)
        fp.append(f[-1])
    torch.cuda.synchronize()
    tps = time.perf_counter() - t0
    fp = np.array(fp)
    out["batched_c64"] = {"instances": count, "seconds": tb, "evaluations": ev, "hvp_evaluations": hv,
                            "evals_per_s": ev / tb, "instance_iterations_per_s": count * niter / tb}
    out["sample"] = {"instances": len(sample), "every": sample_every, "batched_c64_seconds": tbs,
                     "per_instance_c128_seconds": tps,
                     "f_final_max_rel_diff_c64_vs_c128": float(np.max(np.abs(fbs - fp) / np.abs(fp)))}
    out["per_instance_c128_full_seconds_scaled"] = tps * count / len(sample)
    out["speedup"] = tps / tbs
    return out


def serving_c5(gpu, rate=200.0, duration=60.0, wall=70.0, niter=100, grad_tol=1e-8, sizes=(8, 10, 12, 14),
               capacity=128, precisions=("mixed", "plain_c128")):
    """C5: Poisson arrivals (seed 40) of brickwall optimisation requests (even L in 8..14,
    P(L) ~ 2^(-(L-8)/2), depth in {3,5,7,9}, target depth 3), each stopping at gradient
    norm grad_tol or after niter iterations, admitted first come first served into a
    running batch of at most `capacity` requests within a 150 GB device budget, for the
    mixed-precision and the plain complex128 path in turn.  Each run offers `duration`
    seconds of arrivals and is measured for `wall` seconds: p50 / p99 time from arrival to
    completion of the requests completed in that window, completions per second, and the
    requests still running or queued at its end (at 200 req/s the offered load exceeds one
    GPU, so these latencies are queue-dominated)."""
    from rqcopt_hpc_b200 import batch, serving
    code = {"mixed": gpu.PRECISION_MIXED, "plain_c128": gpu.PRECISION_C128}
    out = {"workload": f"Poisson {rate:g} req/s for {duration:g} s (seed 40), L in {set(sizes)}, stop at gradient "
                       f"norm {grad_tol:g} or {niter} iterations, at most {capacity} requests in the running batch, "
                       f"150 GB admission budget, measured for {wall:g} s"}
    for name in precisions:
        reqs = serving.c5_requests(rate=rate, duration=duration, niter=niter, grad_tol=grad_tol,
                                   precision=code[name], sizes=sizes)
        b = batch.Batch(capacity=capacity, max_iterations=niter, sharing=True)
        srv = serving.Server(b, capacity=capacity, hbm_budget_bytes=150e9, footprint=batch.footprint,
                             rounds_per_step=4)
        t0 = time.perf_counter()
        done, left = serving.run_arrivals(srv, reqs, wall_limit=wall)
        el = time.perf_counter() - t0
        ev, hv = b.evaluations()
        b.close()
        r = {"offered": len(reqs), "wall_s": el, "completed": len(done), "still_running_or_queued": len(left),
             "completed_per_s": len(done) / el, "evaluations": ev, "rounds": srv.rounds}
        r.update(serving.latency_stats(done))
        if done:
            r["mean_iterations"] = float(np.mean([q.iterations for q in done]))
            r["converged"] = int(sum(q.iterations < niter for q in done))
        out[name] = r
    if "mixed" in out and "plain_c128" in out:
        out["completed_ratio_mixed_over_plain"] = out["mixed"]["completed"] / max(out["plain_c128"]["completed"], 1)
    return out


def _relerr(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def compare_mixed(gpu, torch, stream, step, res_c128, steps, L, G, Gt, P, hbm_peak, fp32_peak):
    """The same evaluation with complex64 passes and FP64 sums (MIXED mode: direct target
    calls run the complex64 passes), one warm-up and `steps` timed (CUDA events on the
    library stream), its error against the complex128 result of the headline, and the
    roofline of its dominant kernel (k5_rev, HBM) and of the whole evaluation against the
    measured FP32 peak."""
    gpu.set_precision(gpu.PRECISION_MIXED)
    step()
    torch.cuda.synchronize()
    gpu.enable_kernel_timing(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        res = step()
    e1.record(stream)
    torch.cuda.synchronize()
    rev_ms, rev_n = gpu.kernel_time(gpu.KC_REVERSE)
    cfg = gpu.last_config()
    gpu.enable_kernel_timing(False)
    gpu.set_precision(gpu.PRECISION_C128)
    ms = e0.elapsed_time(e1) / steps
    P = G if cfg["gates_per_pass"] == 1 else -(-G // cfg["gates_per_pass"])
    rbytes = reverse_bytes_per_eval(L, P, 8) * steps
    achieved = rbytes / (rev_ms * 1e-3) / 1e9 if rev_ms > 0 else None
    flops = flops_per_eval(L, G, Gt)
    pipe = "FP32 FMA pipe" if cfg["c64_fp32_pipe"] else "3xTF32 MMA"
    out = {"precision": f"complex64 passes ({pipe}), FP64 sums", "evals_per_s": 1e3 / ms, "ms_per_step": ms,
           "tuned": cfg,
           "rel_err_vs_c128": {"f": _relerr(res[0], res_c128[0]), "grad": _relerr(res[1], res_c128[1]),
                               "hvp": _relerr(res[2], res_c128[2])},
           "roofline": {"kernel": ("k7_rev (complex64 reverse pass on the FP32 pipe" if cfg["c64_fp32_pipe"]
                                   else "k5_rev (complex64 reverse pass on the 3xTF32 MMA")
                                  + f", adjoint reconstruction, {cfg['gates_per_pass']} fused gates)",
                        "bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                        "frac": achieved / hbm_peak if achieved else None, "launches": rev_n,
                        "avg_launch_ms": rev_ms / max(rev_n, 1)},
           "eval_flops": {"per_eval": flops, "achieved_tflops": flops / (ms * 1e-3) / 1e12, "peak_tflops": fp32_peak,
                          "frac": flops / (ms * 1e-3) / 1e12 / fp32_peak if fp32_peak else None,
                          "peak_source": "FP32 peak measured in this run (cuBLAS SGEMM, TF32 off)"}}
    return out


def mixed_equal_error(gpu, L=12, depth=3, tdepth=3, niter=80, seed=0, tseed=1):
    """Time to the same optimum: optimize_brickwall_circuit_hvp (reference defaults) from the
    same start, plain complex128 and mixed precision (complex64 HVPs until the gradient norm
    falls below the refinement threshold 1e-5, then complex128; f and gradient always
    complex128), on a workload the trust region drives to convergence within niter
    iterations.  Reports each run's wall time, its final f, the relative difference of the
    final f values, the iteration from which f stays within 1e-10 of its final value, and
    the Hessian-vector products each run made in each precision."""
    vlist, perms, tvlist, tperms, _ = workload(L, depth, tdepth, seed=seed, tseed=tseed, dseed=2)
    target = gpu.Target(brickwall=(tvlist, tperms))
    out = {"workload": f"optimize_brickwall_circuit_hvp, brickwall L={L} depth={depth} vs brickwall target "
                       f"depth={tdepth} (seeds {seed}/{tseed}), {niter} RTR iterations, run to convergence"}
    runs = {}
    for name, p in (("plain_c128", gpu.PRECISION_C128), ("mixed", gpu.PRECISION_MIXED)):
        gpu.set_precision(p)
        # one untimed run of the same length: workspace, kernels and the autotuner's choice
        # for every evaluation kind the run meets (the mixed run's complex128 refinement too)
        gpu.optimize_brickwall_circuit_hvp(target, vlist, perms, L, niter)
        t0 = time.perf_counter()
        f_iter, vopt = gpu.optimize_brickwall_circuit_hvp(target, vlist, perms, L, niter)
        sec = time.perf_counter() - t0
        tr = gpu.optimizer_trace()
        gpu.set_precision(gpu.PRECISION_C128)
        _, g = gpu.brickwall_unitary_target_and_projected_gradient(target, vopt, perms, L)
        near = np.abs(f_iter - f_iter[-1]) <= 1e-10 * abs(f_iter[-1])
        conv = int(np.argmax([np.all(near[k:]) for k in range(len(near))]))
        hv = int(tr["inner"].sum() + len(tr["inner"]))   # tCG products + the model product per iteration
        hv128 = int(((tr["inner"] + 1) * tr["refined"]).sum())
        refine_at = int(np.argmax(tr["refined"])) if tr["refined"].any() else None
        runs[name] = (sec, f_iter)
        out[name] = {"seconds": sec, "f_final": float(f_iter[-1]), "grad_norm_final": float(np.linalg.norm(g)),
                     "converged_at_iteration": conv, "hvp_evaluations": hv, "hvp_complex128": hv128,
                     "hvp_complex64": hv - hv128, "refined_from_iteration": refine_at,
                     "max_tcg_inner_iterations": int(tr["inner"].max())}
    fp, fm = runs["plain_c128"][1][-1], runs["mixed"][1][-1]
    out["f_final_rel_diff"] = abs(fm - fp) / max(abs(fp), 1e-300)
    out["equal_error"] = bool(out["f_final_rel_diff"] <= 1e-10)
    out["speedup"] = runs["plain_c128"][0] / runs["mixed"][0]
    return out


def summary(line):
    """Compact figures of every leg, the last key of the JSON line (so that they stay in
    view where only the end of a long line is kept)."""
    def g(d, *ks):
        for k in ks:
            if not isinstance(d, dict) or k not in d:
                return None
            d = d[k]
        return d

    def r(x, n=3):
        return None if x is None else float(f"{x:.{n}g}")

    out = {"c128_evals_per_s": r(line.get("value")), "c128_e2e_evals_per_s": r(g(line, "e2e", "value")),
           "roofline_frac": r(g(line, "roofline", "frac")), "cpu_ref_evals_per_s": r(g(line, "cpu_baseline", "value"))}
    if "mixed" in line:
        out["mixed_evals_per_s"] = r(g(line, "mixed", "evals_per_s"))
        out["mixed_over_plain"] = r(line.get("mixed_over_plain"))
        out["mixed_rel_err_f_grad_hvp"] = [r(g(line, "mixed", "rel_err_vs_c128", k), 2) for k in ("f", "grad", "hvp")]
        out["c64_reverse_hbm_frac"] = r(g(line, "mixed", "roofline", "frac"))
    me = line.get("mixed_equal_error")
    if me:
        out["equal_error"] = {"rel_diff": r(me.get("f_final_rel_diff"), 2), "speedup": r(me.get("speedup")),
                              "s_plain": r(g(me, "plain_c128", "seconds")), "s_mixed": r(g(me, "mixed", "seconds"))}
    gt = line.get("gate_throughput")
    if gt:
        out["c3_dram_gbs"] = {f"{p}_{k}": r(g(gt, p, f"gates_per_round_trip_{k}", "dram_gbs"))
                              for p in ("c128", "c64") for k in (1, 4)}
        out["c3_gate_equiv_gbs"] = {f"{p}_{k}": r(g(gt, p, f"gates_per_round_trip_{k}", "gate_equivalent_gbs"))
                                    for p in ("c128", "c64") for k in (1, 4)}
    bt = line.get("batched")
    if bt:
        out["c4"] = {"s_batched_512x30": r(g(bt, "batched_c64", "seconds")), "speedup": r(bt.get("speedup")),
                     "s_c128_scaled": r(bt.get("per_instance_c128_full_seconds_scaled"))}
    for key, nm in (("serving", "c5"), ("serving_sustainable", "c5_2req_s")):
        sv = line.get(key)
        if sv:
            out[nm] = {k: {"done": g(sv, k, "completed"), "p50_s": r((g(sv, k, "p50_ms") or 0) / 1e3),
                           "p99_s": r((g(sv, k, "p99_ms") or 0) / 1e3)} for k in ("mixed", "plain_c128") if k in sv}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="c128", choices=["mixed", "c64", "c128"],
                    help="c128 (default): plain complex128, the reference's arithmetic; mixed / c64: complex64 "
                         "passes with FP64 sums")
    ap.add_argument("--L", type=int, default=16)
    ap.add_argument("--depth", type=int, default=9)
    ap.add_argument("--tdepth", type=int, default=5)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--gates-per-pass", type=int, default=0,
                    help="gates fused per HBM round trip (1-4); 0 (default): chosen by the library's autotuner")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-gate-throughput", action="store_true")
    ap.add_argument("--no-compare", action="store_true", help="skip the complex128 comparison and the RTR runs")
    ap.add_argument("--no-batched", action="store_true", help="skip the 512-instance batched measurement")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving measurement")
    ap.add_argument("--no-hmat", action="store_true", help="skip the full-Hessian path measurement")
    ap.add_argument("--no-real", action="store_true", help="skip the real-orthogonal build measurement")
    ap.add_argument("--hmat-case", choices=["target", "single", "sampling", "blockenc", "real"],
                    help="run one evaluation at --L/--depth/--tdepth and exit (a small case for profilers): "
                         "'target' the full Hessian over all basis columns, 'single' one state's forward + "
                         "backward_hessian, 'sampling' the full Hessian from 64 Haar states, 'blockenc' the "
                         "block-encoding Hessian with H of depth --tdepth on L/2 qubits, 'real' the real build's "
                         "f + projected gradient + projected HVP")
    ap.add_argument("--column-chunk", type=int, default=0, help="basis columns per chunk (0: from the workspace)")
    ap.add_argument("--c64-pipe", default="auto", choices=["auto", "fp32", "mma"],
                    help="complex64 passes on the FP32 FMA pipe or the 3xTF32 MMA (auto: the autotuner's choice)")
    ap.add_argument("--reconstruct", type=int, default=-1, choices=[-1, 0, 1],
                    help="complex128 reverse passes rebuild states with adjoint gates (1) or recompute them (0); "
                         "-1 (default): chosen by the autotuner")
    ap.add_argument("--serving-wall", type=float, default=70.0)
    ap.add_argument("--c3-qubits", type=int, default=28, help="qubits of the gate-throughput state (C3: 28)")
    ap.add_argument("--gate-throughput-only", action="store_true",
                    help="run only the gate-throughput leg and print it (a small case for profilers)")
    a = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    L, depth, tdepth = a.L, a.depth, a.tdepth
    G, Gt = depth * (L // 2), tdepth * (L // 2)
    config = {"workload": f"brickwall L={L} depth={depth} vs matrix-free brickwall target depth={tdepth}, "
                          f"grad+HVP over all {1 << L} basis columns",
              "L": L, "depth": depth, "target_depth": tdepth, "columns": 1 << L,
              "l2": "working set of many GB, larger than L2 (no flush needed)",
              "parallelism": f"replicas x{world}"}

    if a.impl == "reference":
        if rank != 0:
            return
        steps = []
        base = None
        for k in range(a.warmup + a.steps):
            base = cpu_baseline(L, depth, tdepth, seconds=a.cpu_seconds / 3)
            if base is None:
                print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref not present"}))
                return
            if k >= a.warmup:
                steps.append(base["value"])
        v = float(np.median(steps))
        base["value"] = v
        print(json.dumps({"impl": "reference", "metric": METRIC, "value": v, "unit": "evals/s", "n_gpus": a.gpus,
                          "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True,
                          "scaling": "weak", "vs_baseline": None, "dtype": "c128 (f64)", "data": "synthetic (seeded)",
                          "config": config, "cpu_baseline": base,
                          "e2e": {"value": v, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return

    if a.hmat_case:
        from rqcopt_hpc_b200 import gpu
        gpu.set_column_chunk(a.column_chunk)
        vlist, perms, tvlist, tperms, _ = workload(L, depth, tdepth)
        if a.hmat_case == "target":
            f, g, H = gpu.brickwall_unitary_target_gradient_vector_hessian_matrix(
                gpu.Target(brickwall=(tvlist, tperms)), vlist, perms, L)
            print(json.dumps({"hmat_case": "target", "L": L, "depth": depth, "f": f.real, "H_norm": float(np.abs(H).max())}))
        elif a.hmat_case == "sampling":
            f, g, H = gpu.brickwall_unitary_target_gradient_vector_hessian_matrix_sampling(
                gpu.Target(brickwall=(tvlist, tperms)), vlist, perms, L, 64, gpu.seed_rng_state(42))
            print(json.dumps({"hmat_case": "sampling", "L": L, "depth": depth, "f": f.real}))
        elif a.hmat_case == "blockenc":
            vl, pm, hv, hp = _benc_case(L, depth, tdepth)
            f, g, H = gpu.brickwall_blockenc_target_gradient_vector_hessian_matrix(gpu.Target(brickwall=(hv, hp)), vl, pm, L)
            print(json.dumps({"hmat_case": "blockenc", "L": L, "depth": depth, "f": float(f)}))
        elif a.hmat_case == "real":
            from rqcopt_hpc_b200 import real
            vl, pm, tv, tp, vd = _real_workload(L, depth, tdepth)
            f, g, h = real.brickwall_unitary_target_projected_hessian_vector_product(real.Target(brickwall=(tv, tp)), vl,
                                                                                     vd, pm, L)
            print(json.dumps({"hmat_case": "real", "L": L, "depth": depth, "f": float(f)}))
        else:
            rng = np.random.default_rng(16)
            psi = (rng.standard_normal(1 << L) + 1j * rng.standard_normal(1 << L)) / np.sqrt(2 << L)
            out, cache = gpu.brickwall_unitary_forward(vlist, perms, psi)
            _, dv, hess = gpu.brickwall_unitary_backward_hessian(vlist, perms, cache, np.conj(out))
            print(json.dumps({"hmat_case": "single", "L": L, "depth": depth, "hess_norm": float(np.abs(hess).max())}))
        return

    import torch
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)

    from rqcopt_hpc_b200 import gpu
    lib = gpu.lib()
    if a.gate_throughput_only:
        print(json.dumps({"gate_throughput": gate_throughput(gpu, torch, L=a.c3_qubits)}))
        return
    prec = {"c128": gpu.PRECISION_C128, "c64": gpu.PRECISION_C64, "mixed": gpu.PRECISION_MIXED}[a.precision]
    gpu.set_precision(prec)
    gpu.set_autotune(True)
    if a.gates_per_pass:
        gpu.set_gates_per_pass(a.gates_per_pass)
    if a.reconstruct >= 0:
        gpu.set_reconstruct(bool(a.reconstruct))
    if a.column_chunk:
        gpu.set_column_chunk(a.column_chunk)
    if a.c64_pipe != "auto":
        gpu.set_c64_fp32_pipe(a.c64_pipe == "fp32")
    vlist, perms, tvlist, tperms, vdirs = workload(L, depth, tdepth)
    target = gpu.Target(brickwall=(tvlist, tperms))

    def step():
        return gpu.brickwall_unitary_target_projected_hessian_vector_product(target, vlist, vdirs, perms, L)

    for _ in range(a.warmup):
        step()
    stream = torch.cuda.ExternalStream(lib.rqcopt_gpu_stream())

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    # device-timed region (value) with per-kernel event timing and clock sampling
    gpu.enable_kernel_timing(True)
    gpu.reset_launch_count()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clk:
        # every step goes through the C ABI with host buffers (gates in; f, gradient and
        # HVP out): the events on the library stream give the device time, the host
        # clock around the same steps the end-to-end time
        t0 = time.perf_counter()
        ev0.record(stream)
        for _ in range(a.steps):
            res = step()
        ev1.record(stream)
        barrier()
        e2e_ms = (time.perf_counter() - t0) * 1e3
    launches = gpu.launch_count()
    tuned = gpu.last_config()
    dev_ms = ev0.elapsed_time(ev1)
    rev_ms, rev_n = gpu.kernel_time(gpu.KC_REVERSE)
    fwd_ms, fwd_n = gpu.kernel_time(gpu.KC_FORWARD)
    app_ms, app_n = gpu.kernel_time(gpu.KC_APPLY)
    fus_ms, fus_n = gpu.kernel_time(gpu.KC_FUSED)
    gpu.enable_kernel_timing(False)

    from rqcopt_hpc_b200.replicas import max_over_ranks, whole_job_rate
    dev_ms, e2e_ms = max_over_ranks([dev_ms, e2e_ms], device="cuda")

    if rank == 0:
        itemsize = 16 if prec == gpu.PRECISION_C128 else 8
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except (OSError, ValueError):
            pass
        hbm_peak = peaks.get("hbm_gbs", 6650.0)
        hbm_src = "measured (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in peaks else "fallback 6650 GB/s"
        fp = measure_fp_peaks(torch) if world == 1 else {}
        gpp = tuned["gates_per_pass"]
        npass = G if gpp == 1 else -(-G // gpp)
        value = whole_job_rate(world, a.steps, dev_ms)
        flops = flops_per_eval(L, G, Gt)
        rbytes = reverse_bytes_per_eval(L, npass, itemsize) * a.steps
        gbs = rbytes / (rev_ms * 1e-3) / 1e9 if rev_ms > 0 else None
        if itemsize == 16:
            # complex128: the reverse pass does ~11 flop per byte it moves, above the FP64
            # ridge (~6 flop/B), so its roofline is the FP64 tensor pipe (DMMA) that runs it
            rflops = reverse_flops_per_eval(L, G) * a.steps
            achieved = rflops / (rev_ms * 1e-3) / 1e12 if rev_ms > 0 else None
            fp64 = fp.get("fp64_tflops")
            roof = {"kernel": (("k6_rev (complex128 reverse pass rebuilding states with adjoint gates"
                                if tuned["reconstruct"] else "k3_rev (complex128 reverse pass recomputing states")
                               + f" on the FP64 tensor pipe, DMMA m8n8k4, {gpp} fused gates over a column chunk)"
                               if gpp > 1 else "k_reverse (complex128 gradient/HVP pass of one gate, FP64)"),
                    "bound": "tensor", "achieved": achieved, "peak": fp64, "unit": "TFLOP/s",
                    "frac": achieved / fp64 if (achieved and fp64) else None,
                    "flops_model": "192 flop per amplitude, gate and basis column (six 4x4 complex products of an "
                                   "amplitude group: the outer sums dG, HZ and the adjoint updates phi, dphi); states "
                                   "rebuilt inside a pass not counted",
                    "peak_source": "FP64 peak measured in this run (cuBLAS DGEMM 8192^3)",
                    "traffic": rbytes / max(rev_n, 1) * 0.99,
                    "traffic_source": "ncu capture of one middle k6_rev pass at L=12 (DRAM bytes / algorithmic = "
                                      "0.99, profiles/k6_rev_c128_L12_d5.md), scaled to the bytes of an average "
                                      "launch here",
                    "hbm_view": {"achieved_gbs": gbs, "peak_gbs": hbm_peak, "frac": gbs / hbm_peak if gbs else None,
                                 "peak_source": hbm_src},
                    "launches": rev_n, "avg_launch_ms": rev_ms / max(rev_n, 1)}
        else:
            ratio = TRAFFIC_RATIO.get(itemsize) if gpp > 1 else None
            roof = {"kernel": "k5_rev (complex64 reverse pass, adjoint reconstruction, 3xTF32 MMA, "
                              f"{gpp} fused gates over a column chunk)",
                    "bytes_model": "(6P-5) * 2^L * 2^L * itemsize per evaluation (P passes): reads of phi, dphi, psi, "
                                   "dpsi and writes of phi', dphi' per pass",
                    "bound": "hbm", "achieved": gbs, "peak": hbm_peak, "unit": "GB/s",
                    "frac": gbs / hbm_peak if gbs else None, "peak_source": hbm_src,
                    "traffic": rbytes / max(rev_n, 1) * ratio if ratio else None,
                    "launches": rev_n, "avg_launch_ms": rev_ms / max(rev_n, 1)}
        peak_eval = fp.get("fp64_tflops") if itemsize == 16 else fp.get("fp32_tflops")
        line = {
            "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": dev_ms / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": "c128 (f64)" if itemsize == 16 else "c64 (f32 passes on 3xTF32 MMA, f64 sums)",
            "precision": a.precision,
            "data": "synthetic (seeded Haar gates)", "config": config,
            "e2e": {"value": whole_job_rate(world, a.steps, e2e_ms), "unit": "evals/s",
                    "h2d_bytes_per_step": int(vlist.nbytes + vdirs.nbytes + tvlist.nbytes + perms.nbytes + tperms.nbytes),
                    "d2h_bytes_per_step": int(16 + 2 * 16 * depth * 8)},
            "roofline": roof,
            "kernel_share": {"reverse_ms": rev_ms, "forward_ms": fwd_ms, "apply_ms": app_ms,
                             "fused_forward_ms": fus_ms, "device_ms": dev_ms},
            "eval_flops": {"per_eval": flops, "achieved_tflops": flops * a.steps / (dev_ms * 1e-3) / 1e12,
                           "peak_tflops": peak_eval,
                           "frac": (flops * a.steps / (dev_ms * 1e-3) / 1e12 / peak_eval) if peak_eval else None,
                           "model": "N^2 (32 G_t + 292 G - 124): the reference's flops of one evaluation",
                           "peak_source": ("FP64" if itemsize == 16 else "FP32") + " peak measured in this run"},
            "measured_peaks": fp,
            "tuned": {"gates_per_pass": gpp, "column_chunk": tuned["column_chunk"] or "from workspace",
                      "reconstruct": tuned["reconstruct"], "chosen_by_autotuner": tuned["tuned"],
                      "sample_ms_per_column": tuned["ms_per_column"]},
            "clocks": clk.summary(), "gpu_launches": int(launches),
        }
        if world == 1 and prec == gpu.PRECISION_C128 and not a.no_compare:
            line["mixed"] = compare_mixed(gpu, torch, stream, step, res, min(a.steps, 3), L, G, Gt, npass, hbm_peak,
                                          fp.get("fp32_tflops"))
            line["mixed_over_plain"] = line["ms_per_step"] / line["mixed"]["ms_per_step"]
            line["mixed_equal_error"] = mixed_equal_error(gpu)
            gpu.set_precision(prec)
        if not a.no_gate_throughput:
            line["gate_throughput"] = gate_throughput(gpu, torch, L=a.c3_qubits)
        if not a.no_batched and world == 1:
            line["batched"] = batched_c4(gpu, torch)
            gpu.set_precision(prec)
        if not a.no_serving and world == 1:
            line["serving"] = serving_c5(gpu, wall=a.serving_wall)
            line["serving_sustainable"] = serving_c5(gpu, rate=2.0, duration=10.0, wall=15.0, sizes=(8, 10),
                                                     capacity=32)
            gpu.set_precision(prec)
        if not a.no_hmat and world == 1:
            line["hmat"] = hmat_path(gpu, torch, stream, hbm_peak, with_reference=not a.no_cpu_baseline,
                                     fp64_peak=fp.get("fp64_tflops"))
            gpu.set_precision(prec)
        if not a.no_hmat and world == 1:
            line["front_end"] = front_end_path(with_reference=not a.no_cpu_baseline)
            gpu.set_precision(prec)
        if not a.no_real and world == 1:
            line["real_build"] = real_build_path(gpu, with_reference=not a.no_cpu_baseline)
            gpu.set_precision(prec)
        if not a.no_cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_baseline(L, depth, tdepth, seconds=a.cpu_seconds)
        line["summary"] = summary(line)
        print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
