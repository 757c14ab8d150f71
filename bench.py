"""Benchmark: adjoint-mode circuit gradients at n = 26 (the headline metric).

Workload (one "step" = one full energy + gradient evaluation):
  26 qubits, FP32 amplitudes with FP64 accumulation; 20 layers of RX, RY, RZ
  on every qubit plus CRX(i, i+1) for i = 1..25 (2,060 parameters, uniform in
  [0, 2 pi), seeded); observable = open-chain XXZ, sum X_iX_{i+1} + Y_iY_{i+1}
  + 0.5 Z_iZ_{i+1} (75 Pauli terms); psi0 = |0...0>.

Arms:
  default            this engine (libvqcb200, sm_100a) through its C ABI;
  --impl reference   the reference's algorithm on the host cores (the C++
                     restatement under oracle/, all host threads), on a
                     bounded sample of the same workload scaled to grads/s.

Multi-GPU (torchrun): every rank runs an independent replica (the path has no
exchange step at this size); value = sum over ranks of grads/s, timed as the
max over ranks.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
for _p in (REPO, os.path.join(REPO, "vqc.jl_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

N_QUBITS = 26
LAYERS = 20
SEED = 20261203
METRIC = "circuit grads/s at n=26 (FP32 states, FP64 accumulation)"
UNIT = "grads/s"


def workload():
    from vqcb200 import workloads as W
    rng = np.random.default_rng(SEED)
    theta = rng.uniform(0, 2 * np.pi, LAYERS * (4 * N_QUBITS - 1))
    spec = W.rxyz_crx_spec(N_QUBITS, LAYERS, theta)
    hspec = W.xxz_spec(N_QUBITS, 0.5)
    return spec, hspec


def peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu_id), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200", "-f", self.path], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 8:
                    continue
                try:
                    sm.append(float(f[0]))
                    smax.append(float(f[1]))
                except ValueError:
                    continue
                for nm, v in zip(names, f[4:8]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
            os.unlink(self.path)
        except Exception:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def traffic_from_profiles(kernel):
    """Per-launch DRAM bytes of `kernel` from the committed ncu summary, if any."""
    try:
        with open(os.path.join(REPO, "profiles", "ncu_traffic.json")) as f:
            d = json.load(f)
        return d.get(kernel, {}).get("dram_bytes_per_launch_full_size")
    except Exception:
        return None


# ----------------------------------------------------------------------------- CPU arm
def cpu_sample(nthreads, reps=1, n=N_QUBITS, dtype=np.complex64):
    """Times the oracle's restatement of the reference's gradient on a bounded
    sample of the workload and scales it to one full gradient.

    Sample: forward + reverse sweep (uncompute of both states, one two-state
    expectation pass per parameter: circuitdiff.jl:23-32) of 2 single-qubit
    rotations and 1 CRX at full n, plus one XXZ key (expectation + the two
    H-apply passes of the expectation pullback); scaled by the workload's
    counts: 20 x (78 rotations + 25 CRX) gates and 25 keys."""
    from oracle import oracle as O
    spec, hspec = workload()
    psi = O.zero_state(n, dtype)
    O.apply_gate(psi, [0], np.array([[1, 1], [1, -1]]) / np.sqrt(2), nthreads)  # a dense-ish start
    lam = psi.copy()
    sample_1q = [g for g in O.from_spec(spec[:3])][:2]
    sample_crx = O.from_spec([s for s in spec if s[0] == "crx"][:1])

    def sweep(gates):
        t0 = time.perf_counter()
        for pos, U, _ in gates:
            O.apply_gate(psi, pos, U, nthreads)
        for pos, U, dUs in reversed(gates):
            Ud = U.conj().T
            O.apply_gate(lam, pos, Ud, nthreads)
            O.apply_gate(psi, pos, Ud, nthreads)
            for dU in dUs:
                O.expect_dense(lam, pos, dU.conj().T @ U, vc=psi, nthreads=nthreads)
        return time.perf_counter() - t0

    t1 = sum(sweep(sample_1q) for _ in range(reps)) / (reps * len(sample_1q))
    tc = sum(sweep(sample_crx) for _ in range(reps)) / reps
    key = O.group_by_key(O.terms_from_spec(hspec[:3]))
    (kpos, kM), = key.items()
    t0 = time.perf_counter()
    O.expect_dense(psi, kpos, kM.astype(dtype), nthreads=nthreads)
    out = np.zeros_like(psi)
    O.apply_gate_add(psi, out, kpos, kM, nthreads)
    O.apply_gate_add(psi, out, kpos, kM.conj().T, nthreads)
    tk = time.perf_counter() - t0
    per_grad = LAYERS * (3 * n * t1 + (n - 1) * tc) + (n - 1) * tk
    sample_s = reps * (2 * t1 + tc) + tk
    return 1.0 / per_grad, sample_s


def cpu_full_check(nthreads, n=20):
    """The extrapolation behind cpu_sample checked against one timed full
    gradient of the same workload at a smaller size (n qubits, all 20 layers,
    FP32): returns the measured and extrapolated seconds per gradient."""
    from oracle import oracle as O
    from vqcb200 import workloads as W
    rng = np.random.default_rng(SEED)
    theta = rng.uniform(0, 2 * np.pi, LAYERS * (4 * n - 1))
    gates = O.from_spec(W.rxyz_crx_spec(n, LAYERS, theta))
    terms = O.terms_from_spec(W.xxz_spec(n, 0.5))
    t0 = time.perf_counter()
    O.energy_and_gradient(gates, terms, O.zero_state(n, np.complex64), nthreads=nthreads)
    measured = time.perf_counter() - t0
    rate, _ = cpu_sample(nthreads, reps=8, n=n)
    return {"n_qubits": n, "measured_s_per_gradient": measured, "extrapolated_s_per_gradient": 1.0 / rate,
            "measured_over_extrapolated": measured * rate}


def run_reference(args, rank, world):
    if rank != 0:
        return
    nthreads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_sample(nthreads)
    vals, secs = [], 0.0
    for _ in range(args.steps):
        v, s = cpu_sample(nthreads)
        vals.append(v)
        secs += s
    value = float(np.median(vals))
    sample = ("per step: 2 rotations + 1 CRX forward and reverse sweep and one XXZ key at n=26, FP32 amplitudes "
              "(the reference's ComplexF32 path, FP32 accumulation), scaled to 20x(78 rotations + 25 CRX) + 25 keys")
    # a step is the bounded sample; value is the sample's rate scaled to whole gradients
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * secs / max(args.steps, 1),
            "ms_per_gradient_extrapolated": 1000.0 / value, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64",
            "data": "synthetic (seeded)", "config": config_dict(args),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def config_dict(args):
    return {"workload": "adjoint gradient, n=26, 20 x (RX,RY,RZ on every qubit + CRX(i,i+1)), XXZ 75 terms",
            "n_qubits": N_QUBITS, "layers": LAYERS, "n_params": LAYERS * (4 * N_QUBITS - 1), "n_pauli_terms": 75,
            "state_bytes": (1 << N_QUBITS) * 8, "l2": "state (512 MiB) larger than L2; no flush needed",
            "parallelism": "replicas" if args.gpus > 1 else "single"}


# ----------------------------------------------------------------------------- GPU arm
def run_ours(args, rank, world, local_rank):
    import torch
    import vqcb200 as V
    from vqcb200 import _lib, replicas
    from vqcb200 import workloads as W
    from vqcb200.circuit import Packed

    torch.cuda.set_device(local_rank)
    lib = V.load()
    spec, hspec = workload()
    circuit = W.to_circuit(spec)
    H = W.to_operator(hspec)
    packed = Packed(circuit)
    terms, nterms = H.packed()

    def make_state(dtype):
        return V.StateVector(N_QUBITS, dtype=dtype, device=local_rank)

    def grad_call(psi0, grads, energy):
        _lib.check(lib.vqc_adjoint_grad(psi0.handle, packed.gates, packed.ngates, packed.mats_ptr(), packed.params,
                                        packed.nparams, terms, nterms, energy, grads.ctypes.data_as(_lib._D)))

    def timed(psi0, steps, warmup, profile=False):
        grads = np.zeros(packed.nparams)
        energy = (ctypes.c_double * 2)()
        stream = torch.cuda.ExternalStream(lib.vqc_state_stream(psi0.handle), device=local_rank)
        for _ in range(warmup):
            grad_call(psi0, grads, energy)
        replicas.barrier()
        torch.cuda.synchronize()
        if profile:
            _lib.profile_enable(True)
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(steps):
            grad_call(psi0, grads, energy)
        end.record(stream)
        end.synchronize()
        torch.cuda.synchronize()
        prof = None
        if profile:
            prof = _lib.profile_read(with_flops=True)
            _lib.profile_enable(False)
        ms = start.elapsed_time(end) / steps
        if world > 1:
            ms = replicas.max_over_ranks(ms, device="cuda")  # slowest replica
            replicas.barrier()
        return ms, prof, complex(energy[0], energy[1]), grads

    def timed_e2e(psis, host, steps, warmup):
        """End to end through the public API: every step uploads its psi0 from
        pinned host memory (vqc_state_upload) and reads E and the gradient back
        (vqc_adjoint_grad).  Two state handles alternate, each on its own
        stream, so the upload of step i + 1's psi0 (copy engine) overlaps the
        gradient of step i (SMs), as a training loop double-buffers its inputs;
        the first upload is not overlapped.  Timed with CUDA events on both
        streams, from before the first upload to the end of the last gradient."""
        nbytes = host.numel() * host.element_size()
        streams = [torch.cuda.ExternalStream(lib.vqc_state_stream(p.handle), device=local_rank) for p in psis]

        def upload(p):
            _lib.check(lib.vqc_state_upload(p.handle, ctypes.c_void_p(host.data_ptr()), nbytes))

        def run(k):
            upload(psis[0])
            for i in range(k):
                if i + 1 < k:
                    upload(psis[(i + 1) % 2])
                V.energy_and_gradient(H, circuit, psis[i % 2])

        run(warmup)
        replicas.barrier()
        torch.cuda.synchronize()
        start = torch.cuda.Event(enable_timing=True)
        start.record(streams[0])
        streams[1].wait_event(start)
        run(steps)
        ends = []
        for st in streams:
            e = torch.cuda.Event(enable_timing=True)
            e.record(st)
            ends.append(e)
        torch.cuda.synchronize()
        ms = max(start.elapsed_time(e) for e in ends) / steps
        if world > 1:
            ms = replicas.max_over_ranks(ms, device="cuda")
            replicas.barrier()
        return ms

    psi32 = make_state(np.complex64)
    try:
        gpu_id = torch.cuda.get_device_properties(local_rank).uuid
        gpu_id = "GPU-" + str(gpu_id) if not str(gpu_id).startswith("GPU-") else str(gpu_id)
    except Exception:
        gpu_id = local_rank
    clocks = Clocks(gpu_id)
    clocks.start()
    ms, prof, energy, grads = timed(psi32, args.steps, args.warmup, profile=True)
    clk = clocks.stop()
    value = world * 1000.0 / ms

    # end to end through the public API with psi0 in pinned host memory
    ms_e2e = None
    if not args.no_e2e:
        host = torch.zeros(2 << N_QUBITS, dtype=torch.float32).pin_memory()
        host[0] = 1.0
        psi_b = make_state(np.complex64)
        ms_e2e = timed_e2e([psi32, psi_b], host, max(2, args.steps // 2), 2)
        del psi_b

    # the plain FP64 path, for the FP32-vs-FP64 speedup
    fp64 = None
    if not args.no_fp64:
        psi64 = make_state(np.complex128)
        ms64, prof64, energy64, grads64 = timed(psi64, max(1, args.steps // 2), 1, profile=True)
        del psi64
        fp64 = {"value": world * 1000.0 / ms64, "unit": UNIT, "ms_per_step": ms64, "fp32_speedup": ms64 / ms,
                "energy_rel_diff_fp32_vs_fp64": abs(energy - energy64) / abs(energy64),
                "grad_rel_diff_fp32_vs_fp64": float(np.linalg.norm(grads - grads64) / np.linalg.norm(grads64))}

    # measured FMA-pipe peaks: the compute roofline of the tile passes
    fma32 = _lib.fma_peak(local_rank, 0)
    fma64 = _lib.fma_peak(local_rank, 2)

    if rank != 0:
        return
    hbm, peak_kind = peaks()
    if fp64 is not None:
        fp64["kernels"] = kernel_rooflines(prof64, max(1, args.steps // 2), ms64, hbm, fma64)
        fp64["fma_peak_tflops_fp64"] = fma64
    dom = max(prof.items(), key=lambda kv: kv[1][1]) if prof else None  # largest total device time
    roof = None
    launches = sum(v[0] for k, v in prof.items() if not k.startswith("plan_")) if prof else 0
    if dom:
        name, (n, tot_ms, tot_bytes, tot_flops) = dom
        achieved = tot_bytes / (tot_ms * 1e-3) / 1e9
        roof = {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "peak_kind": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
                "bytes_per_launch": tot_bytes / n, "avg_launch_ms": tot_ms / n,
                "share_of_step": tot_ms / (ms * args.steps), "traffic": traffic_from_profiles(name),
                "compute": {"pipe": "FP32 FMA (packed fma.rn.f32x2)", "unit": "TFLOP/s",
                            "achieved": tot_flops / (tot_ms * 1e-3) / 1e12, "peak": fma32,
                            "frac": tot_flops / (tot_ms * 1e-3) / 1e12 / fma32 if fma32 else None,
                            "flops_per_launch": tot_flops / n,
                            "peak_kind": "measured on this GPU by vqc_fma_peak (calibration kernel)"}}
    cpu = None
    if world == 1 and not args.no_cpu:
        nthreads = os.cpu_count() or 1
        v, s = cpu_sample(nthreads, reps=8)
        cpu = {"value": v, "unit": UNIT, "cores": nthreads, "kind": "port",
               "sample": "8 x (2 rotations + 1 CRX forward/reverse sweep) + one XXZ key at n=26, FP32, scaled "
                         "to one gradient (%.1f s of CPU work)" % s,
               "extrapolation_check": cpu_full_check(nthreads)}
    secondary = None
    if world == 1 and not args.no_secondary:
        secondary = {"gates_n30": gates_record(30, 3, local_rank), "dm_n13": dm_record(13, local_rank),
                     "serve": serve_record(local_rank, requests=2000, rates=[1000.0], baseline_requests=100,
                                           memory_mib=args.serve_memory, slots=args.serve_slots)}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c64", "data": "synthetic (seeded angles, |0> input)",
            "config": config_dict(args),
            "e2e": None if ms_e2e is None else {
                "value": world * 1000.0 / ms_e2e, "unit": UNIT, "h2d_bytes_per_step": (1 << N_QUBITS) * 8,
                "d2h_bytes_per_step": packed.nparams * 8 + 16,
                "note": "psi0 uploaded from pinned host memory every step through vqc_state_upload, E and the "
                        "gradient read back by vqc_adjoint_grad; two state handles alternate so the next step's "
                        "upload overlaps the current gradient"},
            "fp64_plain": fp64,
            "energy": energy.real,
            "roofline": roof, "kernels": kernel_rooflines(prof, args.steps, ms, hbm, fma32),
            "gpu_launches": launches, "clocks": clk, "cpu_baseline": cpu, "secondary": secondary}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- secondary workloads
def _events(stream):
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def kernel_rooflines(prof, steps, ms_step, hbm, fma):
    """Per kernel class of the profile: launches, device time, algorithmic
    bytes, and for each class its HBM fraction (algorithmic bytes / time over
    the measured HBM peak) and, where it counts FMA-pipe flops, its fraction
    of the measured FMA peak `fma` (TFLOP/s)."""
    out = {}
    for k, v in (prof or {}).items():
        n, tms, tby = v[0], v[1], v[2]
        fl = v[3] if len(v) > 3 else 0.0
        rec = {"launches": n, "ms": tms, "bytes": tby}
        if tms > 0 and tby > 0:
            gbs = tby / (tms * 1e-3) / 1e9
            rec.update({"avg_launch_ms": tms / n, "GB/s": gbs, "frac_of_hbm": gbs / hbm,
                        "share_of_step": tms / (ms_step * steps)})
        if tms > 0 and fl > 0:
            tf = fl / (tms * 1e-3) / 1e12
            rec.update({"fma_pipe_TFLOP/s": tf, "frac_of_fma_peak": tf / fma if fma else None})
        out[k] = rec
    return out


def gates_record(n, steps, local_rank):
    """n qubits (30: 16 GiB in FP64, 8 GiB in FP32): per-gate-class HBM GB/s of
    single gates (algorithmic bytes over event time, fraction of the measured
    HBM peak), and the fused-block speedup of 10 layers of (U3 on every qubit,
    CZ brickwork, one Toffoli)."""
    import torch
    import vqcb200 as V
    from vqcb200 import _lib
    from vqcb200 import workloads as W
    torch.cuda.set_device(local_rank)
    lib = V.load()
    hbm, peak_kind = peaks()
    out = {"metric": "HBM GB/s per gate class and fused-block speedup, n=%d" % n, "unit": "GB/s",
           "config": {"workload": "10 x (U3 on every qubit, CZ brickwork, 1 Toffoli), n=%d" % n}, "classes": {}}
    spec = W.u3_cz_toffoli_spec(n, 10, SEED)
    circuit = W.to_circuit(spec)
    for dtype, name in ((np.complex128, "c128"), (np.complex64, "c64")):
        psi = V.StateVector(n, dtype=dtype, device=local_rank)
        V.apply(W.to_circuit(spec[:n]), psi)  # a dense state
        stream = torch.cuda.ExternalStream(lib.vqc_state_stream(psi.handle), device=local_rank)
        gates = {"u3_q1": V.U3Gate(1, 0.3, 0.2, 0.1), "u3_q%d" % n: V.U3Gate(n, 0.3, 0.2, 0.1),
                 "cz": V.CZGate(n // 2, n // 2 + 1), "toffoli": V.TOFFOLIGate(2, n - 1, n // 2),
                 "cnot": V.CNOTGate(3, n - 2), "crx": V.CRxGate(n - 3, 4, 0.4), "dense2q": V.QuantumGate((5, n - 4),
                 np.linalg.qr(np.random.default_rng(1).standard_normal((4, 4)) + 0j)[0])}
        res = {}
        for gname, g in gates.items():
            for _ in range(2):
                V.apply(g, psi)
            _lib.profile_enable(True)
            a, b = _events(stream)
            reps = max(1, steps)
            a.record(stream)
            for _ in range(reps):
                V.apply(g, psi)
            b.record(stream)
            b.synchronize()
            prof = _lib.profile_read()
            _lib.profile_enable(False)
            ms = a.elapsed_time(b) / reps
            (cls, (nl, tms, tby)), = [(k, v) for k, v in prof.items() if not k.startswith("plan_")]
            res[gname] = {"kernel": cls, "ms": ms, "algorithmic_bytes": tby / nl, "GB/s": tby / nl / (ms * 1e-3) / 1e9,
                          "frac_of_hbm": tby / nl / (ms * 1e-3) / 1e9 / hbm,
                          "full_pass_GB/s": 2 * (1 << n) * psi.dtype.itemsize / (ms * 1e-3) / 1e9}
        # the whole circuit: one by one vs fused
        times = {}
        for fuse in (False, True):
            V.apply(circuit, psi, fuse=fuse)
            a, b = _events(stream)
            a.record(stream)
            V.apply(circuit, psi, fuse=fuse)
            b.record(stream)
            b.synchronize()
            times["fused" if fuse else "unfused"] = a.elapsed_time(b)
        ngates = len(circuit)
        S = (1 << n) * psi.dtype.itemsize
        res["circuit"] = {"gates": ngates, "unfused_ms": times["unfused"], "fused_ms": times["fused"],
                          "fused_speedup": times["unfused"] / times["fused"],
                          "effective_GB/s_fused": ngates * 2 * S / (times["fused"] * 1e-3) / 1e9,
                          "note": "effective GB/s counts 2 x state bytes per gate; it can exceed the HBM roofline"}
        out["classes"][name] = res
        del psi
    out["peak"] = {"hbm_GB/s": hbm, "kind": peak_kind}
    return out


def dm_record(n, local_rank):
    """Density matrix of n qubits (13: 1 GiB complex128): seeded random pure
    state, 8 layers of U3 on every qubit + CNOT ladder as rho <- U rho
    U^dagger, partial trace over the top 4 qubits, basis probabilities."""
    import torch
    import vqcb200 as V
    from vqcb200 import workloads as W
    torch.cuda.set_device(local_rank)
    lib = V.load()
    hbm, _ = peaks()
    rng = np.random.default_rng(SEED)
    psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    psi /= np.linalg.norm(psi)
    spec = W.u3_cnot_spec(n, 8, SEED)
    circuit = W.to_circuit(spec)
    res = {}
    for fuse in (False, True):
        rho = V.DensityMatrix(V.StateVector(psi))
        V.apply(circuit, rho, fuse=fuse)  # warm-up
        rho = V.DensityMatrix(V.StateVector(psi))
        stream = torch.cuda.ExternalStream(lib.vqc_state_stream(rho.handle), device=local_rank)
        a, b = _events(stream)
        a.record(stream)
        V.apply(circuit, rho, fuse=fuse)
        b.record(stream)
        b.synchronize()
        res["fused" if fuse else "unfused"] = a.elapsed_time(b)
    sites = list(range(n - 3, n + 1))
    t0 = time.perf_counter()
    red = V.partial_tr(rho, sites)
    t_ptrace = time.perf_counter() - t0
    t0 = time.perf_counter()
    probs = V.probabilities(rho)
    t_probs = time.perf_counter() - t0
    S = (1 << (2 * n)) * 16
    per_gate = len(circuit) * 2 * S / (res["unfused"] * 1e-3) / 1e9
    return {"metric": "density-matrix circuit time, n=%d (rho %d MiB)" % (n, S >> 20), "unit": "ms",
            "config": {"workload": "8 x (U3 on every qubit + CNOT ladder) on rho, ptrace of the top 4 qubits, "
                                   "probabilities", "gates": len(circuit)},
            "circuit_ms_one_by_one": res["unfused"], "circuit_ms_fused": res["fused"],
            "fused_speedup": res["unfused"] / res["fused"],
            "one_by_one_GB/s_per_gate": per_gate, "one_by_one_frac_of_hbm": per_gate / hbm,
            "ptrace_ms_host_call": t_ptrace * 1e3, "probs_ms_host_call": t_probs * 1e3,
            "trace_of_reduced": float(np.trace(red).real), "sum_probs": float(probs.sum())}


def serve_record(local_rank, requests=2000, rates=(500.0, 1000.0, 2000.0, 4000.0), baseline_requests=200,
                 memory_mib=16384, slots=512):
    """Serving stream (continuous batching): requests with n ~ U{10..22},
    depth ~ U{2..12} layers of the hardware-efficient ansatz (RY, RZ on every
    qubit + CNOT ladder), angles ~ U[0, 2 pi), half energy only and half energy
    + gradient, transverse-field Ising H with g ~ U[0.2, 1.5]; Poisson arrivals
    at each offered rate.  FP32 states, FP64 accumulation.  Baseline: one
    request at a time through the plain FP64 single-request path, same arrival
    sequence."""
    import threading

    import torch
    import vqcb200 as V
    from vqcb200 import workloads as W
    from vqcb200.circuit import Packed
    from vqcb200.serve import Server
    torch.cuda.set_device(local_rank)
    V.load()
    rng = np.random.default_rng(SEED)
    nreq = requests
    reqs = []
    for i in range(nreq):
        n = int(rng.integers(10, 23))
        layers = int(rng.integers(2, 13))
        th = rng.uniform(0, 2 * np.pi, layers * 2 * n)
        g = float(rng.uniform(0.2, 1.5))
        want = bool(rng.integers(0, 2))
        c = W.to_circuit(W.hea_spec(n, layers, th))
        H = W.to_operator(W.tfim_spec(n, g))
        arr, nt = H.packed()
        reqs.append((n, Packed(c, with_params=want), arr, nt, want, c, H))

    def stream(rate, count):
        """Submit `count` requests with Poisson arrivals at `rate`/s; latencies in s."""
        arrivals = np.cumsum(np.random.default_rng(int(rate)).exponential(1.0 / rate, count))
        lat = [None] * count
        with Server(device=local_rank, dtype=np.complex64, memory_bytes=memory_mib << 20,
                    max_active=slots, planner_threads=4) as srv:
            tickets = [None] * count
            done = threading.Event()

            def collector():
                for i in range(count):
                    while tickets[i] is None:
                        time.sleep(0.0002)
                    e, gr, l = srv.wait(tickets[i], timeout=600)
                    lat[i] = l
                done.set()
            th = threading.Thread(target=collector)
            th.start()
            t0 = time.perf_counter()
            for i in range(count):
                dt = arrivals[i] - (time.perf_counter() - t0)
                if dt > 0:
                    time.sleep(dt)
                n, p, arr, nt, want = reqs[i % nreq][:5]
                tickets[i] = srv.submit_packed(n, p, arr, nt, want)
            done.wait()
            makespan = time.perf_counter() - t0
            th.join()
            st = srv.stats()
            tm = srv.timing()
            lt = srv.loop_timing()
        lat = np.array(lat)
        return {"rate_offered": rate, "requests": count, "throughput": count / makespan,
                "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
                "mean_batch": st["request_steps"] / max(st["launches"], 1), "loop_iterations": st["iterations"],
                "phases_ms": {k: round(v * 1e3, 3) for k, v in tm.items()},
                "busy_iteration_ms": {(k if k == "iterations" else k[:-2]): (v if k == "iterations" else round(v * 1e3, 4))
                                      for k, v in lt.items()}}

    # baseline: plain FP64, one request at a time, in arrival order
    def baseline(rate, count):
        arrivals = np.cumsum(np.random.default_rng(int(rate)).exponential(1.0 / rate, count))
        lat = []
        t0 = time.perf_counter()
        for i in range(count):
            dt = arrivals[i] - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            n, p, arr, nt, want, c, H = reqs[i % nreq]
            psi0 = V.StateVector(n, dtype=np.complex128, device=local_rank)
            if want:
                V.energy_and_gradient(H, c, psi0)
            else:
                V.expectation(H, c * psi0)
            lat.append(time.perf_counter() - t0 - arrivals[i])
        makespan = time.perf_counter() - t0
        lat = np.array(lat)
        return {"rate_offered": rate, "requests": count, "throughput": count / makespan,
                "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3)}

    # warm-up (kernel loads, allocator pools, and the batch kernels compiled
    # per pass structure: most of the workload's structures appear in it)
    stream(400.0, min(800, nreq))
    results = [stream(float(r), nreq) for r in rates]
    # the baseline's warm-up: one request of every (size, kind), so that the
    # kernels compiled per structure (the Pauli passes of 2^20+ amplitudes) are
    # built before it is timed
    seen = set()
    for n, p, arr, nt, want, c, H in reqs:
        if (n, want) in seen:
            continue
        seen.add((n, want))
        psi0 = V.StateVector(n, dtype=np.complex128, device=local_rank)
        if want:
            V.energy_and_gradient(H, c, psi0)
        else:
            V.expectation(H, c * psi0)
    # service rate of the one-at-a-time baseline: back-to-back requests
    base_sat = baseline(1e6, min(baseline_requests, nreq))
    base = [baseline(float(r), min(baseline_requests, nreq)) for r in rates if r < 0.9 * base_sat["throughput"]]
    return {"metric": "serving throughput and p50/p99 latency (continuous batching, FP32 states)",
            "unit": "requests/s",
            "config": {"workload": "n~U{10..22}, 2..12 HEA layers, 50% energy / 50% energy+gradient, TFIM "
                                   "g~U[0.2,1.5], Poisson arrivals", "requests_per_rate": nreq,
                       "memory_budget_MiB": memory_mib, "slots": slots},
            "served": results, "baseline_fp64_one_at_a_time": {"saturated": base_sat, "at_rates": base}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-fp64", action="store_true", help="skip the plain FP64 comparison")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end (host buffers) measurement")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the secondary records (gate classes at n=30, density matrix n=13, serving)")
    ap.add_argument("--requests", type=int, default=2000, help="serve: requests per rate")
    ap.add_argument("--rates", default="500,1000,2000,4000", help="serve: offered rates (requests/s)")
    ap.add_argument("--baseline-requests", type=int, default=200, help="serve: requests of the FP64 baseline")
    ap.add_argument("--serve-memory", type=int, default=16384, help="serve: device memory budget (MiB)")
    ap.add_argument("--serve-slots", type=int, default=512, help="serve: requests in flight at most")
    ap.add_argument("--workload", default="adjoint", choices=["adjoint", "gates_n30", "dm_n13", "serve", "fma_peak"],
                    help="adjoint (the headline) or a secondary workload")
    ap.add_argument("--qubits", type=int, default=None,
                    help="state size (default 26, the headline; smaller sizes are for profiling captures)")
    args = ap.parse_args()
    if args.qubits is not None and args.workload == "adjoint":
        global N_QUBITS
        N_QUBITS = args.qubits
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload == "gates_n30":
        print(json.dumps(gates_record(args.qubits or 30, args.steps, local_rank)), flush=True)
        return
    if args.workload == "dm_n13":
        print(json.dumps(dm_record(args.qubits or 13, local_rank)), flush=True)
        return
    if args.workload == "serve":
        print(json.dumps(serve_record(local_rank, args.requests, [float(r) for r in args.rates.split(",")],
                                      args.baseline_requests, args.serve_memory, args.serve_slots)), flush=True)
        return
    if args.workload == "fma_peak":
        import vqcb200 as V
        from vqcb200 import _lib
        V.load()
        print(json.dumps({"metric": "measured FMA-pipe peak", "unit": "TFLOP/s",
                          "fp32_packed": _lib.fma_peak(local_rank, 0), "fp32_scalar": _lib.fma_peak(local_rank, 1),
                          "fp64": _lib.fma_peak(local_rank, 2)}), flush=True)
        return
    if world > 1:
        import torch
        from vqcb200 import replicas
        torch.cuda.set_device(local_rank)
        replicas.init_from_env("nccl")
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
