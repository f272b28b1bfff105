#!/usr/bin/env python
"""Benchmark: time per 30-qubit depth-40 random circuit on one B200.

Workload: the U(theta,phi,lambda)-per-qubit + CX brick-wall circuit, 30
qubits, 40 layers (1200 U + 580 CX), seed 1234, complex64 state (8 GiB,
larger than L2, so no flush is needed between steps), greedy fusion into
k<=6-qubit blocks applied on the tensor cores (tcgen05, 3xFP16).  A step =
ket::run semantics: reset to |0...0> and apply the whole circuit.

Lines printed by rank 0 (one JSON line):
  value        ms per circuit (device time, CUDA events on the state's
               stream, K steps between barriers, max over ranks, / N for
               the aggregate over N replicas)
  e2e          the same through the C ABI with host buffers (ketgpu_run:
               ops from host, the 2^30 amplitudes back into a host
               complex128 buffer)
  roofline     the dense-block kernel: algorithmic bytes per launch / its
               mean CUDA-event duration, against MEASURED_PEAKS.json HBM
  cpu_baseline ket itself (oracle/_ref/libket_ref.so, all host threads): one
               full ket::run of the same circuit, timed; its complex128
               state gives checks.max_abs_vs_ket / fidelity_vs_ket
  --impl reference   full ket::run calls, one per step, as many as fit
               --reference-budget seconds; prints its own line.
"""
from __future__ import annotations

import argparse
import ctypes as ct
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_QUBITS, DEPTH, SEED = 30, 40, 1234
METRIC = "time per 30q circuit"

# DRAM bytes (read + write) of one fused_tc_kernel<k> launch on a 2^26
# complex64 state, from ncu (dram__bytes_read.sum + dram__bytes_write.sum,
# one dense block of the 26-qubit workload `--workload kernels26`; see
# profiles/fused_tc_kernel6_26q.md).  A launch streams the state once, so the
# figure scales with 2^n.
TC_TRAFFIC_BYTES_26Q = {5: 536.966400e6 + 477.739776e6, 6: 537.047552e6 + 477.192448e6}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            if len(r) >= 9:
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def ket_full_run(ops, keep_state=False):
    """One full ket::run of the circuit (oracle/_ref/libket_ref.so: ket built
    from its own sources, set_num_threads(0) = every host thread), timed
    around the call alone.  Returns (seconds, threads, state or None)."""
    from oracle.oracle import Reference
    R = Reference()
    R.set_num_threads(0)
    threads = int(R.num_threads())
    if keep_state:
        secs, st = R.run_timed_state(N_QUBITS, ops)
        return secs, threads, st
    return R.run_timed(N_QUBITS, ops), threads, None


def host_cpu():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def init_dist(n_gpus):
    """One process per GPU (torchrun); replicas share nothing but timings."""
    from ket_b200 import replicas
    if n_gpus > 1 or "RANK" in os.environ:
        return replicas.init("nccl")
    return 0, 1, 0


def barrier_max(x, world):
    from ket_b200 import replicas
    return replicas.max_over_ranks(x, device="cuda") if world > 1 else x


def barrier(world):
    from ket_b200 import replicas
    if world > 1:
        replicas.barrier()


def run_reference_arm(args):
    """ket's own CPU path on this workload: full ket::run calls of the 30-qubit
    depth-40 brick wall (complex128, every host thread), one per step, as many
    steps as fit in --reference-budget seconds (at least one).  Loads only
    ket built from its sources (oracle/_ref) -- not the B200 package.  Under
    torchrun only rank 0 runs; the other ranks exit without work."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    from oracle.oracle import Reference, brickwork_ops
    R = Reference()
    R.set_num_threads(0)
    threads = int(R.num_threads())
    ops = brickwork_ops(N_QUBITS, DEPTH, SEED, R.uniforms)
    times = []
    t_start = time.perf_counter()
    while len(times) < max(1, args.steps):
        times.append(R.run_timed(N_QUBITS, ops))
        if time.perf_counter() - t_start + times[-1] > args.reference_budget:
            break
    v = statistics.median(times) * 1e3
    sample = (f"{len(times)} full ket::run call(s) of the 30-qubit depth-40 brick wall (1200 U + 580 CX, "
              f"complex128, 16 GiB state) through ket's public API (oracle/_ref/libket_ref.so built from "
              f"ket's sources), set_num_threads(0) = {threads} threads on {host_cpu()}; each call timed "
              f"alone: {', '.join(f'{t:.1f} s' for t in times)}")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "ms/circuit", "n_gpus": args.gpus,
        "steps": len(times), "warmup": 0, "steps_requested": args.steps, "warmup_requested": args.warmup,
        "ms_per_step": v, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "c128", "data": "synthetic",
        "config": {"workload": "random U+CX brick wall, 30 qubits, depth 40, seed 1234", "global_batch": 1,
                   "seq_len": None, "parallelism": "host threads",
                   "note": "a step is one full ket::run (about 7-8 minutes on 16 threads), so the run stops "
                           "after the steps that fit the time budget and reports the steps it ran; no "
                           "warm-up step (each call allocates its own state)"},
        "cpu_baseline": {"value": v, "unit": "ms/circuit", "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": v, "unit": "ms/circuit", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_sample33(args):
    """33-qubit complex64 QFT-pattern + GHZ + Rz circuit, then 10^6 shots
    from one FP64 CDF tree, counts checked bit-exact against the CPU
    sampler fed the same std::mt19937{42} draws."""
    import ket_b200 as ket
    from ket_b200 import _lib
    from ket_b200.workloads import qft_ghz_rz
    import torch
    lib = _lib.lib
    n = args.qubits if args.qubits != N_QUBITS else 33
    shots = args.shots
    circ = qft_ghz_rz(n, seed=7)
    ops = circ.to_ops()
    plan = ket.Plan(n, ops, ket.make_options("c64", args.fusion, args.k, True))
    st = plan.stats()
    state = ket.DeviceState(n, "c64")
    stream = torch.cuda.ExternalStream(lib.ketgpu_state_stream(state.handle))
    u = ket.uniforms(42, shots)
    out = np.empty(shots, dtype=np.uint64)

    def step():
        _lib.check(lib.ketgpu_state_reset(state.handle))
        _lib.check(lib.ketgpu_plan_execute(plan._h, state.handle))
        _lib.check(lib.ketgpu_sample(state.handle, u.ctypes.data, shots, out.ctypes.data))

    for _ in range(args.warmup):
        step()
    circ_ms, samp_ms, tot_ms = [], [], []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        _lib.check(lib.ketgpu_state_reset(state.handle))
        e0.record(stream)
        _lib.check(lib.ketgpu_plan_execute(plan._h, state.handle))
        e1.record(stream)
        _lib.check(lib.ketgpu_state_synchronize(state.handle))
        t1 = time.perf_counter()
        _lib.check(lib.ketgpu_sample(state.handle, u.ctypes.data, shots, out.ctypes.data))
        t2 = time.perf_counter()
        circ_ms.append(e0.elapsed_time(e1))
        samp_ms.append((t2 - t1) * 1e3)
        tot_ms.append((t2 - t0) * 1e3)
    line = {"metric": "33q circuit + 1e6 shots", "value": statistics.median(tot_ms), "unit": "ms",
            "higher_is_better": False, "circuit_ms": statistics.median(circ_ms),
            "sampling_ms_e2e": statistics.median(samp_ms), "shots": shots, "passes": int(st["n_passes"]),
            "gates": int(st["n_gates"]), "tensor_passes": int(st["n_tensor"]),
            "hbm_gbs_circuit": st["bytes"] / (statistics.median(circ_ms) * 1e-3) / 1e9}
    if not args.no_checks:
        from oracle.oracle import Oracle
        O = Oracle()
        host = state.to_numpy_raw()
        t0 = time.perf_counter()
        cpu = O.sample_tree(n, host, u)
        t_cpu = time.perf_counter() - t0
        seq = O.measure_sequential(n, host, u)
        counts_gpu = np.unique(out, return_counts=True)
        counts_cpu = np.unique(cpu, return_counts=True)
        line["checks"] = {
            "indices_bit_exact_vs_cpu_tree_sampler": bool(np.array_equal(out, cpu)),
            "counts_bit_exact": bool(np.array_equal(counts_gpu[0], counts_cpu[0]) and
                                     np.array_equal(counts_gpu[1], counts_cpu[1])),
            "distinct_outcomes": int(len(counts_gpu[0])),
            "draws_differing_from_sequential_scan": int((out != seq).sum()),
            "norm": float(state.norm()),
        }
        line["cpu_baseline"] = {"value": t_cpu * 1e3, "unit": "ms", "cores": 1, "kind": "port",
                                "sample": f"oracle ko_sample_tree over the downloaded 2^{n} complex64 state, "
                                          f"{shots} draws (the same fixed tree, one thread)"}
    print(json.dumps(line), flush=True)
    state.close()
    plan.close()


def _adjoint_blocks(n, ops, pidx, ckpt):
    """Number of tile blocks of the tiled adjoint sweep (complex64)."""
    from ket_b200 import _lib
    p = np.ascontiguousarray(pidx, dtype=np.int32)
    length = ct.c_uint64()
    _lib.check(_lib.lib.ketgpu_adjoint_plan_describe(n, ops.ctypes.data, len(ops), p.ctypes.data, _lib.C64, ckpt,
                                                     None, 0, ct.byref(length)))
    out = np.zeros(length.value, dtype=np.int32)
    _lib.check(_lib.lib.ketgpu_adjoint_plan_describe(n, ops.ctypes.data, len(ops), p.ctypes.data, _lib.C64, ckpt,
                                                     out.ctypes.data, length.value, ct.byref(length)))
    return int(out[0])


def run_adjoint24(args):
    """Adjoint gradients: 24-qubit, 8-layer Ry/Rz + CX-ring ansatz (384
    parameters), 64 random Pauli strings, a batch of 64 parameter sets;
    complex64 states, FP64 accumulation, checkpoints every 2 layers."""
    import ket_b200 as ket
    from ket_b200.autograd import adjoint_expval
    from ket_b200.workloads import random_pauli_sum, variational_ansatz
    n = args.qubits if args.qubits != N_QUBITS else 24
    layers, batch = 8, args.batch
    circ, pidx = variational_ansatz(n, layers)
    npar = int((pidx >= 0).sum())
    ham = random_pauli_sum(n, 64, seed=11)
    theta = np.random.default_rng(12).uniform(-np.pi, np.pi, (batch, npar))
    for _ in range(args.warmup):
        adjoint_expval(circ, pidx, theta[:2], ham, "c64", 2)
    ts = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        vals, grads = adjoint_expval(circ, pidx, theta, ham, "c64", 2)
        ts.append(time.perf_counter() - t0)
    t = statistics.median(ts)
    # algorithmic HBM bytes per batch: per tile block and set, the forward
    # reads and writes psi, the reverse psi and lambda; lambda = H psi reads
    # psi and writes lambda once per set (its gathers beyond that are L2 hits)
    blocks = _adjoint_blocks(n, circ.to_ops(), pidx, 2)
    state = 8 * 2 ** n
    byts = batch * (blocks * (2 * state + 4 * state) + 2 * state)
    peak, peak_kind = peaks()
    line = {"metric": "adjoint gradients/s (24q, 8 layers, 384 params, 64 Pauli terms, batch 64)",
            "value": batch * npar / t, "unit": "gradients/s", "higher_is_better": True,
            "seconds_per_batch": t, "batch": batch, "params": npar,
            "roofline": {"bound": "hbm", "achieved": byts / t / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": byts / t / 1e9 / peak, "peak_source": peak_kind, "traffic": None,
                         "bytes_per_batch": byts, "tile_blocks": blocks}}
    if not args.no_checks:
        t0 = time.perf_counter()
        vpg, gpg = adjoint_expval(circ, pidx, theta, ham, "c64", 2, method="per_gate")
        t_pg = time.perf_counter() - t0
        v128, g128 = adjoint_expval(circ, pidx, theta[:2], ham, "c128", 2)
        line["checks"] = {"max_abs_value_vs_fp64_adjoint": float(np.abs(vals[:2] - v128).max()),
                          "max_abs_grad_vs_fp64_adjoint": float(np.abs(grads[:2] - g128).max()),
                          "per_gate_sweep_seconds_per_batch": t_pg,
                          "per_gate_gradients_per_s": batch * npar / t_pg,
                          "max_abs_grad_tiled_vs_per_gate": float(np.abs(grads - gpg).max())}
        # central finite differences (h = 1e-3) of the complex128 GPU forward
        h = 1e-3
        ks = np.random.default_rng(13).choice(npar, 6, replace=False)
        fd_err = 0.0
        ops = circ.to_ops()
        for k in ks:
            vals_fd = []
            for sgn in (1, -1):
                th = theta[0].copy()
                th[k] += sgn * h
                o = ops.copy()
                for i, p in enumerate(pidx):
                    if p >= 0:
                        o[i]["p"][0] = th[p]
                d = ket.DeviceState(n, "c128")
                d.apply(o, ket.make_options("c128", "greedy", 5, True))
                vals_fd.append(d.expval(ham))
                d.close()
            fd = (vals_fd[0] - vals_fd[1]) / (2 * h)
            fd_err = max(fd_err, abs(fd - g128[0][k]))
        line["checks"]["max_abs_fd_minus_adjoint_fp64"] = fd_err
        # the reference's only route to a gradient: two ket::run + expval per parameter
        try:
            from oracle.oracle import Reference
            R = Reference()
            R.set_num_threads(0)
            o = ops.copy()
            for i, p in enumerate(pidx):
                if p >= 0:
                    o[i]["p"][0] = theta[0][p]
            t0 = time.perf_counter()
            stv = R.run(n, o)
            t1 = time.perf_counter()
            R.expval_sum(n, stv, ham)
            t2 = time.perf_counter()
            per_grad = 2 * (t2 - t0)
            line["cpu_baseline"] = {"value": 1.0 / per_grad, "unit": "gradients/s", "cores": R.num_threads(),
                                    "kind": "reference",
                                    "sample": f"one ket::run ({t1 - t0:.2f} s) + ket::expval(State, PauliSum) "
                                              f"({t2 - t1:.2f} s) at {n} qubits; a central difference needs two"}
        except Exception as ex:
            line["cpu_baseline"] = {"value": None, "sample": f"unavailable: {ex}"}
    print(json.dumps(line), flush=True)


def run_kernels26(args):
    """Every kernel family once on a 26-qubit state (1 GiB complex128 /
    512 MiB complex64, larger than L2): per-gate pair / phase kernels and
    shared-memory runs (plain method, both precisions), FP64 dense blocks,
    tensor-core blocks at k = 4, 5, 6, a diagonal run, batched Pauli terms,
    the sampling tree and descent, and the cost model's forward, backward
    and Adam kernels.  Prints each pass kind's time and algorithmic GB/s
    (CUDA events, ketgpu_plan_execute_timed); the profile summaries under
    profiles/ come from ncu runs of this workload."""
    import ket_b200 as ket
    from ket_b200.planner import CostModel
    from ket_b200.workloads import qft_ghz_rz, random_mixed, random_pauli_sum
    n = args.qubits if args.qubits != N_QUBITS else 26
    kinds = {0: "pair", 1: "phase", 2: "dense_block", 3: "norm", 4: "diagonal_run", 5: "shared_run"}
    out = {"metric": "per-kernel time and algorithmic GB/s, 26 qubits", "qubits": n, "passes": {}}
    circ = random_mixed(n, 6, seed=5)
    ops = circ.to_ops()
    cases = [("c64", "none", 5, True), ("c128", "none", 5, True), ("c128", "greedy", 5, True),
             ("c64", "greedy", 4, True), ("c64", "greedy", 5, True), ("c64", "greedy", 6, True)]
    for prec, fusion, k, tc in cases:
        plan = ket.Plan(n, ops, ket.make_options(prec, fusion, k, tc))
        st = ket.DeviceState(n, prec)
        ms = np.zeros(int(plan.stats()["n_passes"]), dtype=np.float32)
        from ket_b200 import _lib
        for _ in range(max(1, args.warmup)):
            st.reset()
            _lib.check(_lib.lib.ketgpu_plan_execute_timed(plan._h, st.handle, ms.ctypes.data))
        agg = {}
        for i in range(len(ms)):
            info = plan.pass_info(i)
            key = f"{prec}/{fusion}/k{k}/{kinds[info['kind']]}" + (f"/k{info['k']}" if info["kind"] == 2 else "")
            a = agg.setdefault(key, [0, 0.0, 0.0])
            a[0] += 1
            a[1] += float(ms[i])
            a[2] += info["bytes"]
        for key, (cnt, t, b) in agg.items():
            out["passes"][key] = {"launches": cnt, "ms": t, "gbs": b / (t * 1e-3) / 1e9 if t > 0 else None}
        st.close()
        plan.close()
    # diagonal run (QFT pattern) and reductions on one complex64 state
    d = ket.run_device(qft_ghz_rz(n, seed=7), options=ket.make_options("c64", "greedy", 5, True))
    ham = random_pauli_sum(n, 64, seed=11)
    t0 = time.perf_counter()
    d.expval(ham)
    out["expval_64_terms_ms_e2e"] = (time.perf_counter() - t0) * 1e3
    t0 = time.perf_counter()
    d.sample_seeded(42, 10 ** 6)
    out["sample_1e6_ms_e2e"] = (time.perf_counter() - t0) * 1e3
    d.close()
    # cost model: forward on 4096 rows, one gradient evaluation, 200 Adam steps
    m = CostModel(seed=3)
    x = np.random.default_rng(1).standard_normal((4096, 48)).astype(np.float32)
    y = np.random.default_rng(2).standard_normal(4096).astype(np.float32)
    m.forward(x)
    m.gradients(x, y)
    m.train(x, y, steps=200, minibatch=512)
    m.close()
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--reference-budget", type=float, default=600.0,
                    help="seconds of full ket::run calls in --impl reference (at least one call)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-checks", action="store_true")
    ap.add_argument("--fusion", default="greedy")
    ap.add_argument("--k", type=int, default=6)
    ap.add_argument("--qubits", type=int, default=N_QUBITS, help="smaller cases for profiling only")
    ap.add_argument("--depth", type=int, default=DEPTH)
    ap.add_argument("--workload", default="circuit30", choices=["circuit30", "sample33", "adjoint24", "kernels26"])
    ap.add_argument("--shots", type=int, default=1000000)
    ap.add_argument("--batch", type=int, default=64)
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "sample33":
        return run_sample33(args)
    if args.workload == "adjoint24":
        return run_adjoint24(args)
    if args.workload == "kernels26":
        return run_kernels26(args)

    rank, world, local = init_dist(args.gpus)
    import ket_b200 as ket
    from ket_b200 import _lib
    from ket_b200.workloads import random_brickwork
    lib = _lib.lib

    nq = args.qubits
    circ = random_brickwork(nq, args.depth, SEED)
    ops = circ.to_ops()
    opt = ket.make_options("c64", args.fusion, args.k, True)
    plan = ket.Plan(nq, ops, opt)
    stats = plan.stats()
    npass = int(stats["n_passes"])
    info = []
    for i in range(npass):
        kind, k, tc, b = ct.c_int32(), ct.c_int32(), ct.c_int32(), ct.c_double()
        _lib.check(lib.ketgpu_plan_pass_info(plan._h, i, ct.byref(kind), ct.byref(k), ct.byref(tc), ct.byref(b)))
        info.append((kind.value, k.value, tc.value, b.value))
    state = ket.DeviceState(nq, "c64")
    import torch
    stream = torch.cuda.ExternalStream(lib.ketgpu_state_stream(state.handle))
    pass_ms = np.zeros(npass, dtype=np.float32)

    def step(timed_passes=None):
        _lib.check(lib.ketgpu_state_reset(state.handle))
        if timed_passes is not None:
            _lib.check(lib.ketgpu_plan_execute_timed(plan._h, state.handle, timed_passes.ctypes.data))
        else:
            _lib.check(lib.ketgpu_plan_execute(plan._h, state.handle))

    for _ in range(args.warmup):
        step()
    _lib.check(lib.ketgpu_state_synchronize(state.handle))
    # per-pass timing (its own sweep, so the headline region has no extra events)
    per_pass = []
    for _ in range(2):
        step(pass_ms)
        per_pass.append(pass_ms.copy())
    per_pass = np.mean(per_pass, axis=0)

    barrier(world)
    torch.cuda.synchronize()
    clk = Clocks(local) if rank == 0 else None
    launches0 = ket.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    _lib.check(lib.ketgpu_state_synchronize(state.handle))
    torch.cuda.synchronize()
    ms_total = e0.elapsed_time(e1)
    launches = ket.launch_count() - launches0
    clocks = clk.stop() if clk else None
    ms_total = barrier_max(ms_total, world)
    ms_step = ms_total / args.steps
    value = ms_step / world  # aggregate: N circuits per step over N replicas

    # accuracy of the timed state against the complex128 path (FP64 SIMT
    # blocks, itself pinned to ket's complex128 ket::run at 1e-12 by the
    # tests), and the plain per-gate GPU method for the fusion speed-up
    checks = {"norm": state.norm()}
    if not args.no_checks:
        ref = ket.DeviceState(nq, "c128")
        ref_plan = ket.Plan(nq, ops, ket.make_options("c128", "greedy", 5, True))
        ref_plan.execute(ref)
        cmp = state.compare(ref)
        checks.update({"max_abs_vs_c128": cmp["max_abs"], "fidelity_vs_c128": cmp["fidelity"],
                       "fidelity_unnormalised_vs_c128": cmp["fidelity_unnormalised"]})
        ref.close()
        ref_plan.close()
        un_plan = ket.Plan(nq, ops, ket.make_options("c64", "none"))
        un_ms = []
        for _ in range(2):
            _lib.check(lib.ketgpu_state_reset(state.handle))
            a0 = torch.cuda.Event(enable_timing=True)
            a1 = torch.cuda.Event(enable_timing=True)
            a0.record(stream)
            _lib.check(lib.ketgpu_plan_execute(un_plan._h, state.handle))
            a1.record(stream)
            _lib.check(lib.ketgpu_state_synchronize(state.handle))
            un_ms.append(a0.elapsed_time(a1))
        checks["unfused_ms"] = min(un_ms)
        checks["speedup_vs_unfused"] = min(un_ms) / ms_step
        un_plan.close()
        # the same circuit planned with blocks of one qubit fewer (more
        # passes): device time per circuit, best of 3
        kalt = args.k - 1 if args.k > 4 else args.k + 1
        alt_plan = ket.Plan(nq, ops, ket.make_options("c64", args.fusion, kalt, True))
        alt_ms = []
        for _ in range(3):
            _lib.check(lib.ketgpu_state_reset(state.handle))
            a0 = torch.cuda.Event(enable_timing=True)
            a1 = torch.cuda.Event(enable_timing=True)
            a0.record(stream)
            _lib.check(lib.ketgpu_plan_execute(alt_plan._h, state.handle))
            a1.record(stream)
            _lib.check(lib.ketgpu_state_synchronize(state.handle))
            alt_ms.append(a0.elapsed_time(a1))
        checks[f"k{kalt}_plan_ms"] = min(alt_ms)
        checks[f"k{kalt}_plan_passes"] = int(alt_plan.stats()["n_passes"])
        alt_plan.close()

    # dense-block kernel roofline (tensor-core passes)
    tc_idx = [i for i, x in enumerate(info) if x[0] == 2 and x[2] == 1]
    peak, peak_kind = peaks()
    roof = None
    if tc_idx:
        # the dominant kernel: the block size most of the tensor-core passes have
        ks = [info[i][1] for i in tc_idx]
        kdom = max(set(ks), key=ks.count)
        dom = [i for i in tc_idx if info[i][1] == kdom]
        dur = float(np.mean(per_pass[dom]))
        byts = float(np.mean([info[i][3] for i in dom]))
        ach = byts / (dur * 1e-3) / 1e9
        traffic = TC_TRAFFIC_BYTES_26Q.get(kdom)
        roof = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                "peak_source": peak_kind, "traffic": traffic * 2.0 ** (nq - 26) if traffic else None,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch at 26 qubits, "
                                  "scaled by 2^(n-26)", "kernel": f"fused_tc_kernel<{kdom}>",
                "bytes_per_launch": byts, "mean_launch_ms": dur, "launches_per_step": len(dom),
                "tensor_passes_all_k": len(tc_idx),
                "all_tensor_passes_gbs": float(np.mean([info[i][3] / (per_pass[i] * 1e-3) / 1e9 for i in tc_idx]))}
    other = [i for i in range(npass) if i not in tc_idx]
    pass_summary = {
        "dense_tc_ms": float(per_pass[tc_idx].sum()) if tc_idx else 0.0,
        "per_gate_ms": float(per_pass[other].sum()) if other else 0.0,
        "hbm_gbs_all_passes": float(stats["bytes"] / (per_pass.sum() * 1e-3) / 1e9),
    }
    # dense blocks by producer / epilogue form (tensor copy or cp.async,
    # direct or staged stores): count and mean GB/s of algorithmic bytes
    forms = {}
    for i in tc_idx:
        f = plan.pass_tc_form(i)
        key = ("tensor_copy" if f["tma_dims"] else "cp_async") + ("_direct" if f["direct"] else "_staged")
        forms.setdefault(key, []).append(info[i][3] / (per_pass[i] * 1e-3) / 1e9)
    pass_summary["dense_tc_by_form"] = {k: {"blocks": len(v), "mean_gbs": float(np.mean(v))}
                                        for k, v in sorted(forms.items())}

    # e2e through the C ABI with host buffers
    e2e = None
    if args.e2e_steps > 0:
        out = np.empty(1 << nq, dtype=np.complex128)
        ops_pinned = ops.copy()
        ts, profs = [], []
        prof = np.zeros(6)
        for i in range(args.e2e_steps + 1):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            _lib.check(lib.ketgpu_run(nq, ops_pinned.ctypes.data, len(ops_pinned), ct.byref(opt),
                                      out.ctypes.data))
            t1 = time.perf_counter()
            _lib.check(lib.ketgpu_run_last_profile(prof.ctypes.data))
            if i > 0:
                ts.append((t1 - t0) * 1e3)
                profs.append(prof.copy())
        e2e_ms = barrier_max(statistics.median(ts), world) / world
        mat_bytes = int(stats["n_tensor"]) * 2 * 64 * 64 * 4
        med = np.median(np.array(profs), axis=0)
        e2e = {"value": e2e_ms, "unit": "ms/circuit", "h2d_bytes_per_step": int(ops.nbytes) + mat_bytes,
               "d2h_bytes_per_step": (1 << nq) * 8,
               "breakdown_ms": {"plan": med[0], "state_reset": med[1], "execute": med[2], "download": med[3],
                                "download_copy_wait": med[4], "download_widen_own_share": med[5],
                                "calls_ms": ts},
               "host": {"cpu": host_cpu(), "threads": os.cpu_count()},
               "note": "ketgpu_run: host ops in, 2^30 amplitudes out to a host complex128 buffer; "
                       "breakdown = host wall time per phase (ketgpu_run_last_profile), median of the timed calls"}
        del out

    # ket itself: one full ket::run of the same circuit on every host thread,
    # timed as the CPU baseline; its complex128 state is the FP64 oracle for
    # the accuracy of the timed complex64 state
    cpu = None
    full_size = nq == N_QUBITS and args.depth == DEPTH
    if rank == 0 and world == 1 and not args.no_cpu_baseline and full_size:
        try:
            secs, threads, ket_state = ket_full_run(ops, keep_state=not args.no_checks)
            cpu = {"value": secs * 1e3, "unit": "ms/circuit", "cores": threads, "kind": "reference",
                   "sample": f"one full ket::run of the same 30-qubit depth-40 circuit (complex128) through "
                             f"ket's public API (oracle/_ref/libket_ref.so built from ket's sources), "
                             f"set_num_threads(0) = {threads} threads on {host_cpu()}, timed around the call"}
            if ket_state is not None:
                kst = ket.DeviceState(nq, "c128")
                kst.from_numpy(ket_state)
                del ket_state
                step()  # the timed plan again: its state is bit-identical to every timed step
                cmp = state.compare(kst)
                checks.update({"max_abs_vs_ket": cmp["max_abs"], "fidelity_vs_ket": cmp["fidelity"],
                               "fidelity_unnormalised_vs_ket": cmp["fidelity_unnormalised"],
                               "oracle": "ket::run complex128 state of the same circuit"})
                kst.close()
        except Exception as ex:  # the reference build may be absent
            cpu = {"value": None, "unit": "ms/circuit", "cores": None, "kind": "reference",
                   "sample": f"unavailable: {ex}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "ms/circuit", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "c64", "data": "synthetic",
            "config": {"workload": f"random U+CX brick wall, {nq} qubits, depth {args.depth}, seed {SEED}, "
                                   f"complex64, {args.fusion} fusion k<={args.k} on tcgen05 3xFP16",
                       "global_batch": world, "seq_len": None, "parallelism": f"replicas x{world}",
                       "l2": f"state {8 * 2 ** nq / 2 ** 30:g} GiB > L2 126 MB, no flush",
                       "gates": int(stats["n_gates"]),
                       "passes": npass, "tensor_passes": int(stats["n_tensor"])},
            "roofline": roof, "passes": pass_summary, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": int(launches), "clocks": clocks, "checks": checks,
        }
        print(json.dumps(line), flush=True)
    state.close()
    plan.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
