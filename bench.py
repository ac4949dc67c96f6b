"""Benchmark of the dense state-vector hot path on B200.

Workload: the random brickwall circuit at n=32 qubits, depth 40 (every layer
a Haar-random SU(2) on each qubit, then CZ on nearest-neighbour pairs with
alternating even/odd offsets), starting from |0...0>, run in the
tensor-core FP32 form (complex64 state, fused 6-qubit blocks as split-BF16x3
tcgen05 GEMMs with FP32 accumulation). The same circuit on this engine's
plain FP64 path is timed beside it, and the TC-FP32 state is compared with
the FP64 state on an n=28 copy of the circuit.

One step = one circuit: reset of the 32 GiB state to |0...0> plus every pass
of the compiled plan (plan tables resident on the device). The state is far
larger than the 126 MB L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

N > 1 runs one independent replica per GPU (the path does not shard; there
is no data-path collective): `value` is the job's wall time per circuit,
max-over-ranks device time / circuits run by all ranks.

`--impl reference` times the reference's default CPU path on the host cores:
the restated final-state CPU pass pipeline (RelabelQubits, CancelInversePairs,
Fuse1qRuns, Fuse2q, FuseKq, TileBlock) and CPU sv kernels in oracle/, on the
n=28 copy of the circuit, one slice of the planned circuit per step, so the
timed steps together run the whole n=28 circuit once; that measured time is
scaled to n=32 by amplitudes and gates.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "circuit wall time & HBM % of peak, n=32 brickwall: TC-FP32 vs plain FP64"
FALLBACK_HBM_GBS = 6650.0


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def measured_hbm_peak() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        v = float(json.loads(p.read_text())["hbm_gbs"])
        return v, "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def workload_name(n: int, depth: int) -> str:
    return (f"random brickwall n={n} depth={depth} (Haar SU(2) on every qubit + CZ on alternating "
            f"nearest-neighbour pairs), |0...0> start")


FORMS = {
    "tc32": "TC-FP32: complex64 state, fused 6-qubit blocks on tcgen05 (split-BF16x3 operands, FP32 accumulate)",
    "f32": "FP32: complex64 state on CUDA cores",
    "f64": "plain FP64: complex128 state on CUDA cores",
}


def base_config(args, gates: int) -> dict:
    return {"workload": workload_name(args.n, args.depth), "n": args.n, "depth": args.depth, "gates": gates,
            "seed": args.seed, "form": FORMS[args.precision],
            "l2": f"inputs larger than L2: {float(1 << args.n) * 8 / 2**30:.0f} GiB complex64 state, no flush",
            "step": "reset to |0..0> + compiled plan (tables resident)"}


def brickwall_gates(n: int, depth: int) -> int:
    return n * depth + sum(len(range(layer % 2, n - 1, 2)) for layer in range(depth))


# ---- clocks sampled during the timed region ----------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---- distributed plumbing (replicas only) -------------------------------------
class Ranks:
    """One process per GPU (torchrun's RANK / LOCAL_RANK / WORLD_SIZE). The
    replicas share no data: the process group carries only the barriers
    around the timed region and the max-over-ranks of the times (NCCL on
    GPUs, gloo on CPU-only hosts)."""

    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = False
        self.cuda = False

    def init(self, timeout_s: int = 600):
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist

            self.cuda = torch.cuda.is_available()
            if self.cuda:
                torch.cuda.set_device(self.local)
                dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=timeout_s),
                                        device_id=torch.device("cuda", self.local))
            else:
                dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=timeout_s))
            self.pg = True

    def barrier(self):
        if self.pg:
            import torch.distributed as dist

            dist.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        import torch.distributed as dist

        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{self.local}" if self.cuda else "cpu")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            import torch.distributed as dist

            dist.destroy_process_group()


# ---- CPU baseline: the reference's default CPU path, restated --------------------
def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def n32_scale(n_full: int, depth: int, n_sample: int) -> float:
    """Work of the n_full circuit over the n_sample copy: amplitudes x gates
    (the depth-40 brickwall's fused plan has the same structure at every n)."""
    return float(1 << (n_full - n_sample)) * brickwall_gates(n_full, depth) / brickwall_gates(n_sample, depth)


def pipeline_run(n: int, depth: int, seed: int, threads: int | None = None):
    """One run of the restated default CPU path on the depth-`depth` brickwall
    at n qubits; returns (state, seconds incl. planning, pass counts)."""
    from aleph_b200 import workloads
    from oracle import oracle

    if threads is not None:
        os.environ["ORACLE_THREADS"] = str(threads)
    c = workloads.brickwall(n, depth, seed=seed)
    psi, info = oracle.run_pipeline(n, c.instructions)
    return psi, info["plan_s"] + info["exec_s"], info


def cpu_baseline(n_full: int, depth: int, seed: int, n_measured: int = 28, n_small: int = 24) -> tuple[dict, object]:
    """The reference's default CPU path (final_state_cpu_pipeline + CPU sv
    kernels, restated in oracle/sv_pipeline.cpp) on the host cores: the whole
    n_measured copy of the circuit once on all cores (its state also serves the
    fidelity check), the n_small copy best of 3 on all cores and once on one
    core. Returns (cpu_baseline dict, n_measured state)."""
    cores = host_cores()
    psi, t_meas, info = pipeline_run(n_measured, depth, seed, threads=cores)
    small = []
    for _ in range(3):
        _, t, _ = pipeline_run(n_small, depth, seed, threads=cores)
        small.append(t)
    _, t1, _ = pipeline_run(n_small, depth, seed, threads=1)
    os.environ["ORACLE_THREADS"] = str(cores)
    value = t_meas * n32_scale(n_full, depth, n_measured)
    out = {
        "value": value, "unit": "s", "cores": cores, "kind": "port",
        "sample": (f"restated reference default CPU path (final_state_cpu_pipeline: RelabelQubits, "
                   f"CancelInversePairs, Fuse1qRuns, Fuse2q, FuseKq k<=4, TileBlock t=15; then the CPU sv kernels), "
                   f"not the reference binary: the whole n={n_measured} depth-{depth} brickwall measured in "
                   f"{t_meas:.2f} s on {cores} threads ({info['input']} gates -> {info['output']} instructions, "
                   f"{info['fused_kq']} UnitaryKq, {info['tiled_blocks']} TiledBlocks), scaled to n={n_full} by "
                   f"amplitudes x gates ({n32_scale(n_full, depth, n_measured):.2f})"),
        "measured": {"n": n_measured, "depth": depth, "seconds": t_meas, "threads": cores},
        "small": {"n": n_small, "best_of_3_s_all_cores": min(small), "one_core_s": t1,
                  "core_speedup": t1 / min(small)},
        "cpu_model": cpu_model(), "nproc": os.cpu_count(),
    }
    return out, psi


def run_reference(args, ranks: Ranks):
    """The reference arm: rank 0 plans the n=28 copy of the circuit with the
    restated default CPU path and runs it in slices, one per step (the W
    warm-up slices run on a scratch state); the K timed slices together are
    the whole circuit once. value = measured time x n=32 scale."""
    if ranks.rank != 0:
        return 0
    from aleph_b200 import workloads
    from oracle import oracle

    cores = host_cores()
    os.environ["ORACLE_THREADS"] = str(cores)
    n = args.ref_n
    c = workloads.brickwall(n, args.depth, seed=args.seed)
    t0 = time.perf_counter()
    plan = oracle.PlannedCircuit(n, c.instructions)
    plan_s = time.perf_counter() - t0
    L = len(plan)
    psi = oracle.zero_state(n)
    for k in range(args.warmup):  # warm-up: the first slices, then back to |0...0>
        plan.execute(psi, k * L // (args.warmup + args.steps), (k + 1) * L // (args.warmup + args.steps), False)
    psi[:] = 0
    psi[0] = 1.0
    cuts = [k * L // args.steps for k in range(args.steps + 1)]
    steps = [plan.execute(psi, a, b, b == L) for a, b in zip(cuts, cuts[1:])]
    plan.free()
    measured = plan_s + sum(steps)
    scale = n32_scale(args.n, args.depth, n)
    value = measured * scale
    norm = float(np.vdot(psi, psi).real)
    sample = (f"restated reference default CPU path (final_state_cpu_pipeline + CPU sv kernels), not the reference "
              f"binary: the n={n} depth-{args.depth} brickwall planned once ({L} instructions, {plan_s:.3f} s) and "
              f"run in {args.steps} slices, one per step, {sum(steps):.2f} s in all on {cores} threads "
              f"(final norm {norm:.12f}); scaled to n={args.n} by amplitudes x gates ({scale:.2f})")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(base_config(args, brickwall_gates(args.n, args.depth)),
                       form="FP64 on the host CPU: the reference's default sv path (fused CPU pass pipeline)",
                       step=f"one slice of the planned n={n} circuit copy; the {args.steps} timed slices are the "
                            f"whole circuit once",
                       l2=f"host memory: {float(1 << n) * 16 / 2**30:.0f} GiB complex128 state",
                       parallelism="host threads (rank 0)",
                       timed="CPU restatement of the reference's default sv path"),
        "cpu_baseline": {"value": value, "unit": "s", "cores": cores, "kind": "port", "sample": sample,
                         "cpu_model": cpu_model(), "measured": {"n": n, "seconds": measured,
                                                                "step_seconds": [round(x, 4) for x in steps]}},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---- the engine arm ---------------------------------------------------------------
def time_plan(be, plan, st, steps: int, warmup: int, ranks: Ranks, record: bool, clocks: ClockSampler | None):
    """Device time of `steps` circuits (reset + plan) on the engine stream."""
    import torch

    stream = torch.cuda.ExternalStream(be.stream_ptr())
    for _ in range(warmup):
        be.reset_state(st)
        plan.execute(st)
    be.synchronize()
    be.set_tuning("record_passes", 1 if record else 0)
    per_pass: list[dict] = []
    l0 = be.stats()
    ranks.barrier()
    torch.cuda.synchronize()
    if clocks:
        clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        be.reset_state(st)
        plan.execute(st)
        if record:
            per_pass.extend(be.pass_records())
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    ranks.barrier()
    clk = clocks.stop() if clocks else None
    be.set_tuning("record_passes", 0)
    l1 = be.stats()
    ms = ev0.elapsed_time(ev1)
    return ms, per_pass, l1["kernel_launches"] - l0["kernel_launches"], clk


def kernel_table(per_pass: list[dict], peak: float) -> dict:
    kinds: dict[str, dict] = {}
    for r in per_pass:
        k = kinds.setdefault(r["kind"], {"launches": 0, "ms": 0.0, "bytes": 0.0})
        k["launches"] += 1
        k["ms"] += r["ms"]
        k["bytes"] += r["bytes"]
    total = sum(k["ms"] for k in kinds.values()) or 1.0
    out = {}
    for name, k in kinds.items():
        gbs = k["bytes"] / (k["ms"] * 1e-3) / 1e9 if k["ms"] > 0 else 0.0
        out[name] = {"launches": k["launches"], "ms_total": round(k["ms"], 4), "share": round(k["ms"] / total, 4),
                     "ms_per_launch": round(k["ms"] / k["launches"], 5), "gbs": round(gbs, 1),
                     "frac_of_peak": round(gbs / peak, 4)}
    return out


def fidelity_check(n: int, depth: int, seed: int, oracle_psi) -> dict:
    """TC-FP32 and the plain FP64 path against the oracle state of the same
    circuit (the restated default CPU path's result, which the CPU tests hold
    to the raw gate-by-gate oracle at 1e-12)."""
    from aleph_b200 import workloads
    from aleph_b200.backend import B200SvBackend

    c = workloads.brickwall(n, depth, seed=seed)
    out = {"n": n, "depth": depth,
           "against": "FP64 oracle (oracle/sv_pipeline.cpp: the reference's default CPU path, restated; held to "
                      "the raw gate-by-gate oracle at 1e-12 by tests; the raw oracle itself is compared at n=28 "
                      "in tests/test_gpu_large.py)"}
    w = oracle_psi
    for prec in ("f64", "tc32"):
        be = B200SvBackend(seed=0, precision=prec)
        st = be.allocate(n)
        be.apply_stream(st, c.instructions)
        got = be.statevector(st)
        st.free()
        be.close()
        f = abs(np.vdot(w, got)) ** 2 / (np.vdot(w, w).real * np.vdot(got, got).real)
        key = "fp64_path" if prec == "f64" else "tc32"
        out[key] = {"max_abs_dpsi": float(np.abs(got - w).max()), "one_minus_fidelity": float(1.0 - f)}
        del got
    out["max_abs_dpsi"] = out["tc32"]["max_abs_dpsi"]
    out["one_minus_fidelity"] = out["tc32"]["one_minus_fidelity"]
    return out


def learned_choice(be, n, flat, precision):
    """The configuration the committed cost model ranks first (None without a model)."""
    from aleph_b200 import learned

    if not learned.MODEL_PATH.exists():
        return None
    model = learned.CostModel.load(be, learned.MODEL_PATH)
    try:
        return learned.LearnedPlanner(model).score(n, flat, precision)[0].choice
    finally:
        model.free()


def learned_greedy():
    from aleph_b200 import learned

    return learned.GREEDY


def qaoa_sweep_bench(dev: int, sets: int, loop_sample: int, seed: int, ranks: "Ranks") -> dict:
    """Batched QAOA Max-Cut sweep: `sets` parameter sets, n uniform in 12..24,
    random 3-regular graphs (odd n: random graphs with 3n/2 edges), p = 4,
    angles uniform in [0, pi]; FP32 and FP64 states, <C> in FP64. With N
    ranks the sets are split into contiguous ranges balanced by sum(2^n), each
    rank runs its range as one persistent launch on its GPU and the <C>
    values are all-gathered (aleph_b200/sweep.py); the time is the max over
    ranks. Rank 0 also times a per-circuit launch loop through the engine's
    gate-stream path."""
    from aleph_b200 import workloads
    from aleph_b200.backend import B200SvBackend
    from aleph_b200.sweep import partition_by_work, sharded_sweep

    rng = np.random.default_rng(seed)
    graphs = []
    for n in rng.integers(12, 25, sets):
        n = int(n)
        if n % 2 == 0:
            graphs.append((n, workloads.random_3_regular(n, rng)))
        else:
            e = set()
            while len(e) < (3 * n) // 2:
                i, j = (int(x) for x in rng.choice(n, 2, replace=False))
                e.add((min(i, j), max(i, j)))
            graphs.append((n, sorted(e)))
    gam = rng.uniform(0, np.pi, (sets, 4))
    bet = rng.uniform(0, np.pi, (sets, 4))
    out = {"sets": sets, "n_range": [12, 24], "p": 4, "ranks": ranks.world,
           "partition": partition_by_work([n for n, _ in graphs], ranks.world)}
    vals = {}
    for prec in ("f32", "f64"):
        be = B200SvBackend(seed=0, device=dev, precision=prec)

        def sweep():
            return sharded_sweep(graphs, gam, bet, be.qaoa_sweep, ranks.rank, ranks.world)

        sweep()  # capture + warm-up
        ts = []
        for _ in range(3):
            ranks.barrier()
            t0 = time.perf_counter()
            vals[prec] = sweep()
            ts.append(ranks.max(time.perf_counter() - t0))
        out[f"{prec}_circuits_per_s"] = round(sets / min(ts), 1)
        if prec == "f32" and ranks.rank == 0:
            # one untimed pass over the sample first: first-call costs (kernel
            # loading, a state buffer of each new size, scratch growth) are
            # not per-circuit costs
            for k in range(loop_sample):
                n, e = graphs[k]
                st = be.allocate(n)
                be.apply_stream(st, workloads.qaoa_maxcut(n, e, gam[k], bet[k]).instructions)
                be.expectation_sum(st, workloads.maxcut_pauli_sum(n, e))
                be.expectation_value(st, [(e[0][0], "Z"), (e[0][1], "Z")])
                st.free()
            # the engine loop through the public API: gate stream, then <H_C>
            # either as one fused Pauli-sum call or term by term (the
            # reference's expectation_pauli_sum loops expectation_value)
            # (the two forms alternate, twice each, and each keeps its better
            # time: the loop is host-bound and the first one after the sweep
            # otherwise absorbs its after-effects)
            best = {True: float("inf"), False: float("inf")}
            for fused in (True, False, True, False):
                t0 = time.perf_counter()
                for k in range(loop_sample):
                    n, e = graphs[k]
                    st = be.allocate(n)
                    be.apply_stream(st, workloads.qaoa_maxcut(n, e, gam[k], bet[k]).instructions)
                    terms = workloads.maxcut_pauli_sum(n, e)
                    if fused:
                        be.expectation_sum(st, terms)
                    else:
                        sum(be.expectation_value(st, s, c) for c, s in terms)
                    st.free()
                best[fused] = min(best[fused], (time.perf_counter() - t0) / loop_sample)
            out["per_circuit_loop_circuits_per_s"] = round(1.0 / best[True], 1)
            out["per_circuit_loop_term_by_term_circuits_per_s"] = round(1.0 / best[False], 1)
            out["per_circuit_loop_sample"] = loop_sample
        be.close()
    if ranks.rank == 0:
        out["sweep_speedup_f32"] = round(out["f32_circuits_per_s"] / out["per_circuit_loop_circuits_per_s"], 1)
    out["max_abs_c_f32_vs_f64"] = float(np.abs(vals["f32"] - vals["f64"]).max())
    return out


def reference_gpu_bench(dev: int, seed: int, depth: int, reps: int = 2) -> dict:
    """The reference's own GPU path on this GPU beside the engine, on the
    depth-`depth` brickwall at the reference's CUDA qubit caps (FP64 n=30,
    crates/aleph-cuda/src/sv/state.rs:41; FP32 n=31, fp32.rs:48). The reference
    arm is its CUDA kernels compiled from its sources (oracle/_ref), launched
    in its run_layered order on the stream its CUDA pass list plans
    (oracle/ref_gpu.cpp; held to the oracle by tests/test_gpu_refgpu.py).
    Each side: best of `reps` runs from |0...0>, device time by events."""
    import torch

    from aleph_b200 import workloads
    from aleph_b200.backend import B200SvBackend
    from aleph_b200.circuit import flatten
    from oracle import oracle

    if not oracle.reference_gpu_available():
        return {"unavailable": "reference kernels not built (oracle/_ref: make -C oracle ref)"}
    out = {"workload": f"random brickwall depth {depth}, seed {seed}, |0...0> start",
           "reference": "the reference's CUDA kernels (kernels.cu, diag.cu, kernels_f32.cu) compiled for sm_100a; "
                        "CUDA pass list CancelInversePairs, FuseDiagonalRuns, Fuse1qRuns, Fuse2q, FuseKq(3); "
                        "run_layered dispatch (apply_1q_multi batches of 3, apply_phase_poly, apply_kq_tiled)"}

    def engine_ms(n, flat, precision):
        be = B200SvBackend(seed=seed, device=dev, precision=precision)
        stream = torch.cuda.ExternalStream(be.stream_ptr())
        plan = be.compile(n, flat)
        st = be.allocate(n)
        be.reset_state(st)
        plan.execute(st)
        ms = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            be.reset_state(st)
            plan.execute(st)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        plan.free()
        st.free()
        be.close()
        return min(ms)

    for key, n, f32, forms in (("fp64_n30", 30, False, ("f64", "tc32")), ("fp32_n31", 31, True, ("f32", "tc32"))):
        c = workloads.brickwall(n, depth, seed=seed)
        plan = oracle.PlannedCircuit(n, c.instructions, max_k=3, gpu=True)
        ref_ms, launches, _ = oracle.run_reference_gpu(plan, f32=f32, repeats=reps)
        counts = plan.counts()
        plan.free()
        torch.cuda.synchronize()
        row = {"n": n, "reference_ms": round(float(ref_ms.min()), 2), "reference_launches": launches,
               "reference_instructions": counts["output"], "reference_diagonal_phases": counts["tiled_blocks"]}
        flat = flatten(c.instructions)
        for prec in forms:
            ms = engine_ms(n, flat, prec)
            row[f"engine_{prec}_ms"] = round(ms, 2)
            row[f"speedup_{prec}"] = round(float(ref_ms.min()) / ms, 2)
        out[key] = row
    return out


def out_of_core_bench(dev: int, seed: int, n: int = 28, depth: int = 4, tile_qubits: int = 20,
                      local_qubits: int = 26) -> dict:
    """The out-of-core path (aleph_b200_paged_run): an FP64 brickwall whose
    state lives in pinned host memory, streamed through the device in tile
    groups of at most 2^local_qubits amplitudes (1 GiB at 26), three device
    buffers in the ring. Reports the host<->device traffic rate."""
    from aleph_b200 import workloads
    from aleph_b200.backend import B200SvBackend

    be = B200SvBackend(seed=0, device=dev, precision="f64").set_tuning("paged_local_qubits", local_qubits)
    c = workloads.brickwall(n, depth, seed=seed)
    ps = be.run_paged(c, tile_qubits, depth=3)
    info = ps.info()
    norm = ps.norm_sqr()
    ps.free()
    be.close()
    moved = info["h2d_bytes"] + info["d2h_bytes"]
    return {"workload": f"brickwall n={n} depth={depth}, FP64, host-resident state", "tile_qubits": tile_qubits,
            "local_qubits": info["local_qubits"], "segments": info["segments"], "groups": info["groups"],
            "bytes_moved": moved, "seconds": round(info["seconds"], 4),
            "host_device_gbs": round(moved / info["seconds"] / 1e9, 1), "norm_sqr": norm}


def small_configs_bench(dev: int, seed: int, greedy: bool = False) -> dict:
    """The two plain-FP64 configurations beside the headline:
    C0: brickwall n=20 depth 20, full state and 1024 shots against the oracle;
    C1: textbook QFT (with bit-reversal swaps) on a random Ry.Rz product state
    at n=30: time, ||psi||^2 and 4096 shots on the device, and max|dpsi|
    against the oracle on the n=24 copy of the circuit. C1 runs the plan
    configuration the committed cost model ranks first (unless ``greedy``)."""
    import torch

    from aleph_b200 import workloads
    from aleph_b200.backend import B200SvBackend
    from oracle import oracle

    out = {}
    be = B200SvBackend(seed=seed, device=dev, precision="f64")
    stream = torch.cuda.ExternalStream(be.stream_ptr())

    def timed(n, circ, reps=3):
        plan = be.compile(n, circ.instructions)
        st = be.allocate(n)
        be.reset_state(st)
        plan.execute(st)
        ms = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            be.reset_state(st)
            plan.execute(st)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        plan.free()
        return st, min(ms)

    c0 = workloads.brickwall(20, 20, seed=seed)
    st, ms = timed(20, c0)
    psi = be.statevector(st)
    want, _ = oracle.run(20, c0.instructions)
    words = workloads.splitmix64_words(seed, 1024)
    shots_ok = bool(np.array_equal(be.sample(st, 1024, variates=words, mode="alias"), oracle.sample_alias(want, words)))
    out["c0_brickwall_n20_d20"] = {"ms": round(ms, 3), "max_abs_dpsi": float(np.abs(psi - want).max()),
                                   "shots_1024_identical": shots_ok}
    st.free()

    c1 = workloads.qft_product(30, seed=seed)
    choice = None
    if not greedy:
        from aleph_b200 import learned

        if learned.MODEL_PATH.exists():  # the learned plan, kept only if measured faster and state-equal
            model = learned.CostModel.load(be, learned.MODEL_PATH)
            try:
                choice = learned.autotune(be, 30, c1.instructions, learned.LearnedPlanner(model), top_k=2).choice
            finally:
                model.free()
    st, ms = timed(30, c1)
    norm = be.norm_sqr(st)
    u = np.random.default_rng(seed).random(4096)
    g0 = be.stats()
    t0 = time.perf_counter()
    be.sample(st, 4096, variates=u, mode="cumulative")
    shots_ms = (time.perf_counter() - t0) * 1e3
    g1 = be.stats()
    st.free()
    c1s = workloads.qft_product(24, seed=seed)
    st24 = be.allocate(24)
    be.apply_stream(st24, c1s.instructions)
    w24, _ = oracle.run(24, c1s.instructions)
    out["c1_qft_n30"] = {"ms": round(ms, 3), "norm_sqr": norm, "shots_4096_ms": round(shots_ms, 2),
                         "plan_choice": None if choice is None else dict(choice.__dict__, source="learned cost model, autotuned"),
                         "shots_mode": "cumulative (alias tables are built up to n=28)",
                         "guard_band_shots": g1["guard_band_shots"] - g0["guard_band_shots"],
                         "guard_band_not_reresolved": g1["guard_band_inexact"] - g0["guard_band_inexact"],
                         "n24_copy_max_abs_dpsi": float(np.abs(be.statevector(st24) - w24).max())}
    st24.free()
    be.close()
    return out


def run_engine(args, ranks: Ranks):
    import torch

    from aleph_b200 import workloads
    from aleph_b200.backend import B200SvBackend
    from aleph_b200.circuit import flatten

    ranks.init()
    dev = ranks.local
    torch.cuda.set_device(dev)
    peak, peak_kind = measured_hbm_peak()
    n, depth = args.n, args.depth
    circ = workloads.brickwall(n, depth, seed=args.seed)
    flat = flatten(circ.instructions)

    # -- TC-FP32, device-resident: the headline value, on the plan configuration
    #    the learned cost model scores best (the greedy configuration without a model)
    be = B200SvBackend(seed=args.seed, device=dev, precision=args.precision)
    choice = learned_choice(be, n, flat, args.precision) if not args.greedy else None
    if choice is not None:
        choice.apply(be)
    plan = be.compile(n, flat)
    st = be.allocate(n)
    clocks = ClockSampler(dev)
    ms, per_pass, launches, clk = time_plan(be, plan, st, args.steps, args.warmup, ranks, True, clocks)
    ms_max = ranks.max(ms)
    norm = be.norm_sqr(st)
    s_per_circuit = ms_max * 1e-3 / (args.steps * ranks.world)
    table = kernel_table(per_pass, peak)
    # dominant kernel and its roofline (algorithmic bytes per launch / mean launch time)
    dom = max(table, key=lambda k: table[k]["ms_total"]) if table else None
    roof = None
    if dom:
        d = table[dom]
        algo_per_launch = 2.0 * float(1 << n) * (16.0 if args.precision == "f64" else 8.0)
        if dom == "measure":
            algo_per_launch *= 1.5
        achieved = algo_per_launch / (d["ms_per_launch"] * 1e-3) / 1e9
        traffic = TRAFFIC_PER_AMP.get((args.precision, dom))
        roof = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "traffic": None if traffic is None else traffic * float(1 << n),
                "algorithmic_bytes_per_launch": algo_per_launch}
    plan.free()

    # -- end to end through the C ABI with host buffers: allocate, the gate
    #    stream from host records (validation, planning, plan upload), 1024
    #    shots back to the host, free
    shots = 1024
    rng = np.random.default_rng(args.seed)
    variates = rng.random(shots)
    st.free()

    def e2e_step():
        s = be.allocate(n)
        be.apply_stream(s, None, flat=flat)
        out = be.sample(s, shots, variates=variates, mode="cumulative")
        s.free()
        return out

    for _ in range(max(1, args.e2e_warmup)):
        e2e_step()
    be.synchronize()
    s0 = be.stats()
    ranks.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        e2e_step()
    be.synchronize()
    t1 = time.perf_counter()
    ranks.barrier()
    s1 = be.stats()
    e2e_s = ranks.max(t1 - t0) / (args.e2e_steps * ranks.world)
    e2e = {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": (s1["h2d_bytes"] - s0["h2d_bytes"]) // args.e2e_steps,
           "d2h_bytes_per_step": (s1["d2h_bytes"] - s0["d2h_bytes"]) // args.e2e_steps,
           "steps": args.e2e_steps, "what": "allocate + apply_gate_stream(host records) + 1024 shots to host + free",
           "guard_band_shots_per_step": (s1["guard_band_shots"] - s0["guard_band_shots"]) / args.e2e_steps,
           "guard_band_not_reresolved_per_step": (s1["guard_band_inexact"] - s0["guard_band_inexact"]) / args.e2e_steps}
    be.close()

    # -- the plain FP64 path on the same circuit
    fp64 = None
    if not args.skip_fp64:
        b64 = B200SvBackend(seed=args.seed, device=dev, precision="f64")
        p64 = b64.compile(n, flat)
        s64 = b64.allocate(n)
        ms64, per64, _, _ = time_plan(b64, p64, s64, args.fp64_steps, max(3, args.warmup), ranks, True, None)
        ms64 = ranks.max(ms64)
        s64_per = ms64 * 1e-3 / (args.fp64_steps * ranks.world)
        fp64 = {"s_per_circuit": s64_per, "steps": args.fp64_steps, "tc32_speedup": s64_per / s_per_circuit,
                "kernels": kernel_table(per64, peak)}
        # The plain FP64 passes fuse many gates each, so their roofline is
        # max(bytes / HBM, DFMA / the FP64 rate), with the DFMA rate measured
        # on this GPU (aleph_b200_fp64_rate). The DFMA are the plan's own: each
        # pass record counts its real multiply-adds per amplitude (8 per dense
        # one-qubit op, 16 per fused 4x4); the CZs are sign flips.
        rate = b64.fp64_rate()  # TFLOP/s, 2 flop per DFMA
        n1q = n * depth
        dfma = sum(r["fma_per_amp"] for r in per64) * float(1 << n) / max(1, args.fp64_steps)
        dfma_s = dfma * 2.0 / (rate * 1e12)
        passes64 = sum(k["launches"] for k in fp64["kernels"].values()) / max(1, args.fp64_steps)
        hbm_s = passes64 * 2.0 * float(1 << n) * 16.0 / (peak * 1e9)
        fp64["roofline"] = {"bound": "max(hbm, fp64)", "fp64_tflops_measured": round(rate, 2), "dfma": dfma,
                            "dfma_gate_by_gate": 8.0 * n1q * float(1 << n),
                            "dfma_floor_s": round(dfma_s, 4), "hbm_floor_s": round(hbm_s, 4),
                            "passes": passes64, "frac": round(max(dfma_s, hbm_s) / s64_per, 4),
                            "what": f"the plan's multiply-adds per amplitude x 2^{n} at the measured DFMA rate "
                                    f"({n1q} Haar gates, pair-fused into 4x4s: 16 DFMA per 4x4 where gate by gate "
                                    f"takes 8 per gate); passes x 2 x 2^{n} x 16 B at the measured HBM copy rate"}
        p64.free()
        # the same path on the configuration the learned cost model ranks first
        # (the planner's own choice; the greedy plan above is its baseline)
        choice64 = learned_choice(b64, n, flat, "f64") if not args.greedy else None
        if choice64 is not None and choice64 != learned_greedy():
            choice64.apply(b64)
            q64 = b64.compile(n, flat)
            ms_l, per_l, _, _ = time_plan(b64, q64, s64, args.fp64_steps, max(3, args.warmup), ranks, True, None)
            s_l = ranks.max(ms_l) * 1e-3 / (args.fp64_steps * ranks.world)
            dfma_l = sum(r["fma_per_amp"] for r in per_l) * float(1 << n) / max(1, args.fp64_steps)
            fp64["learned"] = {"choice": dict(choice64.__dict__), "s_per_circuit": s_l, "tc32_speedup": s_l / s_per_circuit,
                               "gain_over_greedy": s64_per / s_l,
                               "roofline_frac": round(max(dfma_l * 2.0 / (rate * 1e12), hbm_s) / s_l, 4)}
            q64.free()
        s64.free()
        b64.close()

    # the CPU baseline (rank 0 at N=1): the reference's default CPU path on the
    # host cores; its n=28 state is the oracle state of the fidelity check
    cpu, oracle_psi = None, None
    if ranks.world == 1 and not args.skip_cpu:
        cpu, oracle_psi = cpu_baseline(n, depth, args.seed, n_measured=args.fidelity_n or 28)

    fid = None
    if args.fidelity_n and ranks.rank == 0:
        if oracle_psi is None:
            from aleph_b200 import workloads as _w
            from oracle import oracle as _o

            oracle_psi, _ = _o.run_pipeline(args.fidelity_n, _w.brickwall(args.fidelity_n, depth, seed=args.seed).instructions)
        fid = fidelity_check(args.fidelity_n, depth, args.seed, oracle_psi)
    oracle_psi = None

    qaoa = None
    if args.qaoa_sets:  # every rank runs its share of the sets
        qaoa = qaoa_sweep_bench(dev, args.qaoa_sets, 32, args.seed, ranks)
    small = None
    if not args.skip_small and ranks.rank == 0:
        small = small_configs_bench(dev, args.seed, greedy=args.greedy)
    paged = None
    if not args.skip_paged and ranks.rank == 0:
        paged = out_of_core_bench(dev, args.seed)
    refgpu = None
    if not args.skip_refgpu and ranks.rank == 0:
        refgpu = reference_gpu_bench(dev, args.seed, depth)

    if ranks.rank == 0:
        line = {
            "metric": METRIC, "value": s_per_circuit, "unit": "s", "n_gpus": ranks.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (tc32: split-bf16x3 tensor-core blocks, fp32 accumulate)"
            if args.precision == "tc32" else args.precision, "data": "synthetic",
            "config": dict(base_config(args, len(circ.instructions)),
                           parallelism=f"replicas x{ranks.world}" if ranks.world > 1 else "single GPU"),
            "clocks": clk, "e2e": e2e, "gpu_launches": launches, "roofline": roof, "cpu_baseline": cpu,
            "kernels": table, "fp64_plain": fp64, "fidelity": fid, "final_norm_sqr": norm,
            "plan_choice": None if choice is None else dict(choice.__dict__, source="learned cost model"),
            "qaoa_sweep": qaoa, "fp64_configs": small, "out_of_core": paged, "reference_gpu": refgpu,
        }
        print(json.dumps(line), flush=True)
    ranks.close()
    return 0


# DRAM bytes (read + write) per amplitude of one launch of the dominant
# kernel, from an ncu capture of that kernel on a smaller register (n=26),
# scaled by the amplitudes it processes (traffic grows in proportion to 2^n):
# block_kernel 537.0 MB read + 479.2 MB written over 2^26 amplitudes;
# tile_kernel (FP64) 1.074 GB + 1.068 GB over 2^26.
TRAFFIC_PER_AMP: dict[tuple[str, str], float] = {
    ("tc32", "block"): (537.031936e6 + 479.182848e6) / 2**26,
    ("f64", "tile"): (1.074011e9 + 1.067877e9) / 2**26,
}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--n", type=int, default=32)
    ap.add_argument("--depth", type=int, default=40)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--precision", choices=["tc32", "f32", "f64"], default="tc32")
    ap.add_argument("--fp64-steps", type=int, default=3)
    ap.add_argument("--skip-fp64", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--e2e-warmup", type=int, default=1)
    ap.add_argument("--fidelity-n", type=int, default=28)
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--ref-n", type=int, default=28, help="qubits of the reference arm's measured circuit copy")
    ap.add_argument("--qaoa-sets", type=int, default=4096, help="QAOA sweep size (0: skip)")
    ap.add_argument("--greedy", action="store_true", help="the greedy plan configuration, no cost model")
    ap.add_argument("--skip-small", action="store_true", help="skip the n=20 brickwall / n=30 QFT FP64 checks")
    ap.add_argument("--skip-paged", action="store_true", help="skip the out-of-core (host-paged) run")
    ap.add_argument("--skip-refgpu", action="store_true",
                    help="skip the reference's own GPU kernels timed beside the engine (FP64 n=30, FP32 n=31)")
    args = ap.parse_args(argv)
    args.warmup = max(3, args.warmup)  # at least 3 untimed warm-up steps
    ranks = Ranks()
    if args.impl == "reference":
        return run_reference(args, ranks)
    return run_engine(args, ranks)


if __name__ == "__main__":
    sys.exit(main())
