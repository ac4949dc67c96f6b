"""``python -m aleph_b200`` — the reference CLI's ``run`` / ``bench``
commands (crates/aleph-cli/src/cli.rs:96-207, exec.rs:199-560, 915-955) on
the B200 engine.

``run FILE.qasm [--shots N] [--statevector] [--force-statevector]
[--expectation P]... [--seed S] [--precision auto|f64|f32|tc32]
[--backend b200|cuda|cuda-f32] [--execution-stats]`` runs the circuit once
and prints, in this order, the counts, the state vector and the expectation
values, in the reference's text formats. With no view flag it samples 1024
shots. The state vector is capped at 10 qubits unless --force-statevector.

``bench FILE.qasm [--seed S]`` prints parse / run / sample(1024) / total
wall times.

Errors print ``Error: <context>`` and the cause to stderr, exit status 1.
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

from . import frontend, qasm


def _fail(context: str, cause: Exception | None = None) -> int:
    msg = f"Error: {context}"
    if cause is not None:
        msg += f"\n\nCaused by:\n    {cause}"
    print(msg, file=sys.stderr)
    return 1


def _load(path: Path):
    try:
        src = path.read_text(encoding="utf-8")
    except OSError as e:
        return None, _fail(f"reading QASM file: {path}", e)
    try:
        return qasm.parse(src), 0
    except qasm.QasmError as e:
        return None, _fail(f"parsing {path}", e)


def cmd_run(a) -> int:
    t0 = time.perf_counter()
    circ, rc = _load(Path(a.qasm))
    if circ is None:
        return rc
    n = circ.num_qubits
    paulis = []
    for raw in a.expectation:
        try:
            coeff, terms = frontend.parse_pauli_arg(raw)
        except ValueError as e:
            return _fail(f"parsing --expectation argument {raw!r}", e)
        if terms and terms[-1][0] >= n:
            return _fail(f"--expectation {raw!r} references qubit {terms[-1][0]} but circuit has {n} qubits")
        paulis.append((raw, coeff, terms))
    try:
        prec = frontend.resolve(a.backend, a.precision)
    except ValueError as e:
        return _fail(str(e))
    if a.statevector and not a.force_statevector and n > frontend.STATEVECTOR_CAP_QUBITS:
        return _fail(f"state vector has 2^{n} = {1 << n} amplitudes; pass --force-statevector to print anyway")
    shots = a.shots if a.shots is not None else (
        frontend.DEFAULT_SHOTS if not (a.statevector or a.force_statevector or paulis) else None)
    try:
        res = frontend.run(circ, shots=shots or 0, backend=a.backend, precision=a.precision, seed=a.seed)
    except Exception as e:  # the engine's BackendError variants
        return _fail("running circuit", e)
    out = sys.stdout
    try:
        if shots is not None:
            out.write(frontend.format_counts(res.counts(), shots, n, res.seed_label))
        if a.statevector or a.force_statevector:
            out.write(frontend.format_statevector(res.statevector(), n))
        if paulis:
            out.write("expectation values:\n")
            for raw, _, _ in paulis:
                out.write(frontend.format_expectation(raw, res.expectation(raw)))
        if a.execution_stats:
            st = dict(res.execution_stats(), precision=prec, wall_ms=(time.perf_counter() - t0) * 1e3)
            print(json.dumps(st), file=sys.stderr)
    finally:
        res.close()
    return 0


def cmd_bench(a) -> int:
    path = Path(a.qasm)
    t0 = time.perf_counter()
    circ, rc = _load(path)
    if circ is None:
        return rc
    t1 = time.perf_counter()
    from .backend import B200SvBackend, run_with_outcomes

    be = B200SvBackend(seed=a.seed if a.seed is not None else 0, precision=frontend.resolve(a.backend, a.precision))
    try:
        try:
            st, _ = run_with_outcomes(be, circ)
            be.synchronize()
        except Exception as e:
            return _fail("running circuit", e)
        t2 = time.perf_counter()
        try:
            be.sample(st, frontend.DEFAULT_SHOTS)
        except Exception as e:
            return _fail("sampling final state", e)
        t3 = time.perf_counter()
        st.free()
    finally:
        be.close()
    out = sys.stdout
    out.write(f"bench {path.name} (n={circ.num_qubits}):\n")
    for name, dt in (("parse", t1 - t0), ("run", t2 - t1), ("sample(1024)", t3 - t2), ("total", t3 - t0)):
        out.write(f"  {name:<13} {frontend.format_duration(dt)}\n")
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="aleph_b200", description="Run OpenQASM 3 circuits on the B200 engine.")
    sub = ap.add_subparsers(dest="cmd", required=True)
    r = sub.add_parser("run", help="run a QASM circuit and print results")
    r.add_argument("qasm")
    r.add_argument("--shots", type=int)
    r.add_argument("--statevector", action="store_true")
    r.add_argument("--force-statevector", action="store_true")
    r.add_argument("--expectation", action="append", default=[])
    r.add_argument("--seed", type=int)
    r.add_argument("--precision", default="auto", choices=sorted(frontend.PRECISIONS))
    r.add_argument("--backend", default="b200")
    r.add_argument("--execution-stats", action="store_true", help="engine counters as JSON on stderr")
    b = sub.add_parser("bench", help="parse / run / sample wall times of one circuit")
    b.add_argument("qasm")
    b.add_argument("--seed", type=int)
    b.add_argument("--precision", default="auto", choices=sorted(frontend.PRECISIONS))
    b.add_argument("--backend", default="b200")
    a = ap.parse_args(argv)
    if getattr(a, "shots", None) is not None and a.shots < 0:
        return _fail("--shots must be >= 0")
    return cmd_run(a) if a.cmd == "run" else cmd_bench(a)


if __name__ == "__main__":
    sys.exit(main())
