"""Generate tests/golden/reference_fixtures.json from the reference's own
golden vectors: oracle/circuits/*.qasm + oracle/fixtures/*.json of
aleph-sim/aleph (Qiskit-Aer 0.15.1 statevectors, compared by the reference at
|delta| <= 1e-10, crates/aleph-oracle/src/harness.rs:18).

Each circuit is parsed with a minimal reader of the OpenQASM 3 subset the
reference's parser lowers (crates/aleph-parser/src/lower.rs:255-283) and
stored as a list of operations beside the expected amplitudes, so the tests
need neither the reference tree nor a QASM parser at run time.

Usage:  python tests/golden/make_golden.py /path/to/reference
"""
from __future__ import annotations

import json
import math
import re
import sys
from pathlib import Path

GATES = {  # qasm name -> (Gate variant, number of params)
    "h": ("H", 0), "x": ("X", 0), "y": ("Y", 0), "z": ("Z", 0), "s": ("S", 0), "sdg": ("Sdg", 0),
    "t": ("T", 0), "tdg": ("Tdg", 0), "rx": ("Rx", 1), "ry": ("Ry", 1), "rz": ("Rz", 1),
    "p": ("Phase", 1), "u3": ("U3", 3), "cx": ("Cnot", 0), "cz": ("Cz", 0), "swap": ("Swap", 0),
    "ccx": ("Toffoli", 0), "ccz": ("Ccz", 0),
}


def eval_param(expr: str) -> float:
    if not re.fullmatch(r"[0-9eE+\-*/(). pi]+", expr):
        raise ValueError(f"unsupported parameter expression {expr!r}")
    return float(eval(expr, {"__builtins__": {}}, {"pi": math.pi}))


def parse_qasm(src: str):
    n = None
    ops = []
    for raw in src.splitlines():
        line = raw.split("//")[0].strip()
        if not line or line.startswith("OPENQASM") or line.startswith("include"):
            continue
        line = line.rstrip(";").strip()
        m = re.fullmatch(r"qubit\[(\d+)\]\s+\w+", line)
        if m:
            n = int(m.group(1))
            continue
        if re.fullmatch(r"bit\[(\d+)\]\s+\w+", line):
            continue
        m = re.fullmatch(r"measure\s+\w+\[(\d+)\]\s*->\s*\w+\[(\d+)\]", line)
        if m:
            ops.append({"op": "measure", "qubit": int(m.group(1)), "clbit": int(m.group(2))})
            continue
        if line.startswith("barrier"):
            ops.append({"op": "barrier"})
            continue
        m = re.fullmatch(r"(\w+)\s*(?:\(([^)]*)\))?\s+(.*)", line)
        if not m:
            raise ValueError(f"cannot parse {raw!r}")
        name, params, args = m.group(1), m.group(2), m.group(3)
        gate, nparams = GATES[name]
        ps = [eval_param(p.strip()) for p in params.split(",")] if params else []
        assert len(ps) == nparams, raw
        qs = [int(x) for x in re.findall(r"\w+\[(\d+)\]", args)]
        ops.append({"op": "gate", "gate": gate, "qubits": qs, "params": ps})
    return n, ops


def main(ref: Path) -> None:
    out = []
    for fx_path in sorted((ref / "oracle" / "fixtures").glob("*.json")):
        fx = json.loads(fx_path.read_text())
        qasm = (ref / "oracle" / fx["qasm_path"]).read_text()
        n, ops = parse_qasm(qasm)
        assert n == fx["num_qubits"], fx_path
        amps = fx["statevector"]["amplitudes"]
        assert fx["statevector"]["endianness"] == "little"
        entry = {"name": fx["name"], "num_qubits": n, "ops": ops, "amplitudes": amps,
                 "source": f"oracle/fixtures/{fx_path.name} + {fx['qasm_path']} (Qiskit-Aer {fx['aer_version']})"}
        # Mid-circuit measurements: the fixture pins the collapsed branch. A
        # measurement consumes a uniform u only when both branches are
        # non-degenerate and reports outcome = (u < p1)
        # (crates/aleph-sv/src/measure.rs:75-91). The only such fixture
        # (surface_code_cycle) holds outcome 0 on a p1 = 0.5 branch, which
        # u = 0.75 selects; the state comparison in the tests confirms it.
        n_meas = sum(1 for o in ops if o["op"] == "measure")
        entry["measure_uniforms"] = [0.75] * n_meas
        out.append(entry)
    dest = Path(__file__).resolve().parent / "reference_fixtures.json"
    dest.write_text(json.dumps(out, indent=1) + "\n")
    print(f"wrote {len(out)} fixtures to {dest}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the aleph reference checkout>")
    main(Path(sys.argv[1]))
