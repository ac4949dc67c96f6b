"""Helpers to turn the committed golden fixtures into instruction lists."""
import json
from pathlib import Path

import numpy as np

from aleph_b200 import circuit as C

GOLDEN = Path(__file__).resolve().parent / "golden" / "reference_fixtures.json"


def load_reference_fixtures():
    return json.loads(GOLDEN.read_text())


def fixture_instructions(fx):
    out = []
    for op in fx["ops"]:
        if op["op"] == "gate":
            out.append(C.GateInstance(C.Gate(op["gate"], tuple(op["params"])), op["qubits"]))
        elif op["op"] == "measure":
            out.append(C.Measure(op["qubit"], op["clbit"]))
        elif op["op"] == "barrier":
            out.append(C.Barrier())
    return out


def fixture_state(fx):
    a = np.asarray(fx["amplitudes"], dtype=np.float64)
    return a[:, 0] + 1j * a[:, 1]
