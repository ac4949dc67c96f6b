"""Gate stream types mirroring aleph-core / aleph-ir, and their flattening
into the C ABI's instruction records.

* ``Gate``        — ``aleph_core::Gate`` (crates/aleph-core/src/gate/kinds.rs:12-107)
* ``GateInstance``— ``{gate, qubits, controls}`` (crates/aleph-core/src/gate/instance.rs:56-61)
* ``Measure`` / ``Reset`` / ``Barrier`` / ``DiagonalPhase`` / ``TiledBlock``
                  — ``aleph_ir::Instruction`` (crates/aleph-ir/src/instruction.rs:13-34)
* ``Circuit``     — ``aleph_ir::Circuit`` (crates/aleph-ir/src/circuit.rs:39-51)
"""
from __future__ import annotations

import ctypes as ct
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

from . import abi


@dataclass(frozen=True)
class Gate:
    """One ``Gate`` variant. ``params`` holds the parametric angles;
    ``matrix`` holds the payload of the ``Unitary*`` variants (complex128):
    2x2 / 4x4 row-major, 2^k x 2^k for ``UnitaryKq`` (``k`` set), or the
    diagonal entries for ``Unitary1qDiag`` / ``Unitary2qDiag``."""

    name: str
    params: tuple = ()
    matrix: np.ndarray | None = None
    k: int = 0

    def __post_init__(self):
        if self.name not in abi.KIND:
            raise ValueError(f"unknown gate {self.name!r}")

    @property
    def kind(self) -> int:
        return abi.KIND[self.name]

    def arity(self) -> int:
        """``Gate::arity`` (kinds.rs:110-152)."""
        n = self.name
        if n == "UnitaryKq":
            return self.k
        if n in ("Toffoli", "Ccz"):
            return 3
        if n in ("Cnot", "Cz", "Swap", "Iswap", "IswapDg", "CRx", "CRy", "CRz", "Unitary2q", "Unitary2qDiag"):
            return 2
        return 1

    def is_diagonal(self) -> bool:
        """``Gate::is_diagonal`` (kinds.rs:412-444)."""
        return self.name in ("Z", "S", "Sdg", "T", "Tdg", "Rz", "Phase", "CRz", "Cz", "Ccz",
                             "Unitary1qDiag", "Unitary2qDiag")


# Constructors named like the Rust variants.
def H(): return Gate("H")
def X(): return Gate("X")
def Y(): return Gate("Y")
def Z(): return Gate("Z")
def S(): return Gate("S")
def Sdg(): return Gate("Sdg")
def T(): return Gate("T")
def Tdg(): return Gate("Tdg")
def Rx(t): return Gate("Rx", (float(t),))
def Ry(t): return Gate("Ry", (float(t),))
def Rz(t): return Gate("Rz", (float(t),))
def Phase(t): return Gate("Phase", (float(t),))
def U3(t, p, l): return Gate("U3", (float(t), float(p), float(l)))
def Cnot(): return Gate("Cnot")
def Cz(): return Gate("Cz")
def Swap(): return Gate("Swap")
def Iswap(): return Gate("Iswap")
def IswapDg(): return Gate("IswapDg")
def CRx(t): return Gate("CRx", (float(t),))
def CRy(t): return Gate("CRy", (float(t),))
def CRz(t): return Gate("CRz", (float(t),))
def Toffoli(): return Gate("Toffoli")
def Ccz(): return Gate("Ccz")
def Unitary1q(m): return Gate("Unitary1q", matrix=np.asarray(m, dtype=np.complex128).reshape(2, 2))
def Unitary2q(m): return Gate("Unitary2q", matrix=np.asarray(m, dtype=np.complex128).reshape(4, 4))
def Unitary1qDiag(d): return Gate("Unitary1qDiag", matrix=np.asarray(d, dtype=np.complex128).reshape(2))
def Unitary2qDiag(d): return Gate("Unitary2qDiag", matrix=np.asarray(d, dtype=np.complex128).reshape(4))


def UnitaryKq(m):
    m = np.asarray(m, dtype=np.complex128)
    dim = m.shape[0]
    k = dim.bit_length() - 1
    return Gate("UnitaryKq", matrix=m.reshape(dim, dim), k=k)


@dataclass
class GateInstance:
    gate: Gate
    qubits: tuple
    controls: tuple = ()

    def __init__(self, gate: Gate, qubits: Sequence[int], controls: Sequence[int] = ()):
        self.gate = gate
        self.qubits = tuple(int(q) for q in qubits)
        self.controls = tuple(int(c) for c in controls)


@dataclass
class Measure:
    qubit: int
    clbit: int = 0


@dataclass
class Reset:
    qubit: int


@dataclass
class Barrier:
    qubits: tuple = ()


@dataclass
class PhaseTerm:
    """``PhaseTerm`` (crates/aleph-ir/src/diagonal_phase.rs:20-26)."""

    conds: tuple
    angle: float


@dataclass
class DiagonalPhase:
    """``DiagonalPhase`` (crates/aleph-ir/src/diagonal_phase.rs:46-80)."""

    n_qubits: int
    terms: list

    def phase_at(self, x: int) -> float:
        phi = 0.0
        for t in self.terms:
            if all(bin(m & x).count("1") & 1 for m in t.conds):
                phi += t.angle
        return phi


@dataclass
class TiledBlock:
    """``TiledBlock`` (crates/aleph-ir/src/tiled_block.rs): gates applied tile-major."""

    gates: list
    tile_bits: int = 15


@dataclass
class Circuit:
    num_qubits: int
    instructions: list = field(default_factory=list)
    num_clbits: int = 0

    def add(self, gate: Gate, qubits: Sequence[int], controls: Sequence[int] = ()) -> "Circuit":
        self.instructions.append(GateInstance(gate, qubits, controls))
        return self

    def measure(self, qubit: int, clbit: int = 0) -> "Circuit":
        self.instructions.append(Measure(qubit, clbit))
        return self

    def __len__(self):
        return len(self.instructions)

    def gate_count(self) -> int:
        return sum(1 for i in self.instructions if isinstance(i, GateInstance))


class Flat:
    """A circuit flattened to C ABI records plus side pools (kept alive here)."""

    def __init__(self, instrs, matrix_pool, terms, conds):
        self.n = len(instrs)
        self.instrs = (abi.Instr * max(1, self.n))(*instrs)
        self.matrix = np.ascontiguousarray(np.asarray(matrix_pool, dtype=np.float64).reshape(-1))
        self.terms = (abi.PhaseTerm * max(1, len(terms)))(*terms)
        self.n_terms = len(terms)
        self.conds = np.ascontiguousarray(np.asarray(conds, dtype=np.uint64).reshape(-1))
        self.pools = abi.Pools(
            self.matrix.ctypes.data_as(ct.POINTER(ct.c_double)) if self.matrix.size else None,
            self.matrix.size // 2,
            self.terms if self.n_terms else None,
            self.n_terms,
            self.conds.ctypes.data_as(ct.POINTER(ct.c_uint64)) if self.conds.size else None,
            self.conds.size,
        )

    @property
    def matrix_ptr(self):
        return self.matrix.ctypes.data_as(ct.POINTER(ct.c_double)) if self.matrix.size else None

    @property
    def nbytes(self) -> int:
        return self.n * ct.sizeof(abi.Instr) + self.matrix.nbytes + self.n_terms * ct.sizeof(abi.PhaseTerm) \
            + self.conds.nbytes


def _gate_record(inst: GateInstance, matrix_pool: list) -> abi.Instr:
    g = inst.gate
    r = abi.Instr()
    r.kind = g.kind
    if len(inst.qubits) > 8 or len(inst.controls) > 8:
        raise ValueError("at most 8 qubits and 8 controls per record")
    r.num_qubits = len(inst.qubits)
    r.num_controls = len(inst.controls)
    for i, q in enumerate(inst.qubits):
        r.qubits[i] = q
    for i, c in enumerate(inst.controls):
        r.controls[i] = c
    for i, p in enumerate(g.params[:3]):
        r.params[i] = p
    if g.name == "UnitaryKq":
        r.aux = g.k
    if g.matrix is not None:
        flat = np.asarray(g.matrix, dtype=np.complex128).reshape(-1)
        r.data_offset = len(matrix_pool) // 2
        r.data_len = flat.size
        for z in flat:
            matrix_pool.append(float(z.real))
            matrix_pool.append(float(z.imag))
    return r


def flatten(instructions: Sequence) -> Flat:
    """Flatten a list of instructions (or a Circuit) into C ABI records."""
    if isinstance(instructions, Circuit):
        instructions = instructions.instructions
    recs, pool, terms, conds = [], [], [], []

    def emit(inst):
        if isinstance(inst, GateInstance):
            recs.append(_gate_record(inst, pool))
        elif isinstance(inst, Measure):
            r = abi.Instr()
            r.kind = abi.INSTR_MEASURE
            r.num_qubits = 1
            r.qubits[0] = inst.qubit
            r.aux = inst.clbit
            recs.append(r)
        elif isinstance(inst, Reset):
            r = abi.Instr()
            r.kind = abi.INSTR_RESET
            r.num_qubits = 1
            r.qubits[0] = inst.qubit
            recs.append(r)
        elif isinstance(inst, Barrier):
            r = abi.Instr()
            r.kind = abi.INSTR_BARRIER
            r.num_qubits = len(inst.qubits)
            for q in inst.qubits:
                r.data_offset |= 1 << int(q)
            recs.append(r)
        elif isinstance(inst, DiagonalPhase):
            r = abi.Instr()
            r.kind = abi.INSTR_DIAGONAL_PHASE
            r.aux = inst.n_qubits
            r.data_offset = len(terms)
            r.data_len = len(inst.terms)
            for t in inst.terms:
                terms.append(abi.PhaseTerm(float(t.angle), len(conds), len(t.conds)))
                conds.extend(int(m) for m in t.conds)
            recs.append(r)
        elif isinstance(inst, TiledBlock):
            r = abi.Instr()
            r.kind = abi.INSTR_TILED_BLOCK
            r.aux = inst.tile_bits
            r.data_len = len(inst.gates)
            recs.append(r)
            for g in inst.gates:
                emit(g)
        else:
            raise TypeError(f"unknown instruction {inst!r}")

    for inst in instructions:
        emit(inst)
    return Flat(recs, pool, terms, conds)
