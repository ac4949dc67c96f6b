"""ctypes mirror of include/aleph_b200.h and the loader of the engine library.

The engine is the in-tree shared library ``aleph_b200/libaleph_b200.so``
(built by ``aleph_b200/csrc/Makefile``). There is no fallback: if the library
is missing or fails to load, :func:`load_library` raises.
"""
from __future__ import annotations

import ctypes as ct
import os
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libaleph_b200.so"

# ---- status codes (BackendError variants, crates/aleph-backend/src/lib.rs:22-74) ----
OK = 0
DEVICE_FAILURE = 1
QUBIT_OUT_OF_RANGE = 2
DUPLICATE_QUBIT = 3
ARITY_MISMATCH = 4
UNSUPPORTED_GATE = 5
UNSUPPORTED_INSTRUCTION = 6
SYMBOLIC_PARAM = 7
NON_FINITE_PARAM = 8
NON_UNITARY_MATRIX = 9
EMPTY_CIRCUIT = 10
DEGENERATE_MEASUREMENT = 11
TOO_MANY_QUBITS = 12
INVALID_PAULI_STRING = 13
INVALID_STATE = 14
OPTIMIZATION = 15
INVALID_ARGUMENT = 16

STATUS_NAMES = {
    OK: "Ok",
    DEVICE_FAILURE: "DeviceFailure",
    QUBIT_OUT_OF_RANGE: "QubitOutOfRange",
    DUPLICATE_QUBIT: "DuplicateQubit",
    ARITY_MISMATCH: "ArityMismatch",
    UNSUPPORTED_GATE: "UnsupportedGate",
    UNSUPPORTED_INSTRUCTION: "UnsupportedInstruction",
    SYMBOLIC_PARAM: "SymbolicParam",
    NON_FINITE_PARAM: "NonFiniteParam",
    NON_UNITARY_MATRIX: "NonUnitaryMatrix",
    EMPTY_CIRCUIT: "EmptyCircuit",
    DEGENERATE_MEASUREMENT: "DegenerateMeasurement",
    TOO_MANY_QUBITS: "TooManyQubits",
    INVALID_PAULI_STRING: "InvalidPauliString",
    INVALID_STATE: "InvalidState",
    OPTIMIZATION: "Optimization",
    INVALID_ARGUMENT: "InvalidArgument",
}

# ---- gate kinds (Gate enum order, crates/aleph-core/src/gate/kinds.rs:12-107) ----
GATE_KINDS = [
    "H", "X", "Y", "Z", "S", "Sdg", "T", "Tdg", "Rx", "Ry", "Rz", "Phase", "U3",
    "Cnot", "Cz", "Swap", "Iswap", "IswapDg", "CRx", "CRy", "CRz", "Toffoli", "Ccz",
    "Unitary1q", "Unitary2q", "UnitaryKq", "Unitary1qDiag", "Unitary2qDiag",
]
KIND = {name: i for i, name in enumerate(GATE_KINDS)}
INSTR_MEASURE = 100
INSTR_RESET = 101
INSTR_BARRIER = 102
INSTR_DIAGONAL_PHASE = 103
INSTR_TILED_BLOCK = 104

PRECISION = {"f64": 0, "f32": 1, "tc32": 2}
SAMPLE_ALIAS = 0
SAMPLE_CUMULATIVE = 1
SAMPLE_AUTO = 2
PAULI = {"I": 0, "X": 1, "Y": 2, "Z": 3}


class Instr(ct.Structure):
    _fields_ = [
        ("kind", ct.c_uint32),
        ("num_qubits", ct.c_uint32),
        ("num_controls", ct.c_uint32),
        ("aux", ct.c_uint32),
        ("qubits", ct.c_uint32 * 8),
        ("controls", ct.c_uint32 * 8),
        ("params", ct.c_double * 3),
        ("data_offset", ct.c_uint64),
        ("data_len", ct.c_uint64),
    ]


class PhaseTerm(ct.Structure):
    _fields_ = [("angle", ct.c_double), ("cond_offset", ct.c_uint32), ("cond_count", ct.c_uint32)]


class Pools(ct.Structure):
    _fields_ = [
        ("matrix_pool", ct.POINTER(ct.c_double)),
        ("matrix_pool_len", ct.c_uint64),
        ("terms", ct.POINTER(PhaseTerm)),
        ("n_terms", ct.c_uint64),
        ("cond_pool", ct.POINTER(ct.c_uint64)),
        ("n_conds", ct.c_uint64),
    ]


class ErrorInfo(ct.Structure):
    _fields_ = [
        ("status", ct.c_int32),
        ("qubit", ct.c_uint32),
        ("num_qubits", ct.c_uint32),
        ("expected", ct.c_uint32),
        ("got", ct.c_uint32),
        ("requested", ct.c_uint32),
        ("limit", ct.c_uint32),
        ("instruction", ct.c_uint32),
        ("value", ct.c_double),
        ("kind", ct.c_char * 32),
    ]


class Stats(ct.Structure):
    _fields_ = [
        ("kernel_launches", ct.c_uint64),
        ("passes", ct.c_uint64),
        ("tile_passes", ct.c_uint64),
        ("block_passes", ct.c_uint64),
        ("gates_planned", ct.c_uint64),
        ("algorithmic_bytes", ct.c_double),
        ("h2d_bytes", ct.c_uint64),
        ("d2h_bytes", ct.c_uint64),
        ("guard_band_shots", ct.c_uint64),
        ("guard_band_inexact", ct.c_uint64),
    ]


class PagedInfo(ct.Structure):
    _fields_ = [
        ("num_qubits", ct.c_uint32),
        ("tile_qubits", ct.c_uint32),
        ("local_qubits", ct.c_uint32),
        ("depth", ct.c_uint32),
        ("segments", ct.c_uint64),
        ("groups", ct.c_uint64),
        ("h2d_bytes", ct.c_uint64),
        ("d2h_bytes", ct.c_uint64),
        ("seconds", ct.c_double),
    ]


class PassRecord(ct.Structure):
    _fields_ = [
        ("kind", ct.c_uint32),
        ("gates", ct.c_uint32),
        ("n", ct.c_uint32),
        ("nq", ct.c_uint32),
        ("qubits", ct.c_uint32 * 8),
        ("post_ops", ct.c_uint32),
        ("lane_ops", ct.c_uint32),
        ("dense_ops", ct.c_uint32),
        ("diag_ops", ct.c_uint32),
        ("variant", ct.c_uint32),
        ("fma_per_amp", ct.c_uint32),
        ("ms", ct.c_double),
        ("bytes", ct.c_double),
    ]


class QaoaSet(ct.Structure):
    _fields_ = [("num_qubits", ct.c_uint32), ("num_edges", ct.c_uint32), ("edge_offset", ct.c_uint64)]


class PlanConfig(ct.Structure):
    _fields_ = [
        ("precision", ct.c_int32),
        ("tile_r", ct.c_uint32),
        ("smem_max_n", ct.c_uint32),
        ("block_window_search", ct.c_uint32),
        ("tile_occupancy", ct.c_uint32),
        ("keep_swaps", ct.c_uint32),
        ("no_pair_fusion", ct.c_uint32),
    ]


PASS_KINDS = {1: "tile", 2: "smem", 3: "kq", 4: "measure", 5: "block", 6: "renorm", 7: "permute"}

# Every symbol include/aleph_b200.h declares, with its ctypes signature.
_P = ct.c_void_p
_SIGNATURES = {
    "aleph_b200_create": ([ct.c_uint64, ct.c_int, ct.c_int, ct.POINTER(_P)], ct.c_int),
    "aleph_b200_destroy": ([_P], ct.c_int),
    "aleph_b200_set_qubit_cap": ([_P, ct.c_uint32], ct.c_int),
    "aleph_b200_allocate": ([_P, ct.c_uint32, ct.POINTER(_P)], ct.c_int),
    "aleph_b200_free_state": ([_P, _P], ct.c_int),
    "aleph_b200_num_qubits": ([_P, ct.POINTER(ct.c_uint32)], ct.c_int),
    "aleph_b200_apply_gate": ([_P, _P, ct.POINTER(Instr), ct.POINTER(ct.c_double), ct.c_uint64], ct.c_int),
    "aleph_b200_apply_gate_stream": (
        [_P, _P, ct.POINTER(Instr), ct.c_uint64, ct.POINTER(Pools), ct.POINTER(ct.c_double), ct.c_uint64,
         ct.POINTER(ct.c_uint8), ct.c_uint64, ct.POINTER(ct.c_uint64)], ct.c_int),
    "aleph_b200_compile": (
        [_P, ct.c_uint32, ct.POINTER(Instr), ct.c_uint64, ct.POINTER(Pools), ct.POINTER(_P)], ct.c_int),
    "aleph_b200_execute": (
        [_P, _P, _P, ct.POINTER(ct.c_double), ct.c_uint64, ct.POINTER(ct.c_uint8), ct.c_uint64,
         ct.POINTER(ct.c_uint64)], ct.c_int),
    "aleph_b200_plan_free": ([_P, _P], ct.c_int),
    "aleph_b200_apply_diagonal_phase": (
        [_P, _P, ct.POINTER(PhaseTerm), ct.c_uint64, ct.POINTER(ct.c_uint64), ct.c_uint64], ct.c_int),
    "aleph_b200_unpermute": ([_P, _P, ct.POINTER(ct.c_uint32), ct.c_uint32], ct.c_int),
    "aleph_b200_measure": ([_P, _P, ct.c_uint32, ct.c_double, ct.POINTER(ct.c_int), ct.POINTER(ct.c_int)], ct.c_int),
    "aleph_b200_sample": ([_P, _P, ct.c_uint32, ct.c_int, _P, ct.POINTER(ct.c_uint64)], ct.c_int),
    "aleph_b200_sample_seeded": ([_P, _P, ct.c_uint32, ct.POINTER(ct.c_uint64)], ct.c_int),
    "aleph_b200_expectation": (
        [_P, _P, ct.POINTER(ct.c_uint32), ct.POINTER(ct.c_uint8), ct.c_uint32, ct.c_double,
         ct.POINTER(ct.c_double)], ct.c_int),
    "aleph_b200_expectation_sum": (
        [_P, _P, ct.POINTER(ct.c_uint32), ct.POINTER(ct.c_uint8), ct.POINTER(ct.c_uint64), ct.POINTER(ct.c_double),
         ct.c_uint64, ct.POINTER(ct.c_double), ct.POINTER(ct.c_double)], ct.c_int),
    "aleph_b200_probabilities": ([_P, _P, ct.POINTER(ct.c_uint32), ct.c_uint32, ct.POINTER(ct.c_double)], ct.c_int),
    "aleph_b200_get_amplitudes": ([_P, _P, ct.POINTER(ct.c_double)], ct.c_int),
    "aleph_b200_get_amplitude_range": ([_P, _P, ct.c_uint64, ct.c_uint64, ct.POINTER(ct.c_double)], ct.c_int),
    "aleph_b200_fp64_rate": ([_P, ct.POINTER(ct.c_double)], ct.c_int),
    "aleph_b200_state_memory": ([_P, _P, ct.POINTER(ct.c_void_p), ct.POINTER(ct.c_uint64)], ct.c_int),
    "aleph_b200_scale_state": ([_P, _P, ct.c_double], ct.c_int),
    "aleph_b200_gate_matrix": ([ct.POINTER(Instr), ct.POINTER(ct.c_double), ct.c_uint64, ct.POINTER(ct.c_double),
                                ct.POINTER(ct.c_int)], ct.c_int),
    "aleph_b200_set_amplitudes": ([_P, _P, ct.POINTER(ct.c_double)], ct.c_int),
    "aleph_b200_norm_sqr": ([_P, _P, ct.POINTER(ct.c_double)], ct.c_int),
    "aleph_b200_synchronize": ([_P], ct.c_int),
    "aleph_b200_get_stream": ([_P, ct.POINTER(_P)], ct.c_int),
    "aleph_b200_mlp_create": ([_P, ct.c_uint32, ct.c_uint32, ct.c_uint64, ct.POINTER(_P)], ct.c_int),
    "aleph_b200_mlp_free": ([_P, _P], ct.c_int),
    "aleph_b200_mlp_params": ([_P, _P, ct.POINTER(ct.c_float), ct.POINTER(ct.c_float), ct.POINTER(ct.c_uint64)],
                              ct.c_int),
    "aleph_b200_mlp_predict": ([_P, _P, ct.POINTER(ct.c_float), ct.c_uint32, ct.POINTER(ct.c_float)], ct.c_int),
    "aleph_b200_mlp_gradients": ([_P, _P, ct.POINTER(ct.c_float), ct.POINTER(ct.c_float), ct.c_uint32,
                                  ct.POINTER(ct.c_float), ct.POINTER(ct.c_float)], ct.c_int),
    "aleph_b200_mlp_train": ([_P, _P, ct.POINTER(ct.c_float), ct.POINTER(ct.c_float), ct.c_uint32, ct.c_uint32,
                              ct.c_uint32, ct.c_float, ct.c_uint64, ct.POINTER(ct.c_float)], ct.c_int),
    "aleph_b200_qaoa_sweep": (
        [_P, ct.c_uint32, ct.POINTER(QaoaSet), ct.c_uint32, ct.POINTER(ct.c_uint32), ct.c_uint64,
         ct.POINTER(ct.c_double), ct.POINTER(ct.c_double)], ct.c_int),
    "aleph_b200_describe_plan": (
        [ct.c_uint32, ct.POINTER(PlanConfig), ct.POINTER(Instr), ct.c_uint64, ct.POINTER(Pools),
         ct.POINTER(PassRecord), ct.c_uint64, ct.POINTER(ct.c_uint64)], ct.c_int),
    "aleph_b200_sample_cumulative_noalloc": (
        [_P, _P, ct.c_uint32, ct.POINTER(ct.c_double), ct.POINTER(ct.c_uint64)], ct.c_int),
    "aleph_b200_reset_state": ([_P, _P], ct.c_int),
    "aleph_b200_last_error": ([_P, ct.c_char_p, ct.c_uint64], ct.c_int),
    "aleph_b200_last_error_info": ([_P, ct.POINTER(ErrorInfo)], ct.c_int),
    "aleph_b200_set_tuning": ([_P, ct.c_char_p, ct.c_int64], ct.c_int),
    "aleph_b200_get_pass_records": ([_P, ct.POINTER(PassRecord), ct.c_uint64, ct.POINTER(ct.c_uint64)], ct.c_int),
    "aleph_b200_get_stats": ([_P, ct.POINTER(Stats)], ct.c_int),
    "aleph_b200_reset_stats": ([_P], ct.c_int),
    "aleph_b200_paged_run": (
        [_P, ct.c_uint32, ct.POINTER(Instr), ct.c_uint64, ct.POINTER(Pools), ct.c_uint32, ct.c_uint32,
         ct.POINTER(_P)], ct.c_int),
    "aleph_b200_paged_info_get": ([_P, ct.POINTER(PagedInfo)], ct.c_int),
    "aleph_b200_paged_get_amplitudes": ([_P, ct.POINTER(ct.c_double)], ct.c_int),
    "aleph_b200_paged_norm_sqr": ([_P, ct.POINTER(ct.c_double)], ct.c_int),
    "aleph_b200_paged_free": ([_P], ct.c_int),
    "aleph_b200_describe_paged": (
        [ct.c_uint32, ct.POINTER(Instr), ct.c_uint64, ct.c_uint32, ct.c_uint32, ct.POINTER(ct.c_uint64),
         ct.POINTER(ct.c_uint64), ct.POINTER(ct.c_uint64)], ct.c_int),
}

_LIB = None


def declared_symbols() -> list[str]:
    """Names of every function include/aleph_b200.h declares (parsed from the header)."""
    import re

    hdr = (PKG_DIR.parent / "include" / "aleph_b200.h").read_text()
    return sorted(set(re.findall(r"^int\s+(aleph_b200_[a-z0-9_]+)\s*\(", hdr, flags=re.M)))


def load_library(path: str | os.PathLike | None = None) -> ct.CDLL:
    """Load the engine's shared library and bind every declared entry point.

    Raises ``OSError`` if the library is absent: the engine has no CPU path.
    """
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise OSError(f"aleph_b200 engine library not built: {p} (run __graft_entry__.build())")
    lib = ct.CDLL(str(p))
    for name, (args, res) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    if path is None:
        _LIB = lib
    return lib
