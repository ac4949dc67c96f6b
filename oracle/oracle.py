"""ctypes binding of the CPU oracle (oracle/sv_oracle.cpp). TEST INFRASTRUCTURE.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline /
reference arm import this module. It restates the reference's FP64 CPU
``sv`` backend and is the checker of the B200 engine, never its fallback.
"""
from __future__ import annotations

import ctypes as ct
import subprocess
from pathlib import Path

import numpy as np

from aleph_b200 import abi
from aleph_b200.circuit import flatten

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libsv_oracle.so"
_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib() -> ct.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = ct.CDLL(str(LIB))
        D = ct.POINTER(ct.c_double)
        U64 = ct.POINTER(ct.c_uint64)
        U32 = ct.POINTER(ct.c_uint32)
        sig = {
            "orc_last_error": ([ct.POINTER(abi.ErrorInfo)], ct.c_int),
            "orc_init": ([D, ct.c_uint32], ct.c_int),
            "orc_apply_gate": ([D, ct.c_uint32, ct.POINTER(abi.Instr), D, ct.c_uint64], ct.c_int),
            "orc_gate_matrix": ([ct.POINTER(abi.Instr), D, ct.c_uint64, D, ct.POINTER(ct.c_int)], ct.c_int),
            "orc_apply_diagonal_phase": ([D, ct.c_uint32, ct.POINTER(abi.PhaseTerm), ct.c_uint64, U64, ct.c_uint64], ct.c_int),
            "orc_unpermute": ([D, ct.c_uint32, U32], ct.c_int),
            "orc_measure": ([D, ct.c_uint32, ct.c_uint32, ct.c_double, ct.POINTER(ct.c_int), ct.POINTER(ct.c_int)], ct.c_int),
            "orc_sample_cumulative": ([D, ct.c_uint32, ct.c_uint32, D, U64], ct.c_int),
            "orc_sample_alias": ([D, ct.c_uint32, ct.c_uint32, U64, U64], ct.c_int),
            "orc_alias_table": ([D, ct.c_uint64, D, U32], ct.c_int),
            "orc_expectation": ([D, ct.c_uint32, U32, ct.POINTER(ct.c_uint8), ct.c_uint32, ct.c_double, D], ct.c_int),
            "orc_probabilities": ([D, ct.c_uint32, U32, ct.c_uint32, D], ct.c_int),
            "orc_norm_sqr": ([D, ct.c_uint32, D], ct.c_int),
            "orc_run_stream": ([D, ct.c_uint32, ct.POINTER(abi.Instr), ct.c_uint64, ct.POINTER(abi.Pools), D,
                                ct.c_uint64, ct.POINTER(ct.c_uint8), ct.c_uint64, U64, U64], ct.c_int),
            "orc_pipeline_describe": ([ct.c_uint32, ct.POINTER(abi.Instr), ct.c_uint64, ct.POINTER(abi.Pools),
                                       ct.c_uint32, ct.c_uint32, U64], ct.c_int),
            "orc_pipeline_run": ([D, ct.c_uint32, ct.POINTER(abi.Instr), ct.c_uint64, ct.POINTER(abi.Pools),
                                  ct.c_uint32, ct.c_uint32, D, ct.c_uint64, D, U64], ct.c_int),
            "orc_pipeline_plan": ([ct.c_uint32, ct.POINTER(abi.Instr), ct.c_uint64, ct.POINTER(abi.Pools),
                                   ct.c_uint32, ct.c_uint32, ct.POINTER(ct.c_void_p)], ct.c_int),
            "orc_pipeline_len": ([ct.c_void_p], ct.c_uint64),
            "orc_pipeline_free": ([ct.c_void_p], None),
            "orc_pipeline_exec": ([ct.c_void_p, D, ct.c_uint64, ct.c_uint64, ct.c_int, D, ct.c_uint64, U64, D],
                                  ct.c_int),
            "orc_gpu_pipeline_plan": ([ct.c_uint32, ct.POINTER(abi.Instr), ct.c_uint64, ct.POINTER(abi.Pools),
                                       ct.c_uint32, ct.POINTER(ct.c_void_p)], ct.c_int),
            "orc_pipeline_records": ([ct.c_void_p, ct.POINTER(ct.POINTER(abi.Instr)), U64, ct.POINTER(abi.Pools)],
                                     ct.c_int),
            "orc_pipeline_counts": ([ct.c_void_p, U64], None),
            "orc_refgpu_error": ([], ct.c_char_p),
            "orc_refgpu_load": ([ct.c_char_p], ct.c_int),
            "orc_refgpu_run": ([ct.c_uint32, ct.c_int, ct.POINTER(abi.Instr), ct.c_uint64, ct.POINTER(abi.Pools),
                                ct.c_int, D, U64, D], ct.c_int),
        }
        for k, (a, r) in sig.items():
            f = getattr(L, k)
            f.argtypes = a
            f.restype = r
        _lib = L
    return _lib


class OracleError(Exception):
    def __init__(self, status, info):
        self.status = status
        self.info = info
        super().__init__(f"{abi.STATUS_NAMES.get(status, status)}: {info.kind.decode(errors='replace')}")


def _dp(a):
    return a.ctypes.data_as(ct.POINTER(ct.c_double))


def _check(st):
    if st != 0:
        info = abi.ErrorInfo()
        lib().orc_last_error(ct.byref(info))
        raise OracleError(st, info)


def zero_state(n: int) -> np.ndarray:
    s = np.zeros(1 << n, dtype=np.complex128)
    s[0] = 1.0
    return s


def run(n: int, instructions, uniforms=None, state: np.ndarray | None = None):
    """run_with_outcomes on the oracle: returns (state, outcomes)."""
    flat = flatten(instructions)
    psi = zero_state(n) if state is None else np.array(state, dtype=np.complex128, copy=True)
    u = np.ascontiguousarray(np.asarray(uniforms if uniforms is not None else [], dtype=np.float64))
    outs = (ct.c_uint8 * max(1, flat.n))()
    nout = ct.c_uint64()
    failed = ct.c_uint64()
    st = lib().orc_run_stream(_dp(psi), n, flat.instrs, flat.n, ct.byref(flat.pools),
                              _dp(u) if u.size else None, u.size, outs, flat.n, ct.byref(nout), ct.byref(failed))
    _check(st)
    return psi, [int(outs[i]) for i in range(nout.value)]


def sample_alias(psi: np.ndarray, words) -> np.ndarray:
    psi = np.ascontiguousarray(psi, dtype=np.complex128)
    n = psi.size.bit_length() - 1
    w = np.ascontiguousarray(np.asarray(words, dtype=np.uint64))
    out = np.zeros(w.size, dtype=np.uint64)
    _check(lib().orc_sample_alias(_dp(psi), n, w.size, w.ctypes.data_as(ct.POINTER(ct.c_uint64)),
                                  out.ctypes.data_as(ct.POINTER(ct.c_uint64))))
    return out


def sample_cumulative(psi: np.ndarray, uniforms) -> np.ndarray:
    psi = np.ascontiguousarray(psi, dtype=np.complex128)
    n = psi.size.bit_length() - 1
    u = np.ascontiguousarray(np.asarray(uniforms, dtype=np.float64))
    out = np.zeros(u.size, dtype=np.uint64)
    _check(lib().orc_sample_cumulative(_dp(psi), n, u.size, _dp(u), out.ctypes.data_as(ct.POINTER(ct.c_uint64))))
    return out


def alias_table(probs):
    p = np.ascontiguousarray(np.asarray(probs, dtype=np.float64))
    prob = np.zeros_like(p)
    alias = np.zeros(p.size, dtype=np.uint32)
    _check(lib().orc_alias_table(_dp(p), p.size, _dp(prob), alias.ctypes.data_as(ct.POINTER(ct.c_uint32))))
    return prob, alias


def measure(psi: np.ndarray, qubit: int, u: float):
    n = psi.size.bit_length() - 1
    o, c = ct.c_int(), ct.c_int()
    _check(lib().orc_measure(_dp(psi), n, qubit, u, ct.byref(o), ct.byref(c)))
    return o.value, c.value


def expectation(psi: np.ndarray, terms, coefficient=1.0) -> float:
    psi = np.ascontiguousarray(psi, dtype=np.complex128)
    n = psi.size.bit_length() - 1
    qs = (ct.c_uint32 * max(1, len(terms)))(*[q for q, _ in terms])
    ps = (ct.c_uint8 * max(1, len(terms)))(*[abi.PAULI[p] for _, p in terms])
    out = ct.c_double()
    _check(lib().orc_expectation(_dp(psi), n, qs, ps, len(terms), coefficient, ct.byref(out)))
    return out.value


def probabilities(psi: np.ndarray, qubits) -> np.ndarray:
    psi = np.ascontiguousarray(psi, dtype=np.complex128)
    n = psi.size.bit_length() - 1
    qs = (ct.c_uint32 * max(1, len(qubits)))(*qubits)
    out = np.zeros(1 << len(qubits), dtype=np.float64)
    _check(lib().orc_probabilities(_dp(psi), n, qs, len(qubits), _dp(out)))
    return out


def unpermute(psi: np.ndarray, perm) -> np.ndarray:
    psi = np.array(psi, dtype=np.complex128, copy=True)
    n = psi.size.bit_length() - 1
    p = (ct.c_uint32 * n)(*perm)
    _check(lib().orc_unpermute(_dp(psi), n, p))
    return psi


def gate_matrix(inst) -> np.ndarray:
    flat = flatten([inst])
    out = np.zeros(128, dtype=np.float64)
    dim = ct.c_int()
    _check(lib().orc_gate_matrix(flat.instrs, flat.matrix_ptr, flat.matrix.size // 2, _dp(out), ct.byref(dim)))
    d = dim.value
    return (out[0:2 * d * d:2] + 1j * out[1:2 * d * d:2]).reshape(d, d)


# ---- the reference's default optimised CPU path (sv_pipeline.cpp) ----------------
PIPELINE_FIELDS = ("input", "after_cancel", "after_fuse1q", "after_fuse2q", "after_fusekq", "output",
                   "tiled_blocks", "fused_kq", "relabeled")


def describe_pipeline(n: int, instructions, tile_bits: int = 15, max_k: int = 4, flat=None) -> dict:
    """Instruction counts after each pass of final_state_cpu_pipeline (host only)."""
    flat = flat or flatten(instructions)
    out = (ct.c_uint64 * 9)()
    st = lib().orc_pipeline_describe(n, flat.instrs, flat.n, ct.byref(flat.pools), tile_bits, max_k, out)
    if st != 0:
        raise OracleError(st, abi.ErrorInfo())
    return dict(zip(PIPELINE_FIELDS, (int(x) for x in out)))


def run_pipeline(n: int, instructions, uniforms=None, state: np.ndarray | None = None, tile_bits: int = 15,
                 max_k: int = 4, flat=None):
    """run_optimized_cpu_final_state: the final-state CPU pass pipeline, then
    the optimised circuit on the CPU sv kernels (crates/aleph-backend/src/lib.rs:308-318).
    Returns (state, info) with planning / execution seconds and pass counts."""
    flat = flat or flatten(instructions)
    psi = zero_state(n) if state is None else np.array(state, dtype=np.complex128, copy=True)
    u = np.ascontiguousarray(np.asarray(uniforms if uniforms is not None else [], dtype=np.float64))
    secs = (ct.c_double * 2)()
    counts = (ct.c_uint64 * 9)()
    st = lib().orc_pipeline_run(_dp(psi), n, flat.instrs, flat.n, ct.byref(flat.pools), tile_bits, max_k,
                                _dp(u) if u.size else None, u.size, secs, counts)
    if st != 0:
        info = abi.ErrorInfo()
        lib().orc_last_error(ct.byref(info))
        raise OracleError(st, info)
    info = dict(zip(PIPELINE_FIELDS, (int(x) for x in counts)))
    info["plan_s"], info["exec_s"] = secs[0], secs[1]
    return psi, info


class PlannedCircuit:
    """A circuit planned once by the final-state CPU pipeline and executed in
    slices (bench.py's reference arm times it a slice per step). With
    ``gpu=True`` the plan is the reference's CUDA pass list instead
    (fuse_full_state, crates/aleph-cuda/src/fusion.rs:137-152: CancelInversePairs,
    FuseDiagonalRuns, Fuse1qRuns, Fuse2q, FuseKq width 3), which runs here on
    the CPU kernels or on the reference's own GPU kernels (``run_reference_gpu``)."""

    def __init__(self, n: int, instructions, tile_bits: int = 15, max_k: int = 4, flat=None, gpu: bool = False):
        self.n = n
        self._flat = flat or flatten(instructions)
        self._p = ct.c_void_p()
        if gpu:
            _check(lib().orc_gpu_pipeline_plan(n, self._flat.instrs, self._flat.n, ct.byref(self._flat.pools),
                                               max_k, ct.byref(self._p)))
        else:
            _check(lib().orc_pipeline_plan(n, self._flat.instrs, self._flat.n, ct.byref(self._flat.pools),
                                           tile_bits, max_k, ct.byref(self._p)))

    def counts(self) -> dict:
        """Pass counts; for a GPU plan `tiled_blocks` counts DiagonalPhase records."""
        out = (ct.c_uint64 * 9)()
        lib().orc_pipeline_counts(self._p, out)
        return dict(zip(PIPELINE_FIELDS, (int(x) for x in out)))

    def records(self):
        """The planned instructions as flat records: (instr array, count, pools)."""
        ptr = ct.POINTER(abi.Instr)()
        cnt = ct.c_uint64()
        pools = abi.Pools()
        _check(lib().orc_pipeline_records(self._p, ct.byref(ptr), ct.byref(cnt), ct.byref(pools)))
        return ptr, cnt.value, pools

    def __len__(self) -> int:
        return int(lib().orc_pipeline_len(self._p))

    def execute(self, psi: np.ndarray, i0: int = 0, i1: int | None = None, finish: bool = True) -> float:
        """Runs planned instructions [i0, i1) on psi in place; returns seconds."""
        secs = ct.c_double()
        used = ct.c_uint64()
        i1 = len(self) if i1 is None else i1
        _check(lib().orc_pipeline_exec(self._p, _dp(psi), i0, i1, 1 if finish else 0, None, 0, ct.byref(used),
                                       ct.byref(secs)))
        return secs.value

    def free(self):
        if self._p:
            lib().orc_pipeline_free(self._p)
            self._p = ct.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


# ---- the reference's own GPU kernels (ref_gpu.cpp; bench and tests only) ------------------
REF_DIR = HERE / "_ref"


def reference_gpu_available() -> bool:
    return all((REF_DIR / f).exists() for f in ("sv_kernels.cubin", "sv_diag.cubin", "sv_kernels_f32.cubin"))


def run_reference_gpu(plan: PlannedCircuit, f32: bool = False, repeats: int = 1, state: bool = False):
    """Runs a GPU plan (``PlannedCircuit(..., gpu=True)``) on the reference's
    CUDA kernels on device 0, from |0...0>, `repeats` times. Returns
    (ms per run, launches per run, final state as complex128 or None)."""
    L = lib()
    if L.orc_refgpu_load(str(REF_DIR).encode()) != 0:
        raise RuntimeError("reference GPU kernels: " + L.orc_refgpu_error().decode())
    ptr, cnt, pools = plan.records()
    ms = np.zeros(max(1, repeats), dtype=np.float64)
    launches = ct.c_uint64()
    psi = np.zeros(1 << plan.n, dtype=np.complex128) if state else None
    rc = L.orc_refgpu_run(plan.n, 1 if f32 else 0, ptr, cnt, ct.byref(pools), repeats, _dp(ms), ct.byref(launches),
                          _dp(psi) if state else None)
    if rc != 0:
        raise RuntimeError("reference GPU run: " + L.orc_refgpu_error().decode())
    return ms, int(launches.value), psi
