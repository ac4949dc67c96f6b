"""Host-side mirror of aleph's ``Backend`` trait over the engine's C ABI.

``B200SvBackend`` has the trait's methods (crates/aleph-backend/src/lib.rs:86-163):
``allocate``, ``apply_gate``, ``measure``, ``sample``, ``expectation_value``,
``probabilities``, ``apply_diagonal_phase``, ``apply_tiled_block`` and
``unpermute_state``; ``run`` / ``run_with_outcomes`` mirror the drivers of
crates/aleph-backend/src/lib.rs:182-245. Errors raise :class:`BackendError`
subclasses named after the reference's variants. Every call goes to the
CUDA library; there is no host compute path.
"""
from __future__ import annotations

import ctypes as ct
from dataclasses import dataclass

import numpy as np

from . import abi
from .circuit import Circuit, DiagonalPhase, Flat, GateInstance, Measure, TiledBlock, flatten


class BackendError(Exception):
    """``BackendError`` (crates/aleph-backend/src/lib.rs:22-74)."""

    variant = "BackendError"

    def __init__(self, status: int, message: str, info: abi.ErrorInfo | None = None):
        self.status = status
        self.info = info
        super().__init__(message)


_ERRORS: dict[int, type] = {}
for _code, _name in abi.STATUS_NAMES.items():
    if _code == abi.OK:
        continue
    _ERRORS[_code] = type(_name, (BackendError,), {"variant": _name})
    globals()[_name] = _ERRORS[_code]


def _err(lib, handle, status):
    buf = ct.create_string_buffer(512)
    lib.aleph_b200_last_error(handle, buf, 512)
    info = abi.ErrorInfo()
    lib.aleph_b200_last_error_info(handle, ct.byref(info))
    cls = _ERRORS.get(status, BackendError)
    return cls(status, buf.value.decode(errors="replace") or abi.STATUS_NAMES.get(status, str(status)), info)


@dataclass
class State:
    """A device-resident state vector owned by the caller (``CudaSvState``)."""

    ptr: ct.c_void_p
    num_qubits: int
    backend: "B200SvBackend"

    def free(self):
        if self.ptr:
            self.backend.lib.aleph_b200_free_state(self.backend.handle, self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def amplitudes(self) -> np.ndarray:
        return self.backend.statevector(self)


class PagedState:
    """An out-of-core state: the amplitudes live in pinned host memory
    (``PagedSvState``, crates/aleph-cuda/src/sv/paged.rs:53-100)."""

    def __init__(self, lib, ptr, num_qubits: int):
        self.lib, self.ptr, self.num_qubits = lib, ptr, num_qubits

    def statevector(self) -> np.ndarray:
        out = np.empty(2 << self.num_qubits, dtype=np.float64)
        self.lib.aleph_b200_paged_get_amplitudes(self.ptr, out.ctypes.data_as(ct.POINTER(ct.c_double)))
        return out.view(np.complex128)

    def norm_sqr(self) -> float:
        v = ct.c_double()
        self.lib.aleph_b200_paged_norm_sqr(self.ptr, ct.byref(v))
        return v.value

    def info(self) -> dict:
        i = abi.PagedInfo()
        self.lib.aleph_b200_paged_info_get(self.ptr, ct.byref(i))
        return {name: getattr(i, name) for name, _ in abi.PagedInfo._fields_}

    def free(self):
        if self.ptr:
            self.lib.aleph_b200_paged_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


@dataclass
class MeasurementRecord:
    """``MeasurementRecord`` (crates/aleph-backend/src/lib.rs:188-195)."""

    instruction_index: int
    qubit: int
    clbit: int
    outcome: bool


class B200SvBackend:
    """The B200 dense state-vector backend (``--backend b200``).

    precision: ``"f64"`` (complex128), ``"f32"`` (complex64, CUDA cores) or
    ``"tc32"`` (complex64 with 6-qubit dense blocks on tcgen05 tensor cores).
    """

    def __init__(self, seed: int = 0, device: int = 0, precision: str = "f64"):
        self.lib = abi.load_library()
        h = ct.c_void_p()
        st = self.lib.aleph_b200_create(int(seed) & (2**64 - 1), device, abi.PRECISION[precision], ct.byref(h))
        if st != abi.OK:
            raise BackendError(st, f"aleph_b200_create failed with status {abi.STATUS_NAMES.get(st, st)}")
        self.handle = h
        self.precision = precision

    @classmethod
    def with_seed(cls, seed: int, **kw) -> "B200SvBackend":
        return cls(seed=seed, **kw)

    def close(self):
        if getattr(self, "handle", None):
            self.lib.aleph_b200_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, status):
        if status != abi.OK:
            raise _err(self.lib, self.handle, status)

    def set_tuning(self, key: str, value: int) -> "B200SvBackend":
        self._check(self.lib.aleph_b200_set_tuning(self.handle, key.encode(), int(value)))
        return self

    def set_qubit_cap(self, cap: int) -> "B200SvBackend":
        self._check(self.lib.aleph_b200_set_qubit_cap(self.handle, cap))
        return self

    # ---- Backend trait -------------------------------------------------------
    def allocate(self, num_qubits: int) -> State:
        p = ct.c_void_p()
        self._check(self.lib.aleph_b200_allocate(self.handle, num_qubits, ct.byref(p)))
        return State(p, num_qubits, self)

    def apply_gate(self, state: State, gate: GateInstance) -> None:
        flat = flatten([gate])
        self._check(self.lib.aleph_b200_apply_gate(self.handle, state.ptr, flat.instrs, flat.matrix_ptr,
                                                   flat.matrix.size // 2))

    def apply_diagonal_phase(self, state: State, dp: DiagonalPhase) -> None:
        flat = flatten([dp])
        self._check(self.lib.aleph_b200_apply_diagonal_phase(
            self.handle, state.ptr, flat.terms if flat.n_terms else None, flat.n_terms,
            flat.conds.ctypes.data_as(ct.POINTER(ct.c_uint64)) if flat.conds.size else None, flat.conds.size))

    def apply_tiled_block(self, state: State, block: TiledBlock) -> None:
        self.apply_stream(state, [block])

    def unpermute_state(self, state: State, perm) -> None:
        arr = (ct.c_uint32 * len(perm))(*perm)
        self._check(self.lib.aleph_b200_unpermute(self.handle, state.ptr, arr, len(perm)))

    def measure(self, state: State, qubit: int, u: float | None = None) -> bool:
        o, c = ct.c_int(), ct.c_int()
        self._check(self.lib.aleph_b200_measure(self.handle, state.ptr, qubit, -1.0 if u is None else float(u),
                                                ct.byref(o), ct.byref(c)))
        return bool(o.value)

    def sample(self, state: State, shots: int, variates=None, mode: str = "auto") -> np.ndarray:
        out = np.zeros(max(1, shots), dtype=np.uint64)
        optr = out.ctypes.data_as(ct.POINTER(ct.c_uint64))
        if variates is None:
            self._check(self.lib.aleph_b200_sample_seeded(self.handle, state.ptr, shots, optr))
            return out[:shots]
        m = {"alias": abi.SAMPLE_ALIAS, "cumulative": abi.SAMPLE_CUMULATIVE, "auto": abi.SAMPLE_AUTO}[mode]
        if m == abi.SAMPLE_AUTO:
            m = abi.SAMPLE_ALIAS if shots >= 2 else abi.SAMPLE_CUMULATIVE
        v = np.ascontiguousarray(np.asarray(variates, dtype=np.uint64 if m == abi.SAMPLE_ALIAS else np.float64))
        if v.size < shots:
            raise ValueError("need one variate per shot")
        self._check(self.lib.aleph_b200_sample(self.handle, state.ptr, shots, m, v.ctypes.data_as(ct.c_void_p), optr))
        return out[:shots]

    def expectation_value(self, state: State, terms, coefficient: float = 1.0) -> float:
        """``terms``: sequence of (qubit, 'I'|'X'|'Y'|'Z') — a ``PauliString``."""
        k = len(terms)
        qs = (ct.c_uint32 * max(1, k))(*[int(q) for q, _ in terms])
        ps = (ct.c_uint8 * max(1, k))(*[abi.PAULI[p] for _, p in terms])
        out = ct.c_double()
        self._check(self.lib.aleph_b200_expectation(self.handle, state.ptr, qs, ps, k, float(coefficient),
                                                    ct.byref(out)))
        return out.value

    def expectation_sum(self, state: State, terms, with_terms: bool = False):
        """``expectation_pauli_sum`` (crates/aleph-backend/src/lib.rs:422-432):
        ``terms`` is a sequence of (coefficient, [(qubit, 'I'|'X'|'Y'|'Z'), ...]).
        Returns the sum, or (sum, per-term values) with ``with_terms``."""
        k = len(terms)
        offsets = [0]
        qs, ps = [], []
        for _, string in terms:
            for q, p in string:
                qs.append(int(q))
                ps.append(abi.PAULI[p])
            offsets.append(len(qs))
        cq = (ct.c_uint32 * max(1, len(qs)))(*qs)
        cp = (ct.c_uint8 * max(1, len(ps)))(*ps)
        co = (ct.c_uint64 * (k + 1))(*offsets)
        cc = (ct.c_double * max(1, k))(*[float(c) for c, _ in terms])
        vals = (ct.c_double * max(1, k))()
        out = ct.c_double()
        self._check(self.lib.aleph_b200_expectation_sum(self.handle, state.ptr, cq, cp, co, cc, k, ct.byref(out),
                                                        vals if with_terms else None))
        if with_terms:
            return out.value, np.array(vals[:k], dtype=np.float64)
        return out.value

    def probabilities(self, state: State, qubits) -> np.ndarray:
        k = len(qubits)
        qs = (ct.c_uint32 * max(1, k))(*qubits)
        out = np.zeros(1 << k, dtype=np.float64)
        self._check(self.lib.aleph_b200_probabilities(self.handle, state.ptr, qs, k,
                                                      out.ctypes.data_as(ct.POINTER(ct.c_double))))
        return out

    # ---- extras ----------------------------------------------------------------
    def statevector(self, state: State) -> np.ndarray:
        out = np.zeros(2 << state.num_qubits, dtype=np.float64)
        self._check(self.lib.aleph_b200_get_amplitudes(self.handle, state.ptr,
                                                       out.ctypes.data_as(ct.POINTER(ct.c_double))))
        return out[0::2] + 1j * out[1::2]

    def fp64_rate(self) -> float:
        """The FP64 FMA rate of the device's CUDA cores, TFLOP/s, measured now."""
        v = ct.c_double()
        self._check(self.lib.aleph_b200_fp64_rate(self.handle, ct.byref(v)))
        return v.value

    def amplitude_range(self, state: State, first: int, count: int) -> np.ndarray:
        """Amplitudes [first, first + count) of a state of any size."""
        out = np.zeros(2 * max(1, count), dtype=np.float64)
        self._check(self.lib.aleph_b200_get_amplitude_range(self.handle, state.ptr, first, count,
                                                            out.ctypes.data_as(ct.POINTER(ct.c_double))))
        return out[0:2 * count:2] + 1j * out[1:2 * count:2]

    def set_statevector(self, state: State, psi) -> None:
        psi = np.asarray(psi, dtype=np.complex128)
        buf = np.empty(2 * psi.size, dtype=np.float64)
        buf[0::2] = psi.real
        buf[1::2] = psi.imag
        self._check(self.lib.aleph_b200_set_amplitudes(self.handle, state.ptr,
                                                       buf.ctypes.data_as(ct.POINTER(ct.c_double))))

    def norm_sqr(self, state: State) -> float:
        out = ct.c_double()
        self._check(self.lib.aleph_b200_norm_sqr(self.handle, state.ptr, ct.byref(out)))
        return out.value

    def state_memory(self, state: State) -> tuple[int, int]:
        """(device pointer, bytes) of the state's amplitudes, ordered on the
        handle's stream (``stream_ptr``)."""
        ptr, nbytes = ct.c_void_p(), ct.c_uint64()
        self._check(self.lib.aleph_b200_state_memory(self.handle, state.ptr, ct.byref(ptr), ct.byref(nbytes)))
        return int(ptr.value or 0), int(nbytes.value)

    def scale_state(self, state: State, factor: float) -> None:
        """Every amplitude times ``factor`` (> 0), on the device."""
        self._check(self.lib.aleph_b200_scale_state(self.handle, state.ptr, float(factor)))

    def reset_state(self, state: State) -> None:
        """Back to |0...0> on the device, reusing the allocation."""
        self._check(self.lib.aleph_b200_reset_state(self.handle, state.ptr))

    def stream_ptr(self) -> int:
        """The handle's cudaStream_t (every engine kernel runs on it)."""
        p = ct.c_void_p()
        self._check(self.lib.aleph_b200_get_stream(self.handle, ct.byref(p)))
        return p.value or 0

    def synchronize(self):
        self._check(self.lib.aleph_b200_synchronize(self.handle))

    def stats(self) -> dict:
        s = abi.Stats()
        self.lib.aleph_b200_get_stats(self.handle, ct.byref(s))
        return {k: getattr(s, k) for k, _ in abi.Stats._fields_}

    def reset_stats(self):
        self.lib.aleph_b200_reset_stats(self.handle)

    def pass_records(self) -> list[dict]:
        """Per-pass device timings of the last stream run with ``record_passes`` on."""
        n = ct.c_uint64()
        self.lib.aleph_b200_get_pass_records(self.handle, None, 0, ct.byref(n))
        buf = (abi.PassRecord * max(1, n.value))()
        self._check(self.lib.aleph_b200_get_pass_records(self.handle, buf, n.value, ct.byref(n)))
        return [_record_dict(r) for r in buf[: n.value]]

    def apply_stream(self, state: State, instructions, measure_uniforms=None, flat: Flat | None = None):
        """Apply a whole instruction list in one call; returns measurement outcomes."""
        flat = flat or flatten(instructions)
        u = None if measure_uniforms is None else np.ascontiguousarray(np.asarray(measure_uniforms, np.float64))
        outs = (ct.c_uint8 * max(1, flat.n))()
        nout = ct.c_uint64()
        self._check(self.lib.aleph_b200_apply_gate_stream(
            self.handle, state.ptr, flat.instrs, flat.n, ct.byref(flat.pools),
            u.ctypes.data_as(ct.POINTER(ct.c_double)) if u is not None and u.size else None,
            0 if u is None else u.size, outs, flat.n, ct.byref(nout)))
        return [int(outs[i]) for i in range(nout.value)]

    def run_paged(self, circuit: Circuit, tile_qubits: int, depth: int = 3) -> PagedState:
        """``CudaSvBackend::run_paged`` / ``run_paged_overlapped``
        (crates/aleph-cuda/src/sv/paged.rs:138-276): run ``circuit`` with the
        state in pinned host memory, 2^tile_qubits-amplitude tiles streamed
        through the device (``depth`` device buffers; 1 = no copy overlap)."""
        flat = flatten(circuit.instructions)
        out = ct.c_void_p()
        self._check(self.lib.aleph_b200_paged_run(self.handle, circuit.num_qubits, flat.instrs, flat.n,
                                                  ct.byref(flat.pools), int(tile_qubits), int(depth), ct.byref(out)))
        return PagedState(self.lib, out, circuit.num_qubits)

    def qaoa_sweep(self, graphs, gammas, betas) -> np.ndarray:
        """<C> of the build_qaoa Max-Cut circuit (crates/aleph-ir/src/ansatz.rs:71-117)
        for every parameter set k: ``graphs[k] = (num_qubits, [(i, j), ...])``,
        ``gammas[k]`` / ``betas[k]`` of one common length p. One persistent launch."""
        count = len(graphs)
        gam = np.asarray(gammas, dtype=np.float64).reshape(count, -1)
        bet = np.asarray(betas, dtype=np.float64).reshape(count, -1)
        if gam.shape != bet.shape:
            raise ValueError("gammas and betas must have the same shape")
        p = gam.shape[1]
        sets = (abi.QaoaSet * max(1, count))()
        pool = []
        for k, (nq, edges) in enumerate(graphs):
            sets[k].num_qubits, sets[k].num_edges, sets[k].edge_offset = nq, len(edges), len(pool) // 2
            for (i, j) in edges:
                pool += [int(i), int(j)]
        edges_arr = np.ascontiguousarray(np.asarray(pool, dtype=np.uint32))
        ang = np.ascontiguousarray(np.concatenate([gam, bet], axis=1))
        out = np.zeros(max(1, count), dtype=np.float64)
        self._check(self.lib.aleph_b200_qaoa_sweep(
            self.handle, p, sets, count, edges_arr.ctypes.data_as(ct.POINTER(ct.c_uint32)) if edges_arr.size else None,
            edges_arr.size // 2, ang.ctypes.data_as(ct.POINTER(ct.c_double)), out.ctypes.data_as(ct.POINTER(ct.c_double))))
        return out[:count]

    def compile(self, num_qubits: int, instructions) -> "CompiledPlan":
        """``CudaExecutionPlan::compile`` (crates/aleph-cuda/src/execution.rs:78): validate
        and plan once; the plan tables stay resident on the device."""
        flat = instructions if isinstance(instructions, Flat) else flatten(instructions)
        p = ct.c_void_p()
        self._check(self.lib.aleph_b200_compile(self.handle, num_qubits, flat.instrs, flat.n,
                                                ct.byref(flat.pools), ct.byref(p)))
        return CompiledPlan(p, num_qubits, flat, self)


def _record_dict(r) -> dict:
    return {"kind": abi.PASS_KINDS.get(r.kind, r.kind), "gates": r.gates, "n": r.n, "qubits": list(r.qubits[: r.nq]),
            "post_ops": r.post_ops, "lane_ops": r.lane_ops, "dense_ops": r.dense_ops, "diag_ops": r.diag_ops,
            "variant": r.variant, "fma_per_amp": r.fma_per_amp, "ms": r.ms, "bytes": r.bytes}


class CompiledPlan:
    """A plan compiled by :meth:`B200SvBackend.compile`; ``execute`` applies it
    (``CudaExecutionPlan::execute``, crates/aleph-cuda/src/execution.rs:183)."""

    def __init__(self, ptr, num_qubits: int, flat: Flat, backend: B200SvBackend):
        self.ptr, self.num_qubits, self.flat, self.backend = ptr, num_qubits, flat, backend
        self._outs = (ct.c_uint8 * max(1, flat.n))()

    def execute(self, state: State, measure_uniforms=None) -> list[int]:
        b = self.backend
        u = None if measure_uniforms is None else np.ascontiguousarray(np.asarray(measure_uniforms, np.float64))
        nout = ct.c_uint64()
        b._check(b.lib.aleph_b200_execute(
            b.handle, state.ptr, self.ptr,
            u.ctypes.data_as(ct.POINTER(ct.c_double)) if u is not None and u.size else None,
            0 if u is None else u.size, self._outs, self.flat.n, ct.byref(nout)))
        return [int(self._outs[i]) for i in range(nout.value)]

    def free(self) -> None:
        if self.ptr:
            self.backend.lib.aleph_b200_plan_free(self.backend.handle, self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def describe_plan(num_qubits: int, instructions, precision: str = "f64", tile_r: int = 5, smem_max_n: int = 12,
                  block_window_search: bool = True, tile_occupancy: int = 0,
                  relabel_swaps: bool = True, pair_fusion: bool = True) -> list[dict]:
    """The passes the planner makes of ``instructions`` (host only, no device)."""
    lib = abi.load_library()
    flat = instructions if isinstance(instructions, Flat) else flatten(instructions)
    cfg = abi.PlanConfig(abi.PRECISION[precision], tile_r, smem_max_n, int(bool(block_window_search)), tile_occupancy,
                         int(not relabel_swaps), int(not pair_fusion))
    n = ct.c_uint64()
    st = lib.aleph_b200_describe_plan(num_qubits, ct.byref(cfg), flat.instrs, flat.n, ct.byref(flat.pools), None, 0,
                                      ct.byref(n))
    if st != abi.OK:
        raise _ERRORS.get(st, BackendError)(st, abi.STATUS_NAMES.get(st, str(st)))
    buf = (abi.PassRecord * max(1, n.value))()
    lib.aleph_b200_describe_plan(num_qubits, ct.byref(cfg), flat.instrs, flat.n, ct.byref(flat.pools), buf, n.value,
                                 ct.byref(n))
    return [_record_dict(r) for r in buf[: n.value]]


def describe_paged(num_qubits: int, instructions, tile_qubits: int, local_qubits: int):
    """How an out-of-core run cuts ``instructions`` (host only, no device):
    (segment of each instruction, its place in the execution order, segment
    count); barriers get -1 in both lists."""
    lib = abi.load_library()
    flat = instructions if isinstance(instructions, Flat) else flatten(instructions)
    seg = (ct.c_uint64 * max(1, flat.n))()
    pos = (ct.c_uint64 * max(1, flat.n))()
    count = ct.c_uint64()
    st = lib.aleph_b200_describe_paged(num_qubits, flat.instrs, flat.n, tile_qubits, local_qubits, seg, pos,
                                       ct.byref(count))
    if st != abi.OK:
        raise _ERRORS.get(st, BackendError)(st, f"describe_paged: {abi.STATUS_NAMES.get(st, st)}")
    conv = lambda v: -1 if v == 2**64 - 1 else int(v)  # noqa: E731
    return [conv(seg[i]) for i in range(flat.n)], [conv(pos[i]) for i in range(flat.n)], count.value


def run_with_outcomes(backend: B200SvBackend, circuit: Circuit, measure_uniforms=None):
    """``run_with_outcomes`` (crates/aleph-backend/src/lib.rs:211-245)."""
    if circuit.num_qubits == 0 and len(circuit) == 0:
        raise EmptyCircuit(abi.EMPTY_CIRCUIT, "cannot run an empty circuit")  # noqa: F821
    state = backend.allocate(circuit.num_qubits)
    outs = backend.apply_stream(state, circuit.instructions, measure_uniforms)
    records = []
    k = 0
    for idx, inst in enumerate(circuit.instructions):
        if isinstance(inst, Measure):
            records.append(MeasurementRecord(idx, inst.qubit, inst.clbit, bool(outs[k])))
            k += 1
    return state, records


def run(backend: B200SvBackend, circuit: Circuit, measure_uniforms=None) -> State:
    """``run`` (crates/aleph-backend/src/lib.rs:182-185)."""
    state, _ = run_with_outcomes(backend, circuit, measure_uniforms)
    return state
