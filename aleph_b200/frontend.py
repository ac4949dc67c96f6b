"""The user-facing run surface over the engine, mirroring the reference's
Python ``aleph.run`` (crates/aleph-py/src/run.rs:180-360, RunResult :40-135),
``qaoa_energy`` (crates/aleph-py/src/energy.rs:58-90) and the CLI's output
formats (crates/aleph-cli/src/output.rs:13-121, pauli.rs:14-55).

Semantics kept from the reference:

- a circuit runs once; Measure records collapse the state on the way, and
  the ``shots`` samples re-sample that single final state (run.rs:186-189);
- counts are keyed by bitstrings with qubit 0 as the RIGHTMOST character,
  in ascending order (run.rs:55-60, 124-135);
- ``seed=None`` draws an entropy seed (labelled ``seed=entropy``).

Sampled bitstrings come from this engine's own seeded RNG (explicit
variates give the reference's mapping exactly; a seed does not reproduce
the reference's ChaCha12 stream).
"""
from __future__ import annotations

import math
import re
import secrets
from dataclasses import dataclass

import numpy as np

from . import circuit as C
from . import qasm
from .backend import B200SvBackend, run_with_outcomes

DEFAULT_SHOTS = 1024          # crates/aleph-cli/src/exec.rs:66
STATEVECTOR_CAP_QUBITS = 10   # exec.rs:71

# backend names this engine answers to -> the precision they imply (None: the
# `precision` argument decides). "cuda" is the reference's FP64 GPU backend
# and "cuda-f32" its FP32 one; here FP32 runs as TC32 (tensor-core blocks).
BACKENDS = {"b200": None, "auto": None, "gpu": None, "cuda": "f64", "cuda-f32": "tc32"}
PRECISIONS = {"auto": "tc32", "f64": "f64", "f32": "f32", "tc32": "tc32"}


def resolve(backend: str = "b200", precision: str = "auto") -> str:
    """Backend name + precision -> the engine precision ("f64", "f32", "tc32")."""
    if backend not in BACKENDS:
        raise ValueError(f"unknown backend {backend!r}: this engine is the B200 state-vector backend "
                         f"(names: {', '.join(BACKENDS)})")
    if precision not in PRECISIONS:
        raise ValueError(f"unknown precision {precision!r} (expected one of {', '.join(PRECISIONS)})")
    forced = BACKENDS[backend]
    if forced and precision not in ("auto", forced):
        raise ValueError(f"backend {backend!r} runs {forced}; precision {precision!r} contradicts it")
    return forced or PRECISIONS[precision]


def counts_map(samples, num_qubits: int) -> dict[str, int]:
    """Shot indices -> {bitstring: count}, ascending; qubit 0 rightmost."""
    vals, cnt = np.unique(np.asarray(samples, dtype=np.uint64), return_counts=True)
    return {format(int(v), f"0{num_qubits}b"): int(c) for v, c in zip(vals, cnt)}


class RunResult:
    """A run's shot histogram and final state (``RunResult``, run.rs:40-122).

    The state stays on the device until ``statevector()`` is first called;
    that call caches the host copy and releases the device state."""

    def __init__(self, backend: B200SvBackend, state, counts: dict, outcomes: list, seed_label: str):
        self._backend, self._state = backend, state
        self._counts, self._outcomes, self.seed_label = counts, outcomes, seed_label
        self._amps = None
        self.num_qubits = state.num_qubits

    def counts(self) -> dict[str, int]:
        return dict(self._counts)

    def statevector(self) -> np.ndarray:
        """complex128 array of shape (2**n,), index bit q = qubit q."""
        if self._amps is None:
            self._amps = self._backend.statevector(self._state)
            self._release_state()
        return self._amps.copy()

    def measurements(self) -> list:
        """The mid-circuit Measure records (instruction, qubit, clbit, outcome)."""
        return list(self._outcomes)

    def expectation(self, pauli: str) -> float:
        """⟨ψ|P|ψ⟩ for a Pauli argument like ``"ZZ"`` or ``"1.5*XIZ"`` (qubit 0 leftmost)."""
        coeff, terms = parse_pauli_arg(pauli)
        if terms and terms[-1][0] >= self.num_qubits:
            raise ValueError(f"{pauli!r} references qubit {terms[-1][0]} but the circuit has "
                             f"{self.num_qubits} qubits")
        if self._state is None:
            return _expectation_host(self._amps, coeff, terms)
        return self._backend.expectation_value(self._state, terms, coeff)

    def execution_stats(self) -> dict:
        return self._backend.stats()

    def _release_state(self):
        if self._state is not None:
            self._state.free()
            self._state = None

    def close(self):
        self._release_state()
        if self._backend is not None:
            self._backend.close()
            self._backend = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _expectation_host(amps, coeff, terms) -> float:
    # after the device state was released: apply the Pauli string to a copy
    phi = np.array(amps, copy=True)
    idx = np.arange(phi.size, dtype=np.int64)
    for q, p in terms:
        bit = (idx >> q) & 1
        if p in ("X", "Y"):
            phi = phi[idx ^ (1 << q)]
        if p == "Y":
            phi = phi * np.where(bit == 1, 1j, -1j)
        elif p == "Z":
            phi = phi * np.where(bit == 1, -1.0, 1.0)
    return float(coeff * np.vdot(amps, phi).real)


def run(circuit, *, shots: int = DEFAULT_SHOTS, backend: str = "b200", precision: str = "auto",
        seed: int | None = None) -> RunResult:
    """Run ``circuit`` (a Circuit, or OpenQASM 3 source text) once on one
    B200 and sample ``shots`` bitstrings from the final state."""
    if isinstance(circuit, str):
        circuit = qasm.parse(circuit)
    if shots < 0:
        raise ValueError("shots must be >= 0")
    prec = resolve(backend, precision)
    run_seed = seed if seed is not None else secrets.randbits(64)
    be = B200SvBackend(seed=run_seed, precision=prec)
    try:
        state, outcomes = run_with_outcomes(be, circuit)
        samples = be.sample(state, shots) if shots else np.zeros(0, dtype=np.uint64)
    except BaseException:
        be.close()
        raise
    label = f"seed={seed}" if seed is not None else "seed=entropy"
    return RunResult(be, state, counts_map(samples, circuit.num_qubits), outcomes, label)


class PauliSumError(ValueError):
    """``PauliSumError`` (crates/aleph-core/src/pauli.rs:89-108)."""


# Rust's f64 grammar (what `str::parse::<f64>` accepts): optional sign, then
# inf / infinity / nan in any case, or digits with an optional point and
# exponent (".5" and "5." included; no underscores, no surrounding spaces)
_RUST_F64 = re.compile(r"[+-]?(?:inf|infinity|nan|(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?)", re.IGNORECASE)


def _rust_debug_str(s: str) -> str:
    out = []
    for ch in s:
        if ch in ('"', "\\"):
            out.append("\\" + ch)
        elif ch == "\n":
            out.append("\\n")
        elif ch == "\r":
            out.append("\\r")
        elif ch == "\t":
            out.append("\\t")
        elif not ch.isprintable():
            out.append(f"\\u{{{ord(ch):x}}}")
        else:
            out.append(ch)
    return '"' + "".join(out) + '"'


def _rust_debug_char(ch: str) -> str:
    return "'" + ("\\'" if ch == "'" else _rust_debug_str(ch)[1:-1].replace('\\"', '"')) + "'"


def _rust_lines(src: str):
    """``str::lines``: split at \\n, drop one \\r before each \\n, no empty last line."""
    parts = src.split("\n")
    if parts and parts[-1] == "":
        parts.pop()
    for i, p in enumerate(parts):
        if p.endswith("\r") and (i < len(parts) - 1 or src.endswith("\n")):
            p = p[:-1]
        yield p


class PauliSum:
    """``PauliSum`` (crates/aleph-core/src/pauli.rs:84-170): terms as
    (coefficient, [(qubit, letter), ...]) with the qubits ascending and
    identity factors dropped, as ``PauliString::new`` (pauli.rs:48-60) keeps them."""

    def __init__(self, terms):
        self.terms = list(terms)

    @staticmethod
    def parse(src: str, n_qubits: int) -> "PauliSum":
        """One term per line, ``<coeff> <pauli>``; character i of ``<pauli>``
        is the Pauli on qubit i; blank lines and ``#`` lines are skipped."""
        terms = []
        for idx, raw in enumerate(_rust_lines(src)):
            line = idx + 1
            trimmed = raw.strip()
            if not trimmed or trimmed.startswith("#"):
                continue
            parts = trimmed.split()
            if len(parts) != 2:
                raise PauliSumError(f"line {line}: expected '<coeff> <pauli>', got {_rust_debug_str(raw)}")
            coeff_s, pauli_s = parts
            if not _RUST_F64.fullmatch(coeff_s):
                raise PauliSumError(f"line {line}: coefficient {_rust_debug_str(coeff_s)} is not a finite float")
            coeff = float(coeff_s)
            if len(pauli_s) != n_qubits:
                raise PauliSumError(f"line {line}: pauli string has {len(pauli_s)} chars, expected {n_qubits}")
            factors = []
            for q, ch in enumerate(pauli_s):
                if ch not in "IXYZ":
                    raise PauliSumError(f"line {line}: {_rust_debug_char(ch)} is not one of I,X,Y,Z")
                if ch != "I":
                    factors.append((q, ch))
            if not math.isfinite(coeff):
                raise PauliSumError(f"line {line}: non-finite coefficient")
            terms.append((coeff, factors))
        return PauliSum(terms)

    @staticmethod
    def load(path: str, n_qubits: int) -> "PauliSum":
        """``PauliSum.load`` (crates/aleph-py/src/energy.rs:24-31)."""
        try:
            with open(path, encoding="utf-8") as f:
                src = f.read()
        except OSError as e:
            raise ValueError(f"read {path}: {e}") from e
        try:
            return PauliSum.parse(src, n_qubits)
        except PauliSumError as e:
            raise ValueError(f"parse {path}: {e}") from e

    def num_terms(self) -> int:
        return len(self.terms)


def hea_energy(n_qubits: int, depth: int, thetas, ham: PauliSum, backend: str = "b200",
               precision: str = "f64") -> float:
    """⟨ψ(θ)|H|ψ(θ)⟩ of the Ry + CNOT hardware-efficient ansatz (``hea_energy``,
    crates/aleph-py/src/energy.rs:40-55): ``build_hea`` then one fused
    Pauli-sum expectation of ``ham``."""
    from . import workloads

    circuit = workloads.build_hea(n_qubits, depth, list(thetas))
    be = B200SvBackend(seed=0, precision=resolve(backend, precision))
    try:
        state, _ = run_with_outcomes(be, circuit)
        return float(be.expectation_sum(state, ham.terms))
    finally:
        be.close()


def qaoa_energy(n_qubits: int, edges, gammas, betas, backend: str = "b200", precision: str = "f64") -> float:
    """⟨H_C⟩ of QAOA Max-Cut (``build_qaoa`` + ``maxcut_pauli_sum``,
    crates/aleph-ir/src/ansatz.rs:71-117) at the given angles: one set of
    the batched sweep kernel (n <= 26), or the gate stream plus one fused
    Pauli-sum expectation (every ⟨Z_i Z_j⟩ in shared sweeps) beyond it."""
    return float(qaoa_energies([(n_qubits, list(edges))], [gammas], [betas], backend, precision)[0])


def qaoa_energies(graphs, gammas, betas, backend: str = "b200", precision: str = "f64",
                  sweep_max_n: int = 26) -> np.ndarray:
    """Batched ``qaoa_energy``: graphs = [(n, [(u, v), ...]), ...], one angle
    row per graph. Sets of up to ``sweep_max_n`` (<= 26) qubits and 128 edges
    run as one persistent launch; larger ones run gate by gate."""
    from . import workloads

    prec = resolve(backend, precision)
    if prec == "tc32":
        prec = "f32"  # the sweep kernel streams FP32 states on CUDA cores
    gammas = np.atleast_2d(np.asarray(gammas, dtype=np.float64))
    betas = np.atleast_2d(np.asarray(betas, dtype=np.float64))
    if gammas.shape != betas.shape or gammas.shape[0] != len(graphs):
        raise ValueError("need one row of gammas and betas (same length p) per graph")
    be = B200SvBackend(seed=0, precision=prec)
    try:
        small = [i for i, (n, e) in enumerate(graphs) if n <= min(sweep_max_n, 26) and len(e) <= 128]
        out = np.zeros(len(graphs), dtype=np.float64)
        if small:
            out[small] = be.qaoa_sweep([graphs[i] for i in small], gammas[small], betas[small])
        for i, (n, e) in enumerate(graphs):
            if i in small:
                continue
            st = be.allocate(n)
            be.apply_stream(st, workloads.qaoa_maxcut(n, e, gammas[i], betas[i]).instructions)
            out[i] = be.expectation_sum(st, workloads.maxcut_pauli_sum(n, e))
            st.free()
        return out
    finally:
        be.close()


# ---- the CLI's text formats (crates/aleph-cli/src/output.rs) ------------------
def parse_pauli_arg(raw: str):
    """``[coeff "*"] {I|X|Y|Z}+`` (pauli.rs:14-55): position i is qubit i; I
    terms are dropped. Returns (coefficient, [(qubit, letter), ...])."""
    coeff, body = 1.0, raw
    star = raw.find("*")
    if star >= 0:
        try:
            coeff, body = float(raw[:star]), raw[star + 1:]
        except ValueError:
            coeff, body = 1.0, raw
    if not body:
        raise ValueError("empty Pauli string")
    terms = []
    for i, ch in enumerate(body):
        if ch not in "IXYZ":
            raise ValueError(f"invalid character {ch!r} in Pauli string (allowed: I, X, Y, Z)")
        if ch != "I":
            terms.append((i, ch))
    if not math.isfinite(coeff):
        raise ValueError(f"non-finite Pauli coefficient {coeff}")
    return coeff, terms


def _rust_exp(x: float) -> str:
    """``{:+.16e}`` as Rust prints it: exponent without '+' or leading zeros."""
    s = f"{x:+.16e}"
    mant, exp = s.split("e")
    return f"{mant}e{int(exp)}"


def format_counts(counts: dict, total: int, num_qubits: int, seed_label: str) -> str:
    lines = [f"counts ({total} shots, {seed_label}):"]
    for bits, count in sorted(counts.items()):
        lines.append(f"  |{bits}⟩  {count}  ({count / total if total else 0.0:.4f})")
    return "\n".join(lines) + "\n"


def format_statevector(amps, num_qubits: int) -> str:
    lines = [f"statevector ({num_qubits} qubits, {len(amps)} amplitudes):"]
    for i, a in enumerate(amps):
        a = complex(a)
        p = a.real * a.real + a.imag * a.imag
        lines.append(f"  |{i:0{num_qubits}b}⟩   {_rust_exp(a.real)} {_rust_exp(a.imag)}i  |a|² = {p:.6f}")
    return "\n".join(lines) + "\n"


def format_expectation(raw: str, value: float) -> str:
    return f"  {raw}    {value:+.16f}\n"


def format_duration(seconds: float) -> str:
    """Rust's ``{:.1?}`` for a Duration: the largest unit with a non-zero integer part."""
    ns = seconds * 1e9
    if ns >= 1e9:
        return f"{ns / 1e9:.1f}s"
    if ns >= 1e6:
        return f"{ns / 1e6:.1f}ms"
    if ns >= 1e3:
        return f"{ns / 1e3:.1f}µs"
    return f"{ns:.1f}ns"
