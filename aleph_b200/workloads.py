"""Seeded synthetic workloads with the shapes of the benchmark configurations.

* ``brickwall``: random brickwall — every layer applies a Haar-random SU(2)
  (from the seed) to each qubit, then CZ on nearest-neighbour pairs (i, i+1),
  even offsets on even layers and odd offsets on odd layers.
* ``qft_product``: a random product state (Ry(theta) Rz(phi) per qubit,
  theta, phi uniform in [0, 2 pi)) followed by the textbook QFT (H plus
  controlled-phase 2 pi / 2^k on every pair) and the bit-reversal SWAPs.
* ``qaoa_maxcut``: QAOA on a random 3-regular graph as ``build_qaoa``
  (crates/aleph-ir/src/ansatz.rs:71-98): H layer, per edge CX Rz(2 gamma) CX,
  Rx(2 beta) mixer, p layers.

All data are synthetic (generated here from seeds); no benchmark suite items
are reproduced.
"""
from __future__ import annotations

import math

import numpy as np

from . import circuit as C


def haar_su2(rng: np.random.Generator) -> np.ndarray:
    """Haar-random SU(2): QR of a complex Gaussian matrix, phase-fixed, det = 1."""
    z = (rng.standard_normal((2, 2)) + 1j * rng.standard_normal((2, 2))) / math.sqrt(2.0)
    q, r = np.linalg.qr(z)
    d = np.diag(r)
    q = q * (d / np.abs(d))
    q = q / np.sqrt(np.linalg.det(q))
    return q


def brickwall(n: int, depth: int, seed: int = 0) -> C.Circuit:
    rng = np.random.default_rng(seed)
    c = C.Circuit(n)
    for layer in range(depth):
        for q in range(n):
            c.add(C.Unitary1q(haar_su2(rng)), [q])
        for q in range(layer % 2, n - 1, 2):
            c.add(C.Cz(), [q, q + 1])
    return c


def qft_product(n: int, seed: int = 0, swaps: bool = True) -> C.Circuit:
    rng = np.random.default_rng(seed)
    c = C.Circuit(n)
    for q in range(n):
        th, ph = rng.uniform(0.0, 2.0 * math.pi, size=2)
        c.add(C.Ry(th), [q])
        c.add(C.Rz(ph), [q])
    for j in range(n - 1, -1, -1):
        c.add(C.H(), [j])
        for k in range(j - 1, -1, -1):
            # controlled phase 2*pi / 2^(j-k+1), control k, target j
            c.add(C.Phase(2.0 * math.pi / (2 ** (j - k + 1))), [j], controls=[k])
    if swaps:
        for q in range(n // 2):
            c.add(C.Swap(), [q, n - 1 - q])
    return c


def random_3_regular(n: int, rng: np.random.Generator) -> list[tuple[int, int]]:
    """Pairing model with rejection: a uniformly random simple 3-regular graph."""
    if (3 * n) % 2:
        raise ValueError("3-regular graphs need an even vertex count")
    while True:
        stubs = np.repeat(np.arange(n), 3)
        rng.shuffle(stubs)
        edges = set()
        ok = True
        for a, b in zip(stubs[0::2], stubs[1::2]):
            a, b = int(a), int(b)
            if a == b or (min(a, b), max(a, b)) in edges:
                ok = False
                break
            edges.add((min(a, b), max(a, b)))
        if ok:
            return sorted(edges)


def qaoa_maxcut(n: int, edges, gammas, betas) -> C.Circuit:
    c = C.Circuit(n)
    for q in range(n):
        c.add(C.H(), [q])
    for g, b in zip(gammas, betas):
        for (i, j) in edges:
            c.add(C.Cnot(), [i, j])
            c.add(C.Rz(2.0 * g), [j])
            c.add(C.Cnot(), [i, j])
        for q in range(n):
            c.add(C.Rx(2.0 * b), [q])
    return c


def _toffoli_ct(c: C.Circuit, a: int, b: int, t: int) -> None:
    """Toffoli(a, b -> t) in CX, T, Tdg and H (the standard 6-CX circuit)."""
    c.add(C.H(), [t])
    c.add(C.Cnot(), [b, t]).add(C.Tdg(), [t]).add(C.Cnot(), [a, t]).add(C.T(), [t])
    c.add(C.Cnot(), [b, t]).add(C.Tdg(), [t]).add(C.Cnot(), [a, t])
    c.add(C.T(), [b]).add(C.T(), [t]).add(C.H(), [t])
    c.add(C.Cnot(), [a, b]).add(C.T(), [a]).add(C.Tdg(), [b]).add(C.Cnot(), [a, b])


def _mcz_ct(c: C.Circuit, qs: list[int], anc: list[int]) -> None:
    """Z controlled on all of qs (|1..1> gets -1) with a V-chain of Toffolis
    through the ancillas (computed, used, uncomputed), each in CX + T gates."""
    if len(qs) == 1:
        c.add(C.Z(), [qs[0]])
        return
    if len(qs) == 2:
        c.add(C.Cz(), qs)
        return
    *ctrl, t = qs
    c.add(C.H(), [t])
    if len(ctrl) == 2:
        _toffoli_ct(c, ctrl[0], ctrl[1], t)
    else:
        chain = [(ctrl[0], ctrl[1], anc[0])]
        for i in range(2, len(ctrl) - 1):
            chain.append((ctrl[i], anc[i - 2], anc[i - 1]))
        for g in chain:
            _toffoli_ct(c, *g)
        _toffoli_ct(c, ctrl[-1], anc[len(ctrl) - 3], t)
        for g in reversed(chain):
            _toffoli_ct(c, *g)
    c.add(C.H(), [t])


def grover(n_data: int, marked: int, iterations: int) -> C.Circuit:
    """Grover search over n_data qubits for the bitstring `marked`, with the
    oracle's and the diffuser's multi-controlled Z decomposed into CX and T
    gates through n_data - 2 ancillas (qubits n_data .. 2 n_data - 3)."""
    n = max(n_data, 2 * n_data - 2)
    c = C.Circuit(n)
    data = list(range(n_data))
    anc = list(range(n_data, n))
    for q in data:
        c.add(C.H(), [q])
    for _ in range(iterations):
        zeros = [q for q in data if not (marked >> q) & 1]
        for q in zeros:
            c.add(C.X(), [q])
        _mcz_ct(c, data, anc)
        for q in zeros:
            c.add(C.X(), [q])
        for q in data:
            c.add(C.H(), [q]).add(C.X(), [q])
        _mcz_ct(c, data, anc)
        for q in data:
            c.add(C.X(), [q]).add(C.H(), [q])
    return c


def build_hea(n: int, depth: int, params) -> C.Circuit:
    """``build_hea`` (crates/aleph-ir/src/ansatz.rs:32-61): ``depth`` layers of
    Ry on every qubit followed by the CNOT chain (q, q+1), then a final Ry
    layer; ``params[layer * n + q]`` drives qubit q in rotation layer
    ``layer`` (0..=depth)."""
    expected = n * (depth + 1)
    if len(params) != expected:
        raise ValueError(f"expected {expected} params (n_qubits*(depth+1)), got {len(params)}")
    c = C.Circuit(n)
    for layer in range(depth + 1):
        for q in range(n):
            c.add(C.Ry(float(params[layer * n + q])), [q])
        if layer < depth:
            for q in range(n - 1):
                c.add(C.Cnot(), [q, q + 1])
    return c


def maxcut_pauli_sum(n: int, edges):
    """``maxcut_pauli_sum`` (crates/aleph-ir/src/ansatz.rs:105-117): the
    identity with coefficient |E|/2, then -1/2 Z_i Z_j per edge, as
    (coefficient, [(qubit, letter), ...]) terms for ``expectation_sum``."""
    terms = [(0.5 * len(edges), [])]
    for (i, j) in edges:
        if i >= n or j >= n:
            raise ValueError(f"edge ({i}, {j}) out of range for {n} qubits")
        terms.append((-0.5, [(i, "Z"), (j, "Z")]))
    return terms


def splitmix64_words(seed: int, count: int) -> np.ndarray:
    """Deterministic u64 variates (splitmix64) shared by the engine and the oracle in tests."""
    out = np.empty(count, dtype=np.uint64)
    x = seed & 0xFFFFFFFFFFFFFFFF
    M = 0xFFFFFFFFFFFFFFFF
    for i in range(count):
        x = (x + 0x9E3779B97F4A7C15) & M
        z = x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        out[i] = z ^ (z >> 31)
    return out
