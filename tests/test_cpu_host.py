"""CPU-side tests: the C-ABI library loads and exports every declared
symbol, the host-side stream flattening, the workload generators, and
oracle known-answer tests from the reference's own unit tests."""
import ctypes as ct
import math

import numpy as np
import pytest

from aleph_b200 import abi
from aleph_b200 import circuit as C
from aleph_b200 import workloads
from oracle import oracle


def test_library_exports_every_declared_symbol():
    lib = abi.load_library()
    declared = abi.declared_symbols()
    assert len(declared) >= 24
    for name in declared:
        assert hasattr(lib, name), name
        assert name in abi._SIGNATURES, f"{name} has no ctypes signature"


def test_create_without_gpu_reports_device_failure():
    import torch

    if torch.cuda.is_available():
        pytest.skip("GPU present")
    lib = abi.load_library()
    h = ct.c_void_p()
    assert lib.aleph_b200_create(0, 0, 0, ct.byref(h)) == abi.DEVICE_FAILURE
    assert lib.aleph_b200_create(0, 0, 7, ct.byref(h)) == abi.INVALID_ARGUMENT


def test_record_layout_matches_header():
    # struct aleph_b200_instr: 4*4 + 8*4 + 8*4 + 3*8 + 8 + 8 bytes
    assert ct.sizeof(abi.Instr) == 120
    assert ct.sizeof(abi.PhaseTerm) == 16
    assert ct.sizeof(abi.ErrorInfo) == 4 * 8 + 8 + 32


def test_flatten_roundtrip():
    c = C.Circuit(4)
    c.add(C.U3(0.1, 0.2, 0.3), [2]).add(C.Unitary2q(np.eye(4)), [0, 3], [1]).measure(2, 5)
    c.instructions.append(C.DiagonalPhase(4, [C.PhaseTerm((0b11, 0b100), 0.5), C.PhaseTerm((), 0.1)]))
    c.instructions.append(C.TiledBlock([C.GateInstance(C.H(), [0])], 15))
    f = C.flatten(c)
    assert f.n == 6
    assert f.instrs[0].kind == abi.KIND["U3"] and list(f.instrs[0].params) == [0.1, 0.2, 0.3]
    assert f.instrs[1].num_controls == 1 and f.instrs[1].controls[0] == 1 and f.instrs[1].data_len == 16
    assert f.instrs[2].kind == abi.INSTR_MEASURE and f.instrs[2].aux == 5
    assert f.instrs[3].kind == abi.INSTR_DIAGONAL_PHASE and f.instrs[3].data_len == 2
    assert list(f.conds) == [0b11, 0b100]
    assert f.instrs[4].kind == abi.INSTR_TILED_BLOCK and f.instrs[4].data_len == 1
    assert f.instrs[5].kind == abi.KIND["H"]


def test_haar_su2_is_special_unitary():
    rng = np.random.default_rng(0)
    for _ in range(20):
        u = workloads.haar_su2(rng)
        assert np.allclose(u @ u.conj().T, np.eye(2), atol=1e-14)
        assert abs(np.linalg.det(u) - 1) < 1e-14


def test_brickwall_shape():
    c = workloads.brickwall(20, 20, seed=0)
    assert c.gate_count() == 20 * 20 + 10 * 10 + 10 * 9


def test_random_3_regular():
    rng = np.random.default_rng(1)
    for n in (12, 16, 24):
        e = workloads.random_3_regular(n, rng)
        deg = np.zeros(n, int)
        for a, b in e:
            deg[a] += 1
            deg[b] += 1
        assert (deg == 3).all() and len(set(e)) == len(e)


# ---- oracle known-answer tests (reference unit tests) -------------------------
def test_oracle_exact_inverse_boundaries():
    # Boundary known-answer test in the shape of the reference GPU sampler's
    # (crates/aleph-cuda/src/sv/sampling.rs:466-527: mass on indices 1, 255,
    # 256, 511), with exactly representable probabilities so the expected
    # outcomes of cumulative_index (strict `target < cumulative`, zero bins
    # skipped, crates/aleph-sv/src/sampling.rs:59-81) are known in closed form.
    psi = np.zeros(512, dtype=np.complex128)
    psi[[1, 255, 256, 511]] = 0.5
    u = [0.0, np.nextafter(0.25, 0), 0.25, np.nextafter(0.5, 0), 0.5, 0.75, np.nextafter(1.0, 0)]
    assert list(oracle.sample_cumulative(psi, u)) == [1, 1, 255, 255, 256, 511, 511]


def test_oracle_cumulative_boundaries():
    # crates/aleph-sv/src/sampling.rs:205-219: strict comparison skips zero
    # bins and an exact boundary moves to the next positive bin
    psi = np.array([0, 0.5, 0, 0.5, 0.5, 0, 0.5, 0], dtype=np.complex128)
    assert oracle.sample_cumulative(psi, [0.25])[0] == 3
    assert oracle.sample_cumulative(psi, [0.0])[0] == 1
    psi = np.array([0, 1, 0, 0], dtype=np.complex128)
    assert oracle.sample_cumulative(psi, [0.0])[0] == 1
    assert oracle.sample_cumulative(psi, [np.nextafter(1.0, 0)])[0] == 1


def test_oracle_alias_table_reconstructs_distribution():
    rng = np.random.default_rng(2)
    p = rng.random(64)
    p /= p.sum()
    prob, alias = oracle.alias_table(p)
    n = p.size
    recon = prob.copy()
    for j in range(n):
        if alias[j] != j:
            recon[alias[j]] += 1.0 - prob[j]
    assert np.allclose(recon / n, p, atol=1e-12)


def test_oracle_alias_uniform_self_aliased():
    prob, alias = oracle.alias_table(np.full(16, 1 / 16))
    assert (prob == 1.0).all() and (alias == np.arange(16)).all()


def test_oracle_expectation_sign_tables():
    # crates/aleph-sv/src/backend.rs:686-714: |0> -> <Z>=1, |1> -> -1, |+> -> <X>=1
    z0 = np.array([1, 0], dtype=np.complex128)
    z1 = np.array([0, 1], dtype=np.complex128)
    plus = np.array([1, 1], dtype=np.complex128) / math.sqrt(2)
    plus_i = np.array([1, 1j], dtype=np.complex128) / math.sqrt(2)
    assert oracle.expectation(z0, [(0, "Z")]) == 1.0
    assert oracle.expectation(z1, [(0, "Z")]) == -1.0
    assert abs(oracle.expectation(plus, [(0, "X")]) - 1.0) < 1e-15
    assert abs(oracle.expectation(plus_i, [(0, "Y")]) - 1.0) < 1e-15
    assert oracle.expectation(z0, [], 2.5) == 2.5


def test_oracle_matches_numpy_dense_reference():
    """Independent check of the oracle's operand order with numpy kron products."""
    rng = np.random.default_rng(3)
    n = 5
    c = C.Circuit(n)
    mats = []
    for _ in range(15):
        qs = [int(x) for x in rng.permutation(n)[:2]]
        z = rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4))
        q, _ = np.linalg.qr(z)
        c.add(C.Unitary2q(q), qs)
        mats.append((q, qs))
    psi, _ = oracle.run(n, c.instructions)
    ref = np.zeros(1 << n, dtype=np.complex128)
    ref[0] = 1
    for m, (a, b) in mats:
        t = ref.reshape([2] * n)  # axis k <-> qubit n-1-k
        t = np.moveaxis(t, [n - 1 - a, n - 1 - b], [0, 1])
        sh = t.shape
        t = (m @ t.reshape(4, -1)).reshape(sh)
        ref = np.moveaxis(t, [0, 1], [n - 1 - a, n - 1 - b]).reshape(-1)
    assert np.abs(psi - ref).max() < 1e-13


def test_oracle_errors():
    with pytest.raises(oracle.OracleError) as e:
        oracle.run(2, [C.GateInstance(C.H(), [2])])
    assert e.value.status == abi.QUBIT_OUT_OF_RANGE
    with pytest.raises(oracle.OracleError) as e:
        oracle.run(2, [C.GateInstance(C.Unitary1q([[1, 1], [0, 1]]), [0])])
    assert e.value.status == abi.NON_UNITARY_MATRIX
    with pytest.raises(oracle.OracleError) as e:
        oracle.run(2, [C.Reset(0)])
    assert e.value.status == abi.UNSUPPORTED_INSTRUCTION


# ---- planner (host only) -------------------------------------------------------
def test_describe_plan_counts_passes_without_a_device():
    from aleph_b200.backend import describe_plan

    c = workloads.brickwall(32, 40, seed=0)
    greedy = describe_plan(32, c.instructions, "tc32", block_window_search=False)
    search = describe_plan(32, c.instructions, "tc32", block_window_search=True)
    assert all(p["kind"] == "block" for p in search)
    # every gate lands in exactly one pass
    assert sum(p["gates"] for p in search) == sum(p["gates"] for p in greedy) == c.gate_count()
    # the 6-qubit window search follows the brickwall light cone: far fewer passes
    assert len(search) <= 72 < len(greedy)
    f64 = describe_plan(32, c.instructions, "f64")
    assert all(p["kind"] == "tile" for p in f64) and sum(p["gates"] for p in f64) == c.gate_count()
    assert all(p["bytes"] == 2 * 16 * 2.0**32 for p in f64)


def test_describe_plan_reports_validation_errors():
    from aleph_b200.backend import BackendError, describe_plan

    with pytest.raises(BackendError) as e:
        describe_plan(4, [C.GateInstance(C.H(), [4])])
    assert e.value.status == abi.QUBIT_OUT_OF_RANGE


def test_swaps_relabel_into_permutation_passes():
    from aleph_b200.backend import BackendError, describe_plan

    def kinds(n, instrs, **kw):
        return [p["kind"] for p in describe_plan(n, instrs, **kw)]

    sw = lambda a, b, ctrl=(): C.GateInstance(C.Gate("Swap"), [a, b], list(ctrl))
    # the QFT's bit reversal is one involution: one permutation pass instead of tile passes
    c = workloads.qft_product(30, 0)
    on, off = describe_plan(30, c.instructions), describe_plan(30, c.instructions, relabel_swaps=False)
    assert [p["kind"] for p in on].count("permute") == 1 and "permute" not in [p["kind"] for p in off]
    assert len(on) <= len(off) - 4
    assert sum(p["gates"] for p in on) == sum(p["gates"] for p in off) == c.gate_count()
    # a 3-cycle of qubit labels is two involutions; a swap undone costs nothing
    assert kinds(20, [sw(0, 1), sw(1, 2)]) == ["permute", "permute"]
    assert kinds(20, [sw(3, 17), sw(17, 3)]) == []
    assert kinds(20, [sw(3, 17)]) == ["permute"]
    # any relabeling settles in at most two involution passes: a 20-cycle, a
    # 5-cycle beside disjoint transpositions, and a product of disjoint swaps
    cycle = [sw(q, q + 1) for q in range(19)]
    assert kinds(20, cycle) == ["permute", "permute"]
    mixed = [sw(0, 1), sw(1, 2), sw(2, 3), sw(3, 4), sw(10, 11), sw(12, 19)]
    assert kinds(20, mixed) == ["permute", "permute"]
    assert kinds(20, [sw(0, 19), sw(5, 6), sw(8, 13)]) == ["permute"]
    # a controlled SWAP is a gate; so is any SWAP of a state that fits one shared-memory pass
    assert kinds(20, [sw(3, 17, [5])]) == ["tile"]
    assert kinds(12, [sw(3, 7)]) == ["smem"]
    # the labels settle before a DiagonalPhase record, whose masks are logical
    dp = C.DiagonalPhase(20, [C.PhaseTerm((1 << 19,), 0.5)])
    assert kinds(20, [sw(0, 19), dp, C.GateInstance(C.H(), [0])]) == ["permute", "tile"]
    # errors name the qubits as written, and a bad SWAP is still rejected
    with pytest.raises(BackendError) as e:
        describe_plan(20, [sw(0, 19), sw(4, 20)])
    assert e.value.status == abi.QUBIT_OUT_OF_RANGE


# ---- learned planner: host logic ---------------------------------------------------------
def test_learned_candidates_and_features():
    from aleph_b200 import learned
    from aleph_b200.backend import describe_plan

    for prec in ("f64", "f32", "tc32"):
        cs = learned.candidates(prec)
        assert len(set(cs)) == len(cs) and cs[0] == learned.GREEDY
    assert any(not c.tensor_blocks for c in learned.candidates("tc32"))
    c = workloads.brickwall(24, 12, seed=3)
    recs = describe_plan(24, c.instructions, "tc32")
    X = np.stack([learned.pass_features(r, "tc32") for r in recs])
    assert X.shape == (len(recs), learned.N_FEATURES) and np.isfinite(X).all()
    assert (X[:, 1] == 1).all()  # every pass is a tensor-core block
    assert sum(r["dense_ops"] + r["diag_ops"] for r in recs) == c.gate_count()
    t = describe_plan(24, c.instructions, "f64", tile_r=4, tile_occupancy=3, pair_fusion=False)
    assert all(r["variant"] == 3 and len(r["qubits"]) == 4 for r in t)
    assert sum(r["dense_ops"] + r["diag_ops"] for r in t) == c.gate_count()
    # pair fusion: one 4x4 op stands for several gates; the pass still counts them all
    f = describe_plan(24, c.instructions, "f64", tile_r=4, tile_occupancy=3)
    assert sum(r["gates"] for r in f) == c.gate_count()
    assert sum(r["dense_ops"] + r["diag_ops"] for r in f) < c.gate_count()


def test_grover_workload_amplifies_the_marked_state():
    for nd, marked, it in [(3, 5, 1), (5, 17, 3)]:
        c = workloads.grover(nd, marked, it)
        psi, _ = oracle.run(c.num_qubits, c.instructions)
        p = (np.abs(psi) ** 2).reshape(-1, 1 << nd)
        assert p[0, marked] > 0.75  # ancillas back in |0>, marked state amplified
        assert abs(p[1:].sum()) < 1e-12


def _gate_qubits(inst):
    return set(inst.qubits) | set(inst.controls)


def test_paged_segments_keep_dependencies_and_budget():
    """Out-of-core segmentation (host only): every segment gathers at most
    local - m high qubits; gates that share a qubit keep their order; later
    gates move ahead only across gates they share no qubit with."""
    from aleph_b200.backend import describe_paged

    for n, m, local, seed in ((16, 8, 12, 1), (20, 12, 15, 2), (12, 4, 9, 3)):
        c = workloads.brickwall(n, 6, seed=seed)
        c.add(C.Toffoli(), [n - 1, 0, n - 3]).add(C.Swap(), [2, n - 2])
        seg, pos, count = describe_paged(n, c.instructions, m, local)
        gates = c.instructions
        assert all(s >= 0 for s in seg) and sorted(pos) == list(range(len(gates)))
        for s in range(count):
            high = set()
            for i, g in enumerate(gates):
                if seg[i] == s:
                    high |= {q for q in _gate_qubits(g) if q >= m}
            assert len(high) <= local - m
        for i in range(len(gates)):
            for j in range(i + 1, len(gates)):
                if _gate_qubits(gates[i]) & _gate_qubits(gates[j]):
                    assert pos[i] < pos[j] and seg[i] <= seg[j]
        assert count < len(gates)


def test_paged_segments_merge_across_commuting_gates():
    """Two alternating bands of high qubits: a program-order cut would open a
    segment per band switch; commuting gates are pulled forward instead."""
    from aleph_b200.backend import describe_paged

    n, m = 14, 6
    c = C.Circuit(n)
    for _ in range(6):
        c.add(C.Cnot(), [0, 8]).add(C.Cnot(), [1, 9])      # band {8, 9}
        c.add(C.Cnot(), [2, 12]).add(C.Cnot(), [3, 13])    # band {12, 13}
    seg, _, count = describe_paged(n, c.instructions, m, m + 2)
    assert count == 2
    assert {seg[i] for i in range(0, len(seg), 4)} == {0} and {seg[i] for i in range(2, len(seg), 4)} == {1}
    c.instructions.insert(0, C.Barrier((0, 1)))
    seg, pos, count = describe_paged(n, c.instructions, m, m + 2)
    assert seg[0] == -1 and pos[0] == -1 and count == 2


def test_paged_segments_errors():
    from aleph_b200 import backend as B
    from aleph_b200.backend import describe_paged

    c = C.Circuit(10).add(C.Toffoli(), [7, 8, 9])
    with pytest.raises(B.TooManyQubits):
        describe_paged(10, c.instructions, 4, 6)
    with pytest.raises(B.InvalidArgument):
        describe_paged(10, c.instructions, 10, 12)
    with pytest.raises(B.InvalidArgument):
        describe_paged(10, c.instructions, 4, 3)


def test_pair_fusion_keeps_every_gate_and_never_adds_arithmetic():
    """Pair fusion (planner.cpp fuse_pairs), host only: every gate lands in
    exactly one pass, and the plan's real multiply-adds per amplitude never
    grow (a block is fused only when its gates cost at least 24 per amplitude,
    against 16 for the 4x4)."""
    from aleph_b200.backend import describe_plan
    from tests.circuit_gen import random_circuit

    circuits = [(n, random_circuit(n, 300, seed=s)) for n, s in ((14, 1), (17, 2), (20, 3))]
    circuits += [(n, workloads.brickwall(n, 12, seed=n)) for n in (14, 22, 31)]
    circuits += [(24, workloads.qft_product(24, seed=4))]
    for n, c in circuits:
        for prec in ("f64", "f32"):
            for r in (2, 4, 5):
                on = describe_plan(n, c.instructions, prec, tile_r=r, smem_max_n=0)
                off = describe_plan(n, c.instructions, prec, tile_r=r, smem_max_n=0, pair_fusion=False)
                assert sum(p["gates"] for p in on) == sum(p["gates"] for p in off) == c.gate_count()
                assert sum(p["fma_per_amp"] for p in on) <= sum(p["fma_per_amp"] for p in off)
    # the brickwall's even-layer blocks halve its arithmetic
    c = workloads.brickwall(32, 40, seed=0)
    on = describe_plan(32, c.instructions, "f64")
    off = describe_plan(32, c.instructions, "f64", pair_fusion=False)
    assert 2 * sum(p["fma_per_amp"] for p in on) == sum(p["fma_per_amp"] for p in off)
