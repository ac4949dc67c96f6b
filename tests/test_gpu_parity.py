"""GPU parity of the engine against the CPU oracle, through the C ABI.

Tolerances: the plain FP64 path must match the FP64 oracle to
max |dpsi| <= 1e-12; FP32 to 1e-5 (the reference's FP32 oracle tolerance,
crates/aleph-oracle/src/harness.rs:27); golden fixtures at 1e-10
(harness.rs:18). Sampling: given the same variates, bitstrings identical.
"""
import math

import numpy as np
import pytest

from aleph_b200 import circuit as C
from aleph_b200 import workloads
from aleph_b200.backend import B200SvBackend, describe_plan, run, run_with_outcomes
from oracle import oracle
from tests.circuit_gen import random_circuit
from tests.fixtures_util import fixture_instructions, fixture_state, load_reference_fixtures

pytestmark = pytest.mark.gpu

F64_TOL = 1e-12
F32_TOL = 1e-5
FIXTURES = load_reference_fixtures()


def engine_state(circ, precision="f64", uniforms=None, **tuning):
    be = B200SvBackend(seed=0, precision=precision)
    for k, v in tuning.items():
        be.set_tuning(k, v)
    st, rec = run_with_outcomes(be, circ, uniforms)
    return be.statevector(st), rec, be, st


@pytest.mark.parametrize("fx", FIXTURES, ids=[f["name"] for f in FIXTURES])
def test_reference_fixtures(fx):
    c = C.Circuit(fx["num_qubits"], fixture_instructions(fx))
    got, _, _, _ = engine_state(c, uniforms=fx["measure_uniforms"])
    want = fixture_state(fx)
    assert np.abs(got - want).max() <= 1e-10
    ref, _ = oracle.run(fx["num_qubits"], c.instructions, uniforms=fx["measure_uniforms"])
    assert np.abs(got - ref).max() <= F64_TOL


@pytest.mark.parametrize("n,smem", [(6, 12), (9, 12), (12, 12), (7, 0), (11, 0), (13, 12), (16, 12), (18, 12)])
@pytest.mark.parametrize("tile_r", [1, 3, 4, 5])
def test_random_all_gates_f64(n, smem, tile_r):
    if n - 5 < 1:
        pytest.skip("tile path needs n >= 6")
    c = random_circuit(n, 120, seed=n * 31 + tile_r)
    got, _, be, _ = engine_state(c, tile_r=tile_r, smem_max_n=smem)
    want, _ = oracle.run(n, c.instructions)
    assert np.abs(got - want).max() <= F64_TOL


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("k", [3, 4, 5])
def test_dense_kq_pass(k, precision):
    """UnitaryKq (k = 3..5) runs as its own dense k-qubit pass: scattered
    targets in any order (lowest qubit in and out of the set), against the
    oracle. (The reference rejects controls on UnitaryKq.)"""
    n = 15
    rng = np.random.default_rng(60 + k)
    c = workloads.brickwall(n, 2, seed=61)
    for first in (0, 9):
        qs = [first] + [int(q) for q in rng.permutation([q for q in range(n) if q != first])[: k - 1]]
        z = rng.standard_normal((2**k, 2**k)) + 1j * rng.standard_normal((2**k, 2**k))
        c.add(C.UnitaryKq(np.linalg.qr(z)[0]), qs)
    got, _, be, _ = engine_state(c, precision=precision)
    want, _ = oracle.run(n, c.instructions)
    assert np.abs(got - want).max() <= (F64_TOL if precision == "f64" else F32_TOL)


@pytest.mark.parametrize("n", [8, 14, 20])
def test_brickwall_f64(n):
    c = workloads.brickwall(n, 20, seed=1)
    got, _, be, _ = engine_state(c)
    want, _ = oracle.run(n, c.instructions)
    assert np.abs(got - want).max() <= F64_TOL


@pytest.mark.parametrize("n", [10, 17])
def test_brickwall_f32(n):
    c = workloads.brickwall(n, 12, seed=2)
    got, _, _, _ = engine_state(c, precision="f32")
    want, _ = oracle.run(n, c.instructions)
    assert np.abs(got - want).max() <= F32_TOL


@pytest.mark.parametrize("n", [9, 16])
def test_qft_and_qaoa_f64(n):
    c = workloads.qft_product(n, seed=3)
    got, _, _, _ = engine_state(c)
    want, _ = oracle.run(n, c.instructions)
    assert np.abs(got - want).max() <= F64_TOL
    rng = np.random.default_rng(4)
    edges = workloads.random_3_regular(n + (n % 2), rng)
    m = n + (n % 2)
    q = workloads.qaoa_maxcut(m, edges, rng.uniform(0, math.pi, 4), rng.uniform(0, math.pi, 4))
    got, _, _, _ = engine_state(q)
    want, _ = oracle.run(m, q.instructions)
    assert np.abs(got - want).max() <= F64_TOL


def test_diagonal_phase_instruction():
    n = 14
    rng = np.random.default_rng(5)
    terms = [C.PhaseTerm(tuple(int(x) for x in rng.integers(1, 1 << n, size=int(rng.integers(0, 3)))),
                         float(rng.uniform(-3, 3))) for _ in range(12)]
    c = workloads.brickwall(n, 3, seed=6)
    c.instructions.append(C.DiagonalPhase(n, terms))
    c.instructions.extend(workloads.brickwall(n, 2, seed=7).instructions)
    for smem in (0, 12):
        got, _, _, _ = engine_state(c, smem_max_n=smem)
        want, _ = oracle.run(n, c.instructions)
        assert np.abs(got - want).max() <= F64_TOL


@pytest.mark.parametrize("n", [6, 14])
def test_mid_circuit_measurement(n):
    c = workloads.brickwall(n, 4, seed=8)
    for q in (0, n - 1, n // 2):
        c.measure(q, q)
    c.instructions.extend(workloads.brickwall(n, 3, seed=9).instructions)
    c.measure(1, 1)
    us = [0.3, 0.8, 0.5, 0.1]
    got, rec, _, _ = engine_state(c, uniforms=us)
    want, outs = oracle.run(n, c.instructions, uniforms=us)
    assert [int(r.outcome) for r in rec] == outs
    assert np.abs(got - want).max() <= F64_TOL


@pytest.mark.parametrize("n", [1, 5, 12, 18, 22])
def test_sampling_alias_identical(n):
    c = workloads.brickwall(n, 6, seed=10) if n > 1 else C.Circuit(1).add(C.Ry(1.1), [0])
    be = B200SvBackend(seed=0)
    st = run(be, c)
    psi = be.statevector(st)
    words = workloads.splitmix64_words(n, 1024)
    shots = be.sample(st, 1024, variates=words, mode="alias")
    assert np.array_equal(shots, oracle.sample_alias(psi, words))


@pytest.mark.parametrize("n", [1, 6, 12, 16, 22, 24])
def test_sampling_cumulative_identical(n):
    c = workloads.brickwall(n, 6, seed=11) if n > 1 else C.Circuit(1).add(C.Ry(0.7), [0])
    be = B200SvBackend(seed=0)
    st = run(be, c)
    psi = be.statevector(st)
    u = np.random.default_rng(n).random(2048)
    u[:4] = [0.0, 0.5, 1.0 - 2**-53, 0.25]
    shots = be.sample(st, u.size, variates=u, mode="cumulative")
    assert np.array_equal(shots, oracle.sample_cumulative(psi, u))


def test_exact_inverse_boundaries():
    # exact-probability boundary KAT (see test_cpu_host.test_oracle_exact_inverse_boundaries)
    psi = np.zeros(512, dtype=np.complex128)
    psi[[1, 255, 256, 511]] = 0.5
    be = B200SvBackend(seed=0)
    st = be.allocate(9)
    be.set_statevector(st, psi)
    u = [0.0, np.nextafter(0.25, 0), 0.25, np.nextafter(0.5, 0), 0.5, 0.75, np.nextafter(1.0, 0)]
    assert list(be.sample(st, len(u), variates=u, mode="cumulative")) == [1, 1, 255, 255, 256, 511, 511]
    # irrational amplitudes: identical to the oracle whatever the rounding
    psi2 = np.zeros(512, dtype=np.complex128)
    for i, p in [(1, 0.125), (255, 0.125), (256, 0.25), (511, 0.5)]:
        psi2[i] = math.sqrt(p)
    be.set_statevector(st, psi2)
    u2 = [0.0, 0.125, np.nextafter(0.25, 0), 0.25, 0.5, np.nextafter(1.0, 0)]
    assert list(be.sample(st, 6, variates=u2, mode="cumulative")) == list(oracle.sample_cumulative(psi2, u2))


def test_alias_table_uniform_and_forced():
    # uniform superposition: every scaled probability is exactly 1 -> all self-aliased
    be = B200SvBackend(seed=0)
    n = 10
    c = C.Circuit(n)
    for q in range(n):
        c.add(C.H(), [q])
    st = run(be, c)
    psi = be.statevector(st)
    words = workloads.splitmix64_words(99, 4096)
    assert np.array_equal(be.sample(st, 4096, variates=words, mode="alias"), oracle.sample_alias(psi, words))
    # forced basis state
    st2 = run(be, C.Circuit(3).add(C.X(), [1]))
    assert set(be.sample(st2, 64, variates=words[:64], mode="alias").tolist()) == {2}


@pytest.mark.parametrize("n", [4, 13])
def test_expectation_and_probabilities(n):
    c = workloads.brickwall(n, 5, seed=12)
    be = B200SvBackend(seed=0)
    st = run(be, c)
    psi = be.statevector(st)
    rng = np.random.default_rng(13)
    for _ in range(12):
        k = int(rng.integers(0, min(n, 5) + 1))
        qs = [int(x) for x in rng.permutation(n)[:k]]
        ps = [str(x) for x in rng.choice(list("IXYZ"), size=k)]
        terms = list(zip(qs, ps))
        coef = float(rng.uniform(-2, 2))
        assert abs(be.expectation_value(st, terms, coef) - oracle.expectation(psi, terms, coef)) <= 1e-12
        sub = [int(x) for x in rng.permutation(n)[: int(rng.integers(0, n + 1))]]
        assert np.abs(be.probabilities(st, sub) - oracle.probabilities(psi, sub)).max() <= 1e-12


def random_pauli_sum(n, count, rng, flip_pool=3):
    """Terms drawn so that several share their X/Y positions (more than 16
    on the diagonal group), with identity and Y-carrying terms among them."""
    flips = [[]] + [[int(q) for q in rng.permutation(n)[: int(rng.integers(1, 4))]] for _ in range(flip_pool)]
    terms = []
    for k in range(count):
        xq = flips[int(rng.integers(0, len(flips)))] if k % 3 else []
        rest = [int(q) for q in rng.permutation(n) if q not in xq][: int(rng.integers(0, 4))]
        string = [(q, str(rng.choice(["X", "Y"]))) for q in xq] + [(q, str(rng.choice(["Z", "I"]))) for q in rest]
        order = rng.permutation(len(string))
        terms.append((float(rng.uniform(-2, 2)), [string[i] for i in order]))
    return terms


@pytest.mark.parametrize("n,precision", [(13, "f64"), (16, "f32")])
def test_expectation_sum_matches_term_by_term(n, precision):
    """aleph_b200_expectation_sum against the reference's loop over
    expectation_value: each term's value agrees with the single-term result
    to rounding (same reduction order; the compiler may contract the
    per-amplitude products differently), the sum is taken in term order, and
    it matches the oracle's."""
    c = workloads.brickwall(n, 5, seed=40)
    be = B200SvBackend(seed=0, precision=precision)
    st = run(be, c)
    psi = be.statevector(st)
    rng = np.random.default_rng(41)
    terms = random_pauli_sum(n, 45, rng)
    total, vals = be.expectation_sum(st, terms, with_terms=True)
    single = np.array([be.expectation_value(st, s, coef) for coef, s in terms])
    assert np.abs(vals - single).max() <= 1e-13
    assert total == sum(vals)  # summed in term order, as the reference does
    ref = psi / np.linalg.norm(psi)  # the oracle holds a widened FP32 state to the FP64 norm tolerance
    want = sum(oracle.expectation(ref, s, coef) for coef, s in terms)
    assert abs(total - want) <= (1e-11 if precision == "f64" else 1e-5 * len(terms))
    # Max-Cut: |E|/2 - 1/2 sum <Z_i Z_j>
    edges = [(i, (i + 1) % n) for i in range(n)] + [(i, (i + 5) % n) for i in range(0, n, 2)]
    h = workloads.maxcut_pauli_sum(n, edges)
    assert be.expectation_sum(st, h) == pytest.approx(sum(be.expectation_value(st, s, coef) for coef, s in h),
                                                      abs=1e-12)
    be.close()


def test_expectation_sum_errors():
    """Errors in the reference loop's order: nothing for no terms; the state
    first; then per term in order its coefficient, qubit range, duplicates."""
    from aleph_b200 import backend as B

    be = B200SvBackend(seed=0)
    st = be.allocate(4)
    assert be.expectation_sum(st, []) == 0.0
    assert be.expectation_sum(st, [(0.75, [])]) == 0.75
    with pytest.raises(B.DuplicateQubit):
        be.expectation_sum(st, [(1.0, [(0, "Z")]), (1.0, [(1, "X"), (1, "Z")]), (1.0, [(9, "Z")])])
    with pytest.raises(B.QubitOutOfRange):
        be.expectation_sum(st, [(1.0, [(0, "Z")]), (1.0, [(9, "Z")]), (1.0, [(1, "X"), (1, "Z")])])
    with pytest.raises(B.InvalidPauliString):
        be.expectation_sum(st, [(1.0, [(0, "Z")]), (float("nan"), [(9, "Z")])])
    bad = np.zeros(16, dtype=np.complex128)
    bad[3] = 2.0
    be.set_statevector(st, bad)
    assert be.expectation_sum(st, []) == 0.0
    with pytest.raises(B.InvalidState):
        be.expectation_sum(st, [(float("nan"), [(9, "Z")])])
    be.close()


def test_norm_and_unpermute():
    n = 13
    c = workloads.brickwall(n, 4, seed=14)
    be = B200SvBackend(seed=0)
    st = run(be, c)
    psi = be.statevector(st)
    assert abs(be.norm_sqr(st) - 1.0) <= 1e-12
    perm = [int(x) for x in np.random.default_rng(15).permutation(n)]
    be.unpermute_state(st, perm)
    assert np.abs(be.statevector(st) - oracle.unpermute(psi, perm)).max() == 0.0


def test_error_variants():
    from aleph_b200 import backend as B

    be = B200SvBackend(seed=0)
    st = be.allocate(3)
    with pytest.raises(B.QubitOutOfRange):
        be.apply_gate(st, C.GateInstance(C.H(), [3]))
    with pytest.raises(B.DuplicateQubit):
        be.apply_gate(st, C.GateInstance(C.Cnot(), [1, 1]))
    with pytest.raises(B.DuplicateQubit):
        be.apply_gate(st, C.GateInstance(C.X(), [1], [1]))
    with pytest.raises(B.ArityMismatch):
        be.apply_gate(st, C.GateInstance(C.Cnot(), [0]))
    with pytest.raises(B.NonFiniteParam):
        be.apply_gate(st, C.GateInstance(C.Rx(float("nan")), [0]))
    with pytest.raises(B.NonUnitaryMatrix):
        be.apply_gate(st, C.GateInstance(C.Unitary1q([[2, 0], [0, 2]]), [0]))
    with pytest.raises(B.UnsupportedGate):
        be.apply_gate(st, C.GateInstance(C.UnitaryKq(np.eye(4)), [0, 1], [2]))
    with pytest.raises(B.UnsupportedInstruction):
        be.apply_stream(st, [C.Reset(0)])
    with pytest.raises(B.TooManyQubits):
        be.allocate(40)
    with pytest.raises(B.InvalidPauliString):
        be.expectation_value(st, [(0, "Z")], float("inf"))
    # a failing stream leaves the state untouched (validation precedes any launch)
    before = be.statevector(st)
    with pytest.raises(B.QubitOutOfRange):
        be.apply_stream(st, [C.GateInstance(C.H(), [0]), C.GateInstance(C.H(), [7])])
    assert np.array_equal(before, be.statevector(st))
    # corrupted state -> InvalidState from every query
    bad = np.zeros(8, dtype=np.complex128)
    bad[0] = np.nan
    be.set_statevector(st, bad)
    for call in (lambda: be.sample(st, 4, variates=[1, 2, 3, 4], mode="alias"),
                 lambda: be.probabilities(st, [0]),
                 lambda: be.expectation_value(st, [(0, "Z")]),
                 lambda: be.measure(st, 0, 0.5)):
        with pytest.raises(B.InvalidState):
            call()
    # degenerate measurement: the zero vector
    be.set_statevector(st, np.zeros(8))
    with pytest.raises((B.DegenerateMeasurement, B.InvalidState)):
        be.measure(st, 0, 0.5)


def test_seeded_determinism():
    c = workloads.brickwall(10, 4, seed=16)
    a = B200SvBackend(seed=42)
    b = B200SvBackend(seed=42)
    sa, sb = run(a, c), run(b, c)
    assert np.array_equal(a.sample(sa, 500), b.sample(sb, 500))
    assert a.measure(sa, 3) == b.measure(sb, 3)


@pytest.mark.parametrize("n,precision", [(22, "f64"), (29, "f32")])
def test_seeded_sampling_beyond_the_alias_range(n, precision):
    """Seeded sampling of many shots works for every n: above n = 20 it runs
    the parallel inverse CDF (alias tables stop at n = 28)."""
    c = C.Circuit(n).add(C.H(), [0])
    for q in range(n - 1):
        c.add(C.Cnot(), [q, q + 1])
    outs = []
    for _ in range(2):
        be = B200SvBackend(seed=5, precision=precision)
        st = run(be, c)
        outs.append(be.sample(st, 1024))
        be.close()
    assert np.array_equal(outs[0], outs[1])
    vals, cnt = np.unique(outs[0], return_counts=True)
    assert set(int(v) for v in vals) == {0, (1 << n) - 1} and min(cnt) > 400


# ---- TC32: fused 6-qubit blocks on tcgen05 tensor cores, split-BF16x3 ---------
TC_TOL = 1e-5  # per-amplitude, the FP32 tolerance; 1 - fidelity checked at 1e-6


def fidelity(a, b):
    return abs(np.vdot(a, b)) ** 2 / (np.vdot(a, a).real * np.vdot(b, b).real)


@pytest.mark.parametrize("n", [13, 14, 18])
def test_tc32_brickwall(n):
    c = workloads.brickwall(n, 16, seed=21)
    got, _, be, _ = engine_state(c, precision="tc32")
    want, _ = oracle.run(n, c.instructions)
    assert be.stats()["block_passes"] > 0
    assert np.abs(got - want).max() <= TC_TOL
    assert 1.0 - fidelity(got, want) <= 1e-6


@pytest.mark.parametrize("n", [13, 16])
def test_tc32_all_gates(n):
    c = random_circuit(n, 150, seed=200 + n)
    got, _, be, _ = engine_state(c, precision="tc32")
    want, _ = oracle.run(n, c.instructions)
    assert np.abs(got - want).max() <= TC_TOL
    assert 1.0 - fidelity(got, want) <= 1e-6


def test_tc32_qft_measure_sample():
    n = 15
    c = workloads.qft_product(n, seed=22)
    c.measure(3, 0)
    c.instructions.extend(workloads.brickwall(n, 3, seed=23).instructions)
    got, rec, be, st = engine_state(c, precision="tc32", uniforms=[0.4])
    want, outs = oracle.run(n, c.instructions, uniforms=[0.4])
    assert [int(r.outcome) for r in rec] == outs
    assert np.abs(got - want).max() <= TC_TOL
    # sampling from the FP32 state reads the same probabilities the oracle gets from it
    psi = be.statevector(st)
    psi = psi / np.linalg.norm(psi)
    be.set_statevector(st, psi)
    words = workloads.splitmix64_words(5, 512)
    assert np.array_equal(be.sample(st, 512, variates=words, mode="alias"),
                          oracle.sample_alias(be.statevector(st), words))


# ---- compiled plans: compile once, execute many ------------------------------
@pytest.mark.parametrize("precision", ["f64", "tc32"])
def test_compiled_plan_matches_stream(precision):
    n = 14
    c = workloads.brickwall(n, 6, seed=31)
    c.measure(2, 0)
    c.instructions.extend(workloads.brickwall(n, 2, seed=32).instructions)
    be = B200SvBackend(seed=0, precision=precision)
    plan = be.compile(n, c.instructions)
    tol = F64_TOL if precision == "f64" else TC_TOL
    for u in (0.3, 0.9, 0.3):
        st = be.allocate(n)
        outs = plan.execute(st, [u])
        want, wouts = oracle.run(n, c.instructions, uniforms=[u])
        assert outs == wouts
        assert np.abs(be.statevector(st) - want).max() <= tol
        st.free()
    st = be.allocate(n - 1)
    with pytest.raises(Exception):
        plan.execute(st, [0.5])
    plan.free()


BLOCK_LAYOUTS = {
    "octets": [0, 1, 2, 3, 4, 5],      # rows 8k..8k+7 adjacent: staged transpose on store
    "pairs": [0, 3, 5, 8, 9, 11],      # rows 2p, 2p+1 adjacent: 16-byte stores
    "plain": [7, 8, 9, 10, 11, 12],    # one 8-byte store per row
}


@pytest.mark.parametrize("post", ["signs", "folded", "general"])
@pytest.mark.parametrize("layout", sorted(BLOCK_LAYOUTS))
def test_tc32_block_epilogue_paths(layout, post):
    """Every store path of the block epilogue against the oracle, with each
    kind of diagonal op after the block: sign flips (CZ), phases folded into
    per-column factors (controlled phases with at most one block qubit,
    one-qubit diagonals on column qubits) and the general route (two-qubit
    diagonals across the block, phase polynomials)."""
    n = 16
    bq = BLOCK_LAYOUTS[layout]
    out = [q for q in range(n) if q not in bq]
    rng = np.random.default_rng(7)
    psi0 = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    psi0 /= np.linalg.norm(psi0)
    c = C.Circuit(n)
    for _ in range(2):
        for q in bq:
            c.add(C.Unitary1q(workloads.haar_su2(rng)), [q])
        for a, b in zip(bq, bq[1:]):
            c.add(C.Cz(), [a, b])
    ph = np.exp(1j * rng.uniform(0, 2 * np.pi, 4))
    if post == "signs":
        c.add(C.Cz(), [bq[1], out[-1]]).add(C.Cz(), [out[0], out[-2]]).add(C.Cz(), [bq[0], bq[4]])
    elif post == "folded":
        c.add(C.Unitary2qDiag([1, 1, 1, ph[0]]), [bq[2], out[-1]])
        c.add(C.Unitary2qDiag([1, 1, 1, ph[1]]), [out[1], out[-3]])
        c.add(C.Phase(0.37), [out[-2]]).add(C.Rz(0.91), [out[2]])
    else:
        c.add(C.Unitary2qDiag(ph), [bq[0], out[-1]])
        c.add(C.Rz(0.7), [bq[3]], controls=[out[-2]])
        c.instructions.append(C.DiagonalPhase(n, [C.PhaseTerm((1 << bq[1] | 1 << out[0],), 0.43),
                                                  C.PhaseTerm((1 << bq[5], 1 << out[3]), -1.1)]))
        c.add(C.Cz(), [bq[2], out[-3]])
    plan = describe_plan(n, c.instructions, precision="tc32")
    assert plan[0]["kind"] == "block" and plan[0]["qubits"] == bq and plan[0]["post_ops"] > 0
    be = B200SvBackend(seed=0, precision="tc32")
    st = be.allocate(n)
    be.set_statevector(st, psi0)
    be.apply_stream(st, c.instructions)
    got = be.statevector(st)
    want, _ = oracle.run(n, c.instructions, state=psi0)
    assert be.stats()["block_passes"] > 0
    assert np.abs(got - want).max() <= TC_TOL
    assert 1.0 - fidelity(got, want) <= 1e-6
    be.close()


@pytest.mark.parametrize("window_search", [0, 1])
def test_tc32_block_planners(window_search):
    n = 17
    c = workloads.brickwall(n, 12, seed=51)
    got, _, be, _ = engine_state(c, precision="tc32", block_window_search=window_search)
    want, _ = oracle.run(n, c.instructions)
    assert np.abs(got - want).max() <= TC_TOL
    assert 1.0 - fidelity(got, want) <= 1e-6
