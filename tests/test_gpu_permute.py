"""Qubit permutations on the GPU: a SWAP gate as an in-place permutation
pass, SWAPs inside gate streams relabelled and settled at the end, and
unpermute_state (crates/aleph-core/src/perm.rs:25-40) as at most two
involution passes. A permutation moves amplitudes without arithmetic, so the
FP64 results must equal the oracle's bit for bit; streams that mix
relabelled SWAPs with other gates keep the usual tolerances (1e-12 FP64,
1e-5 FP32)."""
import math

import numpy as np
import pytest

from aleph_b200 import circuit as C
from aleph_b200 import workloads
from aleph_b200.backend import B200SvBackend, run_with_outcomes
from oracle import oracle

pytestmark = pytest.mark.gpu

F64_TOL = 1e-12
F32_TOL = 1e-5


def random_state(n, seed):
    rng = np.random.default_rng(seed)
    psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    return psi / np.linalg.norm(psi)


def backend(precision="f64", **tuning):
    be = B200SvBackend(seed=0, precision=precision)
    for k, v in tuning.items():
        be.set_tuning(k, v)
    return be


@pytest.mark.parametrize("n,smem", [(8, 0), (11, 0), (14, 12), (17, 12)])
def test_swap_gate_every_pair_f64(n, smem):
    psi = random_state(n, n)
    be = backend(smem_max_n=smem)
    st = be.allocate(n)
    pairs = [(a, b) for a in range(n) for b in range(a + 1, n)]
    if n > 14:
        pairs = [p for p in pairs if p[0] < 6 or p[1] >= n - 3 or (p[0] + p[1]) % 5 == 0]
    for a, b in pairs:
        be.set_statevector(st, psi)
        be.reset_stats()
        be.apply_gate(st, C.GateInstance(C.Gate("Swap"), [a, b]))
        want, _ = oracle.run(n, [C.GateInstance(C.Gate("Swap"), [b, a])], state=psi)
        got = be.statevector(st)
        assert np.array_equal(got, want), (a, b)
        assert be.stats()["tile_passes"] == 0  # no matrix math
    st.free()
    be.close()


def test_swap_gate_f32_and_controlled_swap():
    n = 15
    psi = random_state(n, 1)
    be = backend("f32")
    st = be.allocate(n)
    for a, b in [(0, 14), (2, 3), (4, 9), (10, 13)]:
        be.set_statevector(st, psi)
        be.apply_gate(st, C.GateInstance(C.Gate("Swap"), [a, b]))
        want, _ = oracle.run(n, [C.GateInstance(C.Gate("Swap"), [a, b])], state=psi)
        assert np.abs(be.statevector(st) - want).max() <= F32_TOL
    # a controlled SWAP keeps the gate path
    be.set_statevector(st, psi)
    g = C.GateInstance(C.Gate("Swap"), [1, 12], [7])
    be.apply_gate(st, g)
    want, _ = oracle.run(n, [g], state=psi)
    assert np.abs(be.statevector(st) - want).max() <= F32_TOL
    st.free()
    be.close()


def swap_heavy_circuit(n, depth, seed, measures=True, phase=True):
    """SWAP networks interleaved with dense gates, controlled SWAPs, a
    DiagonalPhase record and mid-circuit measurements."""
    rng = np.random.default_rng(seed)
    c = C.Circuit(n)
    for layer in range(depth):
        for _ in range(3):
            a, b = (int(x) for x in rng.choice(n, 2, replace=False))
            c.add(C.Gate("Swap"), [a, b])
        qs = [int(x) for x in rng.permutation(n)[:4]]
        c.add(C.Unitary1q(workloads.haar_su2(rng)), [qs[0]])
        c.add(C.Gate("Cnot"), qs[1:3])
        c.add(C.Gate("CRz", (float(rng.uniform(-3, 3)),)), [qs[3], qs[0]])
        if layer % 3 == 1:
            c.add(C.Gate("Swap"), qs[:2], [qs[2]])
        if measures and layer == depth // 2:
            c.measure(qs[0], 0)
        if phase and layer == depth // 3:
            terms = [C.PhaseTerm((int(rng.integers(1, 1 << n)),), float(rng.uniform(-2, 2))) for _ in range(4)]
            c.instructions.append(C.DiagonalPhase(n, terms))
    # end on a bit reversal so the settled map is not an involution of the swaps alone
    for q in range(n // 2):
        c.add(C.Gate("Swap"), [q, n - 1 - q])
    return c


@pytest.mark.parametrize("n", [13, 17, 21])
def test_relabelled_stream_f64(n):
    c = swap_heavy_circuit(n, 12, seed=n)
    us = [0.37]
    want, outs = oracle.run(n, c.instructions, uniforms=us)
    for relabel in (1, 0):
        be = backend(relabel_swaps=relabel)
        st, rec = run_with_outcomes(be, c, us)
        assert [int(r.outcome) for r in rec] == outs
        assert np.abs(be.statevector(st) - want).max() <= F64_TOL
        st.free()
        be.close()


@pytest.mark.parametrize("precision", ["f32", "tc32"])
def test_relabelled_stream_f32_tc32(precision):
    n = 18
    c = swap_heavy_circuit(n, 10, seed=3, measures=False)
    want, _ = oracle.run(n, c.instructions)
    be = backend(precision)
    st, _ = run_with_outcomes(be, c)
    assert np.abs(be.statevector(st) - want).max() <= F32_TOL
    be.close()


def test_qft_bit_reversal_is_one_permutation_pass():
    n = 20
    c = workloads.qft_product(n, seed=5)
    want, _ = oracle.run(n, c.instructions)
    passes = {}
    for relabel in (1, 0):
        be = backend(relabel_swaps=relabel, record_passes=1)
        st, _ = run_with_outcomes(be, c)
        assert np.abs(be.statevector(st) - want).max() <= F64_TOL
        kinds = [r["kind"] for r in be.pass_records()]
        passes[relabel] = kinds
        be.close()
    assert passes[1].count("permute") == 1 and "permute" not in passes[0]
    assert len(passes[1]) < len(passes[0])


def test_compiled_plan_with_swaps():
    n = 16
    c = swap_heavy_circuit(n, 8, seed=9, measures=False)
    want, _ = oracle.run(n, c.instructions)
    be = backend()
    plan = be.compile(n, c.instructions)
    st = be.allocate(n)
    for _ in range(2):
        be.reset_state(st)
        plan.execute(st)
        assert np.abs(be.statevector(st) - want).max() <= F64_TOL
    plan.free()
    be.close()


def cycle_perm(n, length, rng):
    perm = list(range(n))
    cyc = [int(x) for x in rng.permutation(n)[:length]]
    for i, q in enumerate(cyc):
        perm[q] = cyc[(i + 1) % length]
    return perm


@pytest.mark.parametrize("n", [3, 6, 11, 15, 20])
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_unpermute_in_place(n, precision):
    rng = np.random.default_rng(n)
    psi = random_state(n, n + 100)
    perms = [list(range(n)), [int(x) for x in rng.permutation(n)], cycle_perm(n, n, rng),
             cycle_perm(n, min(3, n), rng), list(reversed(range(n)))]
    be = backend(precision)
    st = be.allocate(n)
    for perm in perms:
        be.set_statevector(st, psi)
        be.unpermute_state(st, perm)
        got = be.statevector(st)
        want = oracle.unpermute(psi, perm)
        if precision == "f64":
            assert np.array_equal(got, want), perm
        else:
            assert np.abs(got - want).max() <= F32_TOL, perm
    st.free()
    be.close()


def test_swap_pass_traffic_and_norm():
    """A SWAP of two outer qubits leaves half the tiles untouched; the state
    norm is preserved exactly."""
    n = 22
    psi = random_state(n, 7)
    be = backend()
    st = be.allocate(n)
    be.set_statevector(st, psi)
    be.apply_gate(st, C.GateInstance(C.Gate("Swap"), [15, 21]))
    got = be.statevector(st)
    want, _ = oracle.run(n, [C.GateInstance(C.Gate("Swap"), [15, 21])], state=psi)
    assert np.array_equal(got, want)
    assert math.isclose(be.norm_sqr(st), float(np.vdot(psi, psi).real), rel_tol=0, abs_tol=1e-12)
    st.free()
    be.close()
