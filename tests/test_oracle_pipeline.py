"""The restated default CPU path (oracle/sv_pipeline.cpp: final_state_cpu_pipeline
+ the CPU sv kernels), which bench.py times as the CPU baseline.

It is held to the raw gate-by-gate oracle at 1e-12, the reference's own
guarantee for the optimised path (crates/aleph-backend/tests/run_optimized_oracle.rs:18),
and to the reference's golden fixtures at 1e-10. The pass-count cases restate
the reference's pipeline and FuseKq unit tests
(crates/aleph-ir/src/passes/mod.rs:229-300, fuse_kq.rs:622-794) at the
pipeline level.
"""
import math

import numpy as np
import pytest

from aleph_b200 import circuit as C
from aleph_b200 import workloads
from oracle import oracle
from tests.circuit_gen import random_circuit
from tests.fixtures_util import fixture_instructions, fixture_state, load_reference_fixtures

TOL = 1e-12


def swap2q():
    m = np.zeros((4, 4), dtype=np.complex128)
    m[0, 0] = m[1, 2] = m[2, 1] = m[3, 3] = 1.0
    return C.Unitary2q(m)


def counts(n, insts, **kw):
    return oracle.describe_pipeline(n, insts, **kw)


def test_fuse_2q_absorbs_a_1q_neighbour():
    # Rx(0.5) q0; CNOT(0,1) -> one Unitary2q (mod.rs: default_pipeline_includes_fuse_2q)
    c = C.Circuit(2).add(C.Rx(0.5), [0]).add(C.Cnot(), [0, 1])
    k = counts(2, c.instructions)
    assert k["input"] == 2 and k["after_fuse2q"] == 1 and k["output"] == 1


def test_inverse_pair_cancels_before_fusion():
    # H(0); H(0); H(1) -> H(1) (mod.rs: default_pipeline_cancels_inverse_pair_before_fusion)
    c = C.Circuit(2).add(C.H(), [0]).add(C.H(), [0]).add(C.H(), [1])
    k = counts(2, c.instructions)
    assert k["after_cancel"] == 1 and k["output"] == 1


def test_inverse_pairs_of_parametric_and_matrix_gates():
    u = workloads.haar_su2(np.random.default_rng(3))
    c = C.Circuit(3)
    c.add(C.Rz(0.7), [1]).add(C.Rz(-0.7), [1])
    c.add(C.S(), [0]).add(C.Sdg(), [0])
    c.add(C.U3(0.1, 0.2, 0.3), [2]).add(C.U3(-0.1, -0.3, -0.2), [2])
    c.add(C.Unitary1q(u), [2]).add(C.Unitary1q(u.conj().T), [2])
    c.add(C.Cnot(), [0, 1]).add(C.Cnot(), [0, 1])
    c.add(C.Cnot(), [0, 1]).add(C.Cnot(), [1, 0])  # different targets: kept
    assert counts(3, c.instructions)["after_cancel"] == 2


def test_two_chained_2q_blocks_fuse_into_one_3q():
    c = C.Circuit(3).add(swap2q(), [0, 1]).add(swap2q(), [1, 2])
    k = counts(3, c.instructions)
    assert k["fused_kq"] == 1 and k["output"] == 1


def test_lone_2q_block_and_lone_toffoli_are_not_fused():
    assert counts(2, C.Circuit(2).add(swap2q(), [0, 1]).instructions)["fused_kq"] == 0
    assert counts(3, C.Circuit(3).add(C.Toffoli(), [0, 1, 2]).instructions)["fused_kq"] == 0


def test_barrier_is_a_fence():
    c = C.Circuit(3).add(swap2q(), [0, 1])
    c.instructions.append(C.Barrier((0, 1, 2)))
    c.add(swap2q(), [1, 2])
    assert counts(3, c.instructions)["fused_kq"] == 0


def test_independent_blocks_fuse_separately_under_max_3():
    c = C.Circuit(6).add(swap2q(), [0, 1]).add(swap2q(), [3, 4]).add(swap2q(), [1, 2]).add(swap2q(), [4, 5])
    assert counts(6, c.instructions, max_k=3)["fused_kq"] == 2


def test_non_finite_gate_is_a_fence():
    c = C.Circuit(3).add(swap2q(), [0, 1]).add(C.Rz(float("nan")), [1]).add(swap2q(), [1, 2])
    assert counts(3, c.instructions)["fused_kq"] == 0


def test_relabel_moves_high_traffic_qubits_low():
    # relabel.rs: high_qubit_circuit_relabels_to_low_bits (tile_bits 2)
    c = C.Circuit(6).add(C.H(), [4]).add(C.H(), [5]).add(C.Cnot(), [4, 5]).add(C.H(), [4]).add(C.Cnot(), [5, 4])
    assert counts(6, c.instructions, tile_bits=2)["relabeled"] == 1
    assert counts(6, c.instructions)["relabeled"] == 0  # all targets already below 15


def test_brickwall_plan_shape():
    # depth-40 brickwall: 1q runs fold into the CZ neighbours, 4-qubit blocks
    k = counts(24, workloads.brickwall(24, 40, seed=0).instructions)
    assert k["input"] == 1420 and k["relabeled"] == 0
    assert k["after_fuse2q"] < k["after_fuse1q"] < k["input"]
    assert k["fused_kq"] > 100 and k["output"] < 300


@pytest.mark.parametrize("n,depth,seed", [(5, 60, 1), (8, 120, 2), (11, 150, 3), (14, 150, 4)])
def test_random_all_gates_match_raw(n, depth, seed):
    c = random_circuit(n, depth, seed)
    raw, _ = oracle.run(n, c.instructions)
    got, _ = oracle.run_pipeline(n, c.instructions)
    assert np.abs(got - raw).max() <= TOL


@pytest.mark.parametrize("tile_bits", [3, 6, 9])
def test_tiled_blocks_with_high_controls_match_raw(tile_bits):
    # small tiles: every TiledBlock runs tile by tile, and controls at or
    # above tile_bits skip the tiles where they are 0 (backend.rs:231-253)
    n = 12
    rng = np.random.default_rng(tile_bits)
    c = C.Circuit(n)
    for _ in range(200):
        q = [int(x) for x in rng.permutation(n)]
        lo = [x for x in q if x < tile_bits]
        if len(lo) >= 2 and rng.random() < 0.4:
            c.add(C.Unitary2q(np.linalg.qr(rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4)))[0]),
                  lo[:2], [x for x in q if x >= tile_bits][:1])
        else:
            c.add(C.Unitary1q(workloads.haar_su2(rng)), [q[0]], [q[1]] if rng.random() < 0.5 else [])
    k = counts(n, c.instructions, tile_bits=tile_bits)
    assert k["tiled_blocks"] > 0
    raw, _ = oracle.run(n, c.instructions)
    got, _ = oracle.run_pipeline(n, c.instructions, tile_bits=tile_bits)
    assert np.abs(got - raw).max() <= TOL


def test_relabelled_run_is_unpermuted():
    n = 10
    rng = np.random.default_rng(9)
    c = C.Circuit(n)
    for _ in range(120):  # traffic on the high qubits, tiles of 4 qubits
        a, b = (int(x) for x in rng.choice([6, 7, 8, 9], 2, replace=False))
        c.add(C.Unitary1q(workloads.haar_su2(rng)), [a]).add(C.Cz(), [a, b])
    c.add(C.H(), [0])
    assert counts(n, c.instructions, tile_bits=4)["relabeled"] == 1
    raw, _ = oracle.run(n, c.instructions)
    got, _ = oracle.run_pipeline(n, c.instructions, tile_bits=4)
    assert np.abs(got - raw).max() <= TOL


@pytest.mark.parametrize("name", ["brickwall", "qft", "qaoa", "grover"])
def test_workloads_match_raw(name):
    if name == "brickwall":
        n, c = 16, workloads.brickwall(16, 20, seed=11)
    elif name == "qft":
        n, c = 14, workloads.qft_product(14, seed=2)
    elif name == "qaoa":
        rng = np.random.default_rng(5)
        n = 12
        c = workloads.qaoa_maxcut(n, workloads.random_3_regular(n, rng), [0.4, 1.1], [0.8, 0.3])
    else:
        c = workloads.grover(6, 37, 3)
        n = c.num_qubits
    raw, _ = oracle.run(n, c.instructions)
    got, _ = oracle.run_pipeline(n, c.instructions)
    assert np.abs(got - raw).max() <= TOL


FIXTURES = load_reference_fixtures()


@pytest.mark.parametrize("fx", FIXTURES, ids=[f["name"] for f in FIXTURES])
def test_reference_fixtures(fx):
    n = fx["num_qubits"]
    got, _ = oracle.run_pipeline(n, fixture_instructions(fx), uniforms=fx["measure_uniforms"])
    assert np.abs(got - fixture_state(fx)).max() <= 1e-10


def test_sliced_execution_equals_whole():
    n = 14
    c = workloads.brickwall(n, 16, seed=4)
    whole, _ = oracle.run_pipeline(n, c.instructions)
    P = oracle.PlannedCircuit(n, c.instructions)
    psi = oracle.zero_state(n)
    L = len(P)
    cuts = [0, L // 4, L // 2, L]
    for a, b in zip(cuts, cuts[1:]):
        assert P.execute(psi, a, b, finish=b == L) >= 0.0
    P.free()
    assert np.abs(psi - whole).max() == 0.0
    assert math.isclose(float(np.vdot(psi, psi).real), 1.0, abs_tol=1e-12)


# ---- the reference's CUDA pass list (fuse_full_state), executed on the CPU kernels ----------
def gpu_plan_state(n, insts):
    plan = oracle.PlannedCircuit(n, insts, max_k=3, gpu=True)
    psi = oracle.zero_state(n)
    plan.execute(psi)
    return psi, plan.counts()


@pytest.mark.parametrize("make", [
    lambda: (10, workloads.brickwall(10, 8, seed=4).instructions),
    lambda: (9, workloads.qft_product(9, seed=2).instructions),
    lambda: (8, workloads.grover(3, 5, 2).instructions),
    lambda: (9, random_circuit(9, 160, seed=11).instructions),
    lambda: (7, random_circuit(7, 300, seed=12).instructions),
])
def test_gpu_pass_list_matches_the_raw_oracle(make):
    n, insts = make()
    want, _ = oracle.run(n, insts)
    got, _ = gpu_plan_state(n, insts)
    assert np.abs(got - want).max() <= TOL


def test_fuse_diagonal_runs_one_phase_per_cz_layer():
    # every CZ layer of the brickwall is a run of diagonal gates between two
    # Haar layers: one DiagonalPhase each (fuse_diagonal.rs:23-68)
    n, depth = 12, 10
    _, k = gpu_plan_state(n, workloads.brickwall(n, depth, seed=1).instructions)
    assert k["tiled_blocks"] == depth
    assert k["fused_kq"] == 0  # disjoint one-qubit gates never share a FuseKq block


def test_fuse_diagonal_runs_absorbs_cnot_conjugation():
    # CNOT(0,1) Rz(0.3) on 1 CNOT(0,1): net permutation identity, two diagonal
    # members -> one DiagonalPhase over parity(b0 ^ b1); a lone Rz is left alone
    c = C.Circuit(3).add(C.Cnot(), [0, 1]).add(C.Rz(0.3), [1]).add(C.Cnot(), [0, 1]).add(C.Cz(), [1, 2])
    got, k = gpu_plan_state(3, c.instructions)
    assert k["tiled_blocks"] == 1 and k["output"] == 1
    want, _ = oracle.run(3, c.instructions)
    assert np.abs(got - want).max() <= TOL
    lone = C.Circuit(2).add(C.Rz(0.3), [1])
    assert gpu_plan_state(2, lone.instructions)[1]["tiled_blocks"] == 0
    # a run whose CNOTs do not cancel is emitted as it is
    odd = C.Circuit(2).add(C.Cnot(), [0, 1]).add(C.Rz(0.3), [1]).add(C.Cz(), [0, 1])
    got, k = gpu_plan_state(2, odd.instructions)
    assert k["tiled_blocks"] == 0
    assert np.abs(got - oracle.run(2, odd.instructions)[0]).max() <= TOL


def test_gpu_pass_list_on_the_golden_fixtures():
    for fx in load_reference_fixtures():
        name = fx["name"]
        insts = fixture_instructions(fx)
        if any(isinstance(i, C.Measure) for i in insts):
            continue
        n = fx["num_qubits"]
        got, _ = gpu_plan_state(n, insts)
        assert np.abs(got - fixture_state(fx)).max() <= 1e-10, name
