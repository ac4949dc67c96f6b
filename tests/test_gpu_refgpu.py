"""The GPU reference arm (oracle/ref_gpu.cpp): the reference's own CUDA kernels,
compiled unchanged from its sources into oracle/_ref/, launched in the order of
its run_layered / apply_gate dispatch on a stream planned by its CUDA pass list
(fuse_full_state, crates/aleph-cuda/src/fusion.rs:137-152).

bench.py times this arm beside the engine on the same device. These tests hold
it to the oracle at the reference's own tolerances (1e-10 for FP64,
crates/aleph-oracle/src/harness.rs:18; 1e-5 for FP32), so that the timed runs
are runs of a correct reference path. The circuits reach every reference
kernel: layered one-qubit batches, CNOT permutations, phase polynomials, dense
k-qubit blocks (generic and warp-tiled), controlled one-qubit gates and the
diagonal kernels.
"""
import numpy as np
import pytest

from aleph_b200 import workloads
from oracle import oracle
from tests.circuit_gen import random_circuit

pytestmark = pytest.mark.gpu

CIRCUITS = {
    "brickwall": lambda: (12, workloads.brickwall(12, 10, seed=3).instructions),
    "qft": lambda: (11, workloads.qft_product(11, seed=5).instructions),
    "grover": lambda: (9, workloads.grover(4, 9, 2).instructions),
    "random": lambda: (9, random_circuit(9, 240, seed=21).instructions),
    "random_small": lambda: (6, random_circuit(6, 200, seed=22).instructions),
}


@pytest.fixture(scope="module", autouse=True)
def need_cubins():
    if not oracle.reference_gpu_available():
        pytest.skip("reference kernels not built (make -C oracle ref needs the reference sources)")


@pytest.mark.parametrize("name", sorted(CIRCUITS))
@pytest.mark.parametrize("f32", [False, True])
def test_reference_kernels_match_the_oracle(name, f32):
    n, insts = CIRCUITS[name]()
    want, _ = oracle.run(n, insts)
    plan = oracle.PlannedCircuit(n, insts, max_k=3, gpu=True)
    ms, launches, got = oracle.run_reference_gpu(plan, f32=f32, repeats=2, state=True)
    assert launches > 0 and np.all(ms > 0)
    tol = 1e-5 if f32 else 1e-10
    assert np.abs(got - want).max() <= tol, name


def layered_launches(plan):
    """Kernel launches of run_layered (crates/aleph-cuda/src/sv/backend.rs:515-575)
    on the planned records: plain one-qubit gates gather into a pending layer,
    flushed in batches of 3 on a repeated qubit and before anything else; every
    other instruction is one launch."""
    ptr, cnt, _ = plan.records()
    launches, pending, mask = 0, 0, 0
    for i in range(cnt):
        r = ptr[i]
        if r.kind < 28 and r.num_qubits == 1 and r.num_controls == 0:
            if (mask >> r.qubits[0]) & 1:
                launches, pending, mask = launches + -(-pending // 3), 0, 0
            mask |= 1 << r.qubits[0]
            pending += 1
            continue
        launches, pending, mask = launches + -(-pending // 3) + 1, 0, 0
    return launches + -(-pending // 3)


def test_reference_layer_batches_on_the_brickwall():
    # every CZ layer is one apply_phase_poly sweep and the one-qubit gates go
    # out in apply_1q_multi batches of 3 (DEFAULT_LAYER_BATCH)
    n, depth = 12, 10
    plan = oracle.PlannedCircuit(n, workloads.brickwall(n, depth, seed=3).instructions, max_k=3, gpu=True)
    assert plan.counts()["tiled_blocks"] == depth  # DiagonalPhase records
    _, launches, _ = oracle.run_reference_gpu(plan, repeats=1)
    assert launches == layered_launches(plan)
    assert depth * 5 <= launches <= depth * (-(-n // 3) + 1) + 2
