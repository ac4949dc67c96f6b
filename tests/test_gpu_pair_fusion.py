"""Pair fusion in warp-tile passes (planner.cpp `fuse_pairs`): a gate on two
qubits and the one-qubit gates beside it run as one 4x4. The fused plan must
match the oracle as the unfused one does (FP64 1e-12, FP32 1e-5), for every
op kind a block can take: dense and diagonal one-qubit gates, CZ and
controlled phases, controlled one-qubit gates (CNOT, CRx), dense 4x4s and
same-pair repeats, with blocks on lane qubits (0..4), register qubits and
both."""
import numpy as np
import pytest

from aleph_b200 import circuit as C
from aleph_b200 import workloads
from aleph_b200.backend import B200SvBackend, describe_plan
from oracle import oracle
from tests.circuit_gen import random_circuit

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-12, "f32": 1e-5}


def pair_heavy_circuit(n, gates, seed, hot=(0, 3, 4, 5, 9)):
    """Many two-qubit gates on a few qubits, with one-qubit gates of every
    kind between them: most of it ends up in fused blocks."""
    rng = np.random.default_rng(seed)
    hot = [q for q in hot if q < n]
    c = C.Circuit(n)
    one = [lambda: C.H(), lambda: C.T(), lambda: C.S(), lambda: C.Rz(rng.uniform(-3, 3)),
           lambda: C.Ry(rng.uniform(-3, 3)), lambda: C.U3(*rng.uniform(-3, 3, 3)),
           lambda: C.Unitary1q(workloads.haar_su2(rng)), lambda: C.X()]
    two = [lambda: C.Cz(), lambda: C.Cnot(), lambda: C.CRx(rng.uniform(-3, 3)), lambda: C.CRz(rng.uniform(-3, 3)),
           lambda: C.Iswap(), lambda: C.Unitary2q(np.linalg.qr(rng.standard_normal((4, 4))
                                                                + 1j * rng.standard_normal((4, 4)))[0])]
    for _ in range(gates):
        r = rng.random()
        if r < 0.55:
            c.add(one[int(rng.integers(len(one)))](), [int(rng.choice(hot))])
        elif r < 0.92:
            a, b = (int(x) for x in rng.choice(hot, 2, replace=False))
            c.add(two[int(rng.integers(len(two)))](), [a, b])
        else:  # a wider gate closes the open blocks on its qubits
            a, b, d = (int(x) for x in rng.choice(hot, 3, replace=False))
            c.add(C.Toffoli(), [a, b, d])
    # a few gates on the other qubits, so tiles have outer work too
    for q in range(n):
        if q not in hot:
            c.add(C.H(), [q])
    return c


def run_engine(circ, precision, **tuning):
    be = B200SvBackend(seed=0, precision=precision)
    for k, v in tuning.items():
        be.set_tuning(k, v)
    st = be.allocate(circ.num_qubits)
    be.apply_stream(st, circ.instructions)
    got = be.statevector(st)
    st.free()
    be.close()
    return got


CIRCUITS = {
    "pair_heavy": lambda n: pair_heavy_circuit(n, 400, seed=n),
    "brickwall": lambda n: workloads.brickwall(n, 14, seed=n + 1),
    "qft": lambda n: workloads.qft_product(n, seed=n + 2),
    "random": lambda n: random_circuit(n, 250, seed=n + 3),
}


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("tile_r", [2, 5])
@pytest.mark.parametrize("name", sorted(CIRCUITS))
def test_fused_and_unfused_plans_match_the_oracle(name, tile_r, precision):
    n = 14
    c = CIRCUITS[name](n)
    want, _ = oracle.run(n, c.instructions)
    fused = run_engine(c, precision, tile_r=tile_r, smem_max_n=0)
    plain = run_engine(c, precision, tile_r=tile_r, smem_max_n=0, pair_fusion=0)
    assert np.abs(fused - want).max() <= TOL[precision]
    assert np.abs(plain - want).max() <= TOL[precision]


def test_fusion_takes_the_pair_heavy_circuit_apart_into_blocks():
    # the planner really fused: fewer dense ops per pass, same gate total
    c = pair_heavy_circuit(16, 400, seed=5)
    on = describe_plan(16, c.instructions, "f64", smem_max_n=0)
    off = describe_plan(16, c.instructions, "f64", smem_max_n=0, pair_fusion=False)
    assert sum(p["dense_ops"] for p in on) < 0.8 * sum(p["dense_ops"] for p in off)
    want, _ = oracle.run(16, c.instructions)
    assert np.abs(run_engine(c, "f64", smem_max_n=0) - want).max() <= TOL["f64"]
