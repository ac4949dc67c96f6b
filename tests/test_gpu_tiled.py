"""TiledBlock records through the engine against the oracle, through the C ABI.

The reference's CPU backend applies a TiledBlock tile by tile
(NaiveSvBackend::apply_tiled_block, crates/aleph-sv/src/backend.rs:173-299):
controls at or above tile_bits skip the tiles where they are 0, gates take
their fixed-size 2x2 / 4x4 matrix with no unitarity check, and a gate with an
8x8 matrix (or a UnitaryKq, which has none) is UnsupportedGate. Tolerances:
FP64 1e-12 against the FP64 oracle, FP32 1e-5.
"""
import numpy as np
import pytest

from aleph_b200 import abi
from aleph_b200 import circuit as C
from aleph_b200 import workloads
from aleph_b200.backend import B200SvBackend, BackendError, run
from oracle import oracle

pytestmark = pytest.mark.gpu


def tiled_circuit(n, tile_bits, seed, blocks=6, per_block=30):
    """Runs of tile-confinable gates (targets < tile_bits) with controls on
    any qubit, including qubits at or above tile_bits, between plain gates."""
    rng = np.random.default_rng(seed)
    insts = []
    t = min(tile_bits, n)
    for _ in range(blocks):
        gates = []
        for _ in range(per_block):
            lo = [int(x) for x in rng.permutation(t)]
            ctrl = [int(rng.integers(t, n))] if n > t and rng.random() < 0.4 else []
            if not ctrl and rng.random() < 0.2:
                ctrl = [lo[2]]
            if rng.random() < 0.4:
                z = rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4))
                gates.append(C.GateInstance(C.Unitary2q(np.linalg.qr(z)[0]), lo[:2], ctrl))
            else:
                g = [C.Unitary1q(workloads.haar_su2(rng)), C.H(), C.Rz(float(rng.uniform(-3, 3))), C.Cz()][
                    int(rng.integers(0, 4))]
                gates.append(C.GateInstance(g, lo[: g.arity()], ctrl))
        insts.append(C.TiledBlock(gates, tile_bits))
        q = int(rng.integers(0, n))
        insts.append(C.GateInstance(C.Unitary1q(workloads.haar_su2(rng)), [q]))
    return insts


@pytest.mark.parametrize("n,tile_bits", [(12, 15), (18, 15), (20, 15), (16, 6)])
def test_tiled_blocks_match_oracle_f64(n, tile_bits):
    insts = tiled_circuit(n, tile_bits, seed=n * 7 + tile_bits)
    want, _ = oracle.run(n, insts)
    be = B200SvBackend(seed=0, precision="f64")
    st = run(be, C.Circuit(n, insts))
    assert np.abs(be.statevector(st) - want).max() <= 1e-12


@pytest.mark.parametrize("precision", ["f32", "tc32"])
def test_tiled_blocks_match_oracle_f32(precision):
    n = 18
    insts = tiled_circuit(n, 15, seed=99)
    want, _ = oracle.run(n, insts)
    be = B200SvBackend(seed=0, precision=precision)
    st = run(be, C.Circuit(n, insts))
    assert np.abs(be.statevector(st) - want).max() <= 1e-5


def test_tiled_block_applies_a_non_unitary_matrix_like_the_reference():
    # apply_tiled_block takes Gate::matrix() as it is: no unitarity check
    n = 10
    m = np.array([[1.0, 0.5], [0.0, 1.0]], dtype=np.complex128)
    insts = [C.GateInstance(C.H(), [3]), C.TiledBlock([C.GateInstance(C.Unitary1q(m), [3]),
                                                      C.GateInstance(C.H(), [1])], 15)]
    want, _ = oracle.run(n, insts)
    be = B200SvBackend(seed=0, precision="f64")
    st = be.allocate(n)
    be.apply_stream(st, insts)
    assert np.abs(be.statevector(st) - want).max() <= 1e-12
    # outside a TiledBlock the same gate is NonUnitaryMatrix
    st2 = be.allocate(n)
    with pytest.raises(BackendError) as e:
        be.apply_stream(st2, [C.GateInstance(C.Unitary1q(m), [3])])
    assert e.value.status == abi.NON_UNITARY_MATRIX


@pytest.mark.parametrize("gate,qubits", [(C.Toffoli(), [0, 1, 2]), (C.Ccz(), [2, 0, 1]),
                                         ("kq", [0, 1, 2])])
def test_tiled_block_rejects_3q_and_unitary_kq(gate, qubits):
    if gate == "kq":
        z = np.random.default_rng(1).standard_normal((8, 8)) + 0j
        gate = C.UnitaryKq(np.linalg.qr(z)[0])
    n = 8
    insts = [C.TiledBlock([C.GateInstance(C.H(), [0]), C.GateInstance(gate, qubits)], 15)]
    with pytest.raises(oracle.OracleError) as oe:
        oracle.run(n, insts)
    assert oe.value.status == abi.UNSUPPORTED_GATE
    be = B200SvBackend(seed=0, precision="f64")
    st = be.allocate(n)
    with pytest.raises(BackendError) as e:
        be.apply_stream(st, insts)
    assert e.value.status == abi.UNSUPPORTED_GATE
    assert e.value.info.instruction == 2  # the record of the 3-qubit gate
    # the same gate outside a TiledBlock is applied
    st2 = be.allocate(n)
    be.apply_stream(st2, [C.GateInstance(gate, qubits)])
