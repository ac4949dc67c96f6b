"""Out-of-core runs (aleph_b200_paged_run) against the oracle.

The state lives in pinned host memory and tile groups stream through the
device (crates/aleph-cuda/src/sv/paged.rs). As the reference's paged oracle
tests do, small states force a small tile split; the `paged_local_qubits`
tuning key also caps the device tile group, so that the runs below cut the
gate list into many segments and gather many groups per segment.
"""
import numpy as np
import pytest

from aleph_b200 import backend as B
from aleph_b200 import circuit as C
from aleph_b200 import workloads
from aleph_b200.backend import B200SvBackend
from oracle import oracle
from tests.circuit_gen import random_circuit

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,m,local", [(12, 4, 9), (14, 6, 11), (16, 9, 14)])
def test_paged_f64_matches_the_oracle(n, m, local):
    c = random_circuit(n, 120, seed=500 + n)
    be = B200SvBackend(seed=0).set_tuning("paged_local_qubits", local)
    ps = be.run_paged(c, m)
    want, _ = oracle.run(n, c.instructions)
    assert np.abs(ps.statevector() - want).max() <= 1e-12
    assert ps.norm_sqr() == pytest.approx(1.0, abs=1e-12)
    info = ps.info()
    assert info["tile_qubits"] == m and info["local_qubits"] <= local
    assert info["segments"] > 1 and info["groups"] > info["segments"]
    # every segment writes the whole host state once; every segment after the
    # first reads it once (the first generates |0...0> on the device)
    assert info["d2h_bytes"] == info["segments"] * (16 << n)
    assert info["h2d_bytes"] == (info["segments"] - 1) * (16 << n)
    ps.free()
    be.close()


def test_paged_ring_depth_does_not_change_the_state():
    """Depth 1 (no overlap), 2 and 4 run the same groups with the same plans:
    the states are bitwise equal."""
    n = 15
    c = random_circuit(n, 80, seed=77)
    states = []
    for depth in (1, 2, 4):
        be = B200SvBackend(seed=0).set_tuning("paged_local_qubits", 12)
        ps = be.run_paged(c, 7, depth=depth)
        assert ps.info()["depth"] == depth
        states.append(ps.statevector())
        ps.free()
        be.close()
    assert np.array_equal(states[0], states[1]) and np.array_equal(states[0], states[2])


@pytest.mark.parametrize("precision", ["f32", "tc32"])
def test_paged_fp32_and_tensor_core_segments(precision):
    n = 18
    c = workloads.brickwall(n, 8, seed=78)
    be = B200SvBackend(seed=0, precision=precision).set_tuning("paged_local_qubits", 15)
    ps = be.run_paged(c, 10)
    want, _ = oracle.run(n, c.instructions)
    got = ps.statevector()
    assert np.abs(got - want).max() <= 1e-5
    assert 1.0 - abs(np.vdot(got, want)) ** 2 / np.vdot(got, got).real <= 1e-6
    assert ps.info()["segments"] > 1
    if precision == "tc32":
        assert be.stats()["block_passes"] > 0
    ps.free()
    be.close()


def test_paged_errors():
    """run_paged's error order (paged.rs:143-197): empty circuit, tile split,
    unsupported instructions, device capacity; then gate validation."""
    be = B200SvBackend(seed=0)
    with pytest.raises(B.EmptyCircuit):
        be.run_paged(C.Circuit(0), 1)
    c = C.Circuit(6).add(C.H(), [0]).add(C.Cnot(), [0, 5])
    with pytest.raises(B.InvalidState, match="tile_qubits"):
        be.run_paged(c, 0)
    with pytest.raises(B.InvalidState, match="tile_qubits"):
        be.run_paged(c, 6)
    for inst, kind in ((C.Measure(1, 0), "measure"), (C.Reset(2), "reset"),
                       (C.DiagonalPhase(6, [C.PhaseTerm((3,), 0.2)]), "diagonal-phase")):
        bad = C.Circuit(6).add(C.H(), [0])
        bad.instructions.append(inst)
        with pytest.raises(B.UnsupportedInstruction) as e:
            be.run_paged(bad, 3)
        assert e.value.info.kind.decode() == kind
    wide = C.Circuit(10).add(C.Toffoli(), [7, 8, 9])
    be.set_tuning("paged_local_qubits", 6)
    with pytest.raises(B.TooManyQubits) as e:
        be.run_paged(wide, 4)
    assert (e.value.info.requested, e.value.info.limit) == (7, 6)
    with pytest.raises(B.QubitOutOfRange):
        be.run_paged(C.Circuit(6).add(C.H(), [6]), 3)
    be.close()
