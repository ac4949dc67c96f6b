"""The CPU oracle against the reference's own golden vectors.

Mirrors the reference's generated per-fixture tests
(crates/aleph-oracle/build.rs:95-170, harness.rs:35-80): every fixture's
circuit is run raw, gate by gate, and each amplitude must match Qiskit-Aer's
statevector within |delta| <= 1e-10 (STATE_TOLERANCE, harness.rs:18).
"""
import numpy as np
import pytest

from oracle import oracle
from tests.fixtures_util import fixture_instructions, fixture_state, load_reference_fixtures

STATE_TOLERANCE = 1e-10
FIXTURES = load_reference_fixtures()


@pytest.mark.parametrize("fx", FIXTURES, ids=[f["name"] for f in FIXTURES])
def test_oracle_matches_reference_fixture(fx):
    psi, _ = oracle.run(fx["num_qubits"], fixture_instructions(fx), uniforms=fx["measure_uniforms"])
    want = fixture_state(fx)
    assert np.all(np.isfinite(psi))
    delta = np.abs(psi - want)
    assert delta.max() <= STATE_TOLERANCE, (fx["name"], int(delta.argmax()), float(delta.max()))


def test_fixture_count():
    # 31 QASM circuits with Aer statevectors in the reference's oracle/ tree.
    assert len(FIXTURES) == 31
