"""The run surface on the GPU: OpenQASM text -> engine -> counts /
statevector / expectation, checked against the golden fixtures and the
oracle; the CLI end to end; ``qaoa_energy`` against the oracle."""
import math
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from aleph_b200 import circuit as C
from aleph_b200 import frontend, qasm, workloads
from oracle import oracle
from tests.fixtures_util import fixture_instructions, fixture_state, load_reference_fixtures

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
FIXTURES = [f for f in load_reference_fixtures() if not any(o["op"] == "measure" for o in f["ops"])]


@pytest.mark.parametrize("fx", FIXTURES, ids=lambda f: f["name"])
def test_qasm_text_through_run_matches_golden(fx):
    src = qasm.emit(C.Circuit(fx["num_qubits"], fixture_instructions(fx)))
    res = frontend.run(src, shots=64, backend="cuda", seed=1)
    psi = res.statevector()
    assert np.abs(psi - fixture_state(fx)).max() <= 1e-10
    want, _ = oracle.run(fx["num_qubits"], qasm.parse(src).instructions)
    assert np.abs(psi - want).max() <= 1e-12
    assert sum(res.counts().values()) == 64
    res.close()


def test_counts_are_seeded_and_follow_the_distribution():
    n = 14
    c = workloads.brickwall(n, 6, seed=3)
    src = None  # brickwall uses Unitary1q records: run the Circuit directly
    r1 = frontend.run(c, shots=4096, backend="b200", precision="f64", seed=11)
    r2 = frontend.run(c, shots=4096, backend="b200", precision="f64", seed=11)
    r3 = frontend.run(c, shots=4096, backend="b200", precision="f64", seed=12)
    assert r1.counts() == r2.counts() and r1.counts() != r3.counts()
    assert r1.seed_label == "seed=11" and frontend.run(c, shots=1).seed_label == "seed=entropy"
    psi, _ = oracle.run(n, c.instructions)
    p = np.abs(psi) ** 2
    # every sampled bitstring has non-zero probability; the heaviest ones show up
    for bits in r1.counts():
        assert p[int(bits, 2)] > 0
    top = np.argsort(p)[::-1][:5]
    assert any(format(int(i), f"0{n}b") in r1.counts() for i in top)
    for r in (r1, r2, r3):
        r.close()
    del src


def test_expectation_and_measurements_on_a_ghz_state():
    src = 'OPENQASM 3.0;\ninclude "stdgates.inc";\nqubit[3] q;\nbit[1] c;\nh q[0];\ncx q[0], q[1];\ncx q[1], q[2];\n'
    res = frontend.run(src, shots=500, backend="cuda", seed=4)
    assert set(res.counts()) <= {"000", "111"} and sum(res.counts().values()) == 500
    assert res.expectation("ZZI") == pytest.approx(1.0, abs=1e-12)
    assert res.expectation("XXX") == pytest.approx(1.0, abs=1e-12)
    assert res.expectation("-0.5*ZII") == pytest.approx(0.0, abs=1e-12)
    amps = res.statevector()  # releases the device state; expectations still answer on the host copy
    assert res.expectation("XXX") == pytest.approx(1.0, abs=1e-12)
    assert abs(amps[0]) == pytest.approx(1 / math.sqrt(2), abs=1e-12)
    res.close()
    # a mid-circuit measurement collapses the state once; shots re-sample it
    res = frontend.run(src + "measure q[0] -> c[0];\n", shots=200, backend="cuda", seed=9)
    m = res.measurements()
    assert len(m) == 1 and set(res.counts()) == {"111" if m[0].outcome else "000"}
    res.close()


def test_reset_is_rejected_like_the_reference_sv_backend():
    from aleph_b200.backend import BackendError

    with pytest.raises(BackendError):
        frontend.run("qubit[2] q; h q[0]; reset q[0];", shots=1)


def run_cli(*args):
    return subprocess.run([sys.executable, "-m", "aleph_b200", *args], cwd=ROOT, capture_output=True, text=True,
                          timeout=300)


def test_cli_run_views(tmp_path):
    f = tmp_path / "bell.qasm"
    f.write_text('OPENQASM 3.0;\ninclude "stdgates.inc";\nqubit[2] q;\nh q[0];\ncx q[0], q[1];\n')
    r = run_cli("run", str(f), "--shots", "1000", "--seed", "5", "--statevector", "--expectation", "ZZ",
                "--expectation", "0.5*XX", "--backend", "cuda")
    assert r.returncode == 0, r.stderr
    lines = r.stdout.splitlines()
    assert lines[0] == "counts (1000 shots, seed=5):"
    counted = {l.split()[0]: int(l.split()[1]) for l in lines[1:3]}
    assert set(counted) == {"|00⟩", "|11⟩"} and sum(counted.values()) == 1000
    assert lines[3] == "statevector (2 qubits, 4 amplitudes):"
    assert lines[4].startswith("  |00⟩   +7.07106781186547") and lines[4].endswith("|a|² = 0.500000")
    assert lines[8] == "expectation values:"
    name, value = lines[9].split()
    assert name == "ZZ" and abs(float(value) - 1.0) <= 1e-12 and len(value.split(".")[1]) == 16
    name, value = lines[10].split()
    assert name == "0.5*XX" and abs(float(value) - 0.5) <= 1e-12
    # default view: 1024 shots
    r = run_cli("run", str(f), "--seed", "1")
    assert r.returncode == 0 and r.stdout.startswith("counts (1024 shots, seed=1):")
    # same seed, same counts
    assert run_cli("run", str(f), "--seed", "1").stdout == r.stdout
    # bench
    r = run_cli("bench", str(f))
    assert r.returncode == 0, r.stderr
    assert r.stdout.splitlines()[0] == "bench bell.qasm (n=2):"
    assert [l.split()[0] for l in r.stdout.splitlines()[1:]] == ["parse", "run", "sample(1024)", "total"]


def test_qaoa_energy_against_the_oracle():
    rng = np.random.default_rng(7)
    n = 10
    edges = workloads.random_3_regular(n, rng)
    g, b = rng.uniform(0, np.pi, 3), rng.uniform(0, np.pi, 3)
    psi, _ = oracle.run(n, workloads.qaoa_maxcut(n, edges, g, b).instructions)
    want = sum(0.5 * (1 - oracle.expectation(psi, [(i, "Z"), (j, "Z")])) for i, j in edges)
    assert frontend.qaoa_energy(n, edges, g, b) == pytest.approx(want, abs=1e-9)
    # the gate-by-gate path (above the sweep's size limit) agrees
    got = frontend.qaoa_energies([(n, edges)], [g], [b], sweep_max_n=0)[0]
    assert got == pytest.approx(want, abs=1e-9)
    assert frontend.qaoa_energy(n, edges, g, b, precision="f32") == pytest.approx(want, rel=2e-5)


def _synthetic_hamiltonian(n, count, seed):
    """A seeded stand-in for a VQE Hamiltonian in the committed text format."""
    rng = np.random.default_rng(seed)
    lines = ["# synthetic: seeded Pauli terms"]
    for _ in range(count):
        lines.append(f"{rng.uniform(-1, 1):.12f} " + "".join(rng.choice(list("IIXYZ"), size=n)))
    return "\n".join(lines) + "\n"


def test_hea_energy_against_the_oracle():
    n, depth = 6, 3
    ham = frontend.PauliSum.parse(_synthetic_hamiltonian(n, 40, 11), n)
    rng = np.random.default_rng(12)
    thetas = rng.uniform(-np.pi, np.pi, n * (depth + 1))
    psi, _ = oracle.run(n, workloads.build_hea(n, depth, thetas).instructions)
    want = sum(oracle.expectation(psi, s, c) for c, s in ham.terms)
    assert frontend.hea_energy(n, depth, thetas, ham) == pytest.approx(want, abs=1e-12)
    assert frontend.hea_energy(n, depth, thetas, ham, precision="f32") == pytest.approx(want, abs=5e-5)
    assert frontend.hea_energy(n, depth, thetas, ham, precision="tc32") == pytest.approx(want, abs=5e-5)


def test_hea_energy_is_sinusoidal_in_each_angle():
    """Each Ry angle enters as exp(-i theta Y / 2): E(theta_j) = A cos(theta_j - phi) + c,
    so E(b) + E(b + pi) = E(b + pi/2) + E(b - pi/2) (the identity rotosolve
    steps on, benches/tests/vqe_h2_convergence.rs)."""
    n, depth = 5, 2
    ham = frontend.PauliSum.parse(_synthetic_hamiltonian(n, 25, 13), n)
    base = [0.1 * (i + 1) for i in range(n * (depth + 1))]
    for j in (0, 7, len(base) - 1):
        def e(shift):
            t = list(base)
            t[j] += shift
            return frontend.hea_energy(n, depth, t, ham)
        assert e(0.0) + e(np.pi) == pytest.approx(e(np.pi / 2) + e(-np.pi / 2), abs=1e-12)
