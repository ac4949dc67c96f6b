"""Host-side tests of the OpenQASM 3 front end, the run surface's text
formats and the CLI's argument / error handling (no GPU).

The grammar cases follow the reference parser's own unit tests
(crates/aleph-parser/src/parser.rs:341-540, expr.rs:120-189, lower.rs
tests); the formats follow crates/aleph-cli/src/output.rs:123-217 and
pauli.rs."""
import math

import numpy as np
import pytest

from aleph_b200 import circuit as C
from aleph_b200 import frontend, qasm
from aleph_b200.__main__ import main as cli_main
from tests.fixtures_util import fixture_instructions, load_reference_fixtures


def ops(circ):
    out = []
    for i in circ.instructions:
        if isinstance(i, C.GateInstance):
            out.append(("gate", i.gate.name, i.qubits, tuple(i.gate.params)))
        elif isinstance(i, C.Measure):
            out.append(("measure", i.qubit, i.clbit))
        elif isinstance(i, C.Barrier):
            out.append(("barrier",) + tuple(i.qubits))
        elif isinstance(i, C.Reset):
            out.append(("reset", i.qubit))
    return out


def test_header_includes_and_declarations():
    assert qasm.parse("").num_qubits == 0
    c = qasm.parse('OPENQASM 3.0;\ninclude "stdgates.inc";\nqubit[2] q;\nqubit[3] aux;\nbit[5] c;')
    assert (c.num_qubits, c.num_clbits) == (5, 5)
    assert qasm.parse("OPENQASM 3; qubit[1] q;").num_qubits == 1
    # registers flatten in declaration order
    c = qasm.parse("qubit[2] a; qubit[3] b; h b[0]; x a[1];")
    assert ops(c) == [("gate", "H", (2,), ()), ("gate", "X", (1,), ())]


def test_statements_and_comments():
    src = """// leading comment
OPENQASM 3.0; /* block
comment */
include "stdgates.inc";
qubit[3] q; bit[3] c;
h q[0];  // trailing
rx(pi/2) q[1];
u3(0.1, 0.2, 0.3) q[2];
cx q[0], q[1]; cz q[1],q[2]; swap q[0], q[2];
ccx q[0], q[1], q[2]; ccz q[2], q[1], q[0];
barrier q[0], q[1];
barrier q;
measure q[1] -> c[0];
measure q -> c;
reset q[2];
"""
    got = ops(qasm.parse(src))
    assert got[0] == ("gate", "H", (0,), ())
    assert got[1][:3] == ("gate", "Rx", (1,)) and math.isclose(got[1][3][0], math.pi / 2, rel_tol=0, abs_tol=1e-15)
    assert got[2] == ("gate", "U3", (2,), (0.1, 0.2, 0.3))
    assert [g[1] for g in got[3:8]] == ["Cnot", "Cz", "Swap", "Toffoli", "Ccz"]
    assert got[8] == ("barrier", 0, 1) and got[9] == ("barrier", 0, 1, 2)
    assert got[10] == ("measure", 1, 0)
    assert got[11:14] == [("measure", 0, 0), ("measure", 1, 1), ("measure", 2, 2)]
    assert got[14] == ("reset", 2)


@pytest.mark.parametrize("expr,want", [
    ("1.5", 1.5), ("pi", math.pi), ("pi/2", math.pi / 2), ("1 + 2 * 3", 7.0), ("(1 + 2) * 3", 9.0),
    ("-pi", -math.pi), ("-(1 + 2)", -3.0), ("10 - 3 - 2", 5.0), ("1e-3", 1e-3), ("2.5E2", 250.0),
    ("  2 *  pi ", 2 * math.pi), ("-2*pi/3", -2 * math.pi / 3), (".5", 0.5)])
def test_parameter_expressions(expr, want):
    c = qasm.parse(f"qubit[1] q; rz({expr}) q[0];")
    assert c.instructions[0].gate.params[0] == pytest.approx(want, rel=0, abs=1e-15)


@pytest.mark.parametrize("src,kind,line,col", [
    ("qubit[2] q; h q[2];", "IndexOutOfBounds", 1, 15),
    ("qubit[2] q; foo q[0];", "UnknownGate", 1, 13),
    ("qubit[1] q; rx(1/0) q[0];", "BadExpression", 1, 17),
    ("qubit[1] q; rx(1/(2-2)) q[0];", "BadExpression", 1, 17),
    ("qubit[1] q; rx(1e308*10) q[0];", "BadExpression", 1, 16),
    ("qubit[2] q; cx q[0], q[0];", "IrRejected", 1, 13),
    ("qubit[2] q; cx q[0];", "IrRejected", 1, 13),
    ("qubit[2] q; bit[1] c; measure q -> c;", "SizeMismatch", 1, 23),
    ("qubit[2] q; bit[2] c; measure q -> c[0];", "UnsupportedFeature", 1, 23),
    ("OPENQASM 2.0; qubit[1] q;", "UnsupportedFeature", 1, 10),
    ('include "qelib1.inc"; qubit[1] q;', "UnsupportedFeature", 1, 1),
    ("qubit[1] q; h q[0]; qubit[1] r;", "UnsupportedFeature", 1, 21),
    ("qubit[1] q; rx q[0];", "UnexpectedToken", 1, 13),
    ("qubit[1] q; h r[0];", "UnknownRegister", 1, 15),
    ("qubit[1] q; qubit[2] q;", "DuplicateRegister", 1, 13),
    ("qubit[1] q;\nh q[0]", "UnexpectedToken", 2, 7),
    ("qubit[1] q; measure q[0] -> d[0];", "UnknownRegister", 1, 29),
])
def test_errors_carry_kind_and_position(src, kind, line, col):
    with pytest.raises(qasm.QasmError) as e:
        qasm.parse(src)
    assert (e.value.kind, e.value.line, e.value.col) == (kind, line, col)
    r = e.value.render().splitlines()
    assert r[0].startswith(f"error at {line}:{col}: ") and r[2] == " " * (col - 1) + "^"


def test_too_many_qubits():
    with pytest.raises(qasm.QasmError) as e:
        qasm.parse("qubit[65535] a; qubit[1] b;")
    assert e.value.kind == "TooManyQubits" and "declared 65536, max 65535" in str(e.value)


@pytest.mark.parametrize("fx", load_reference_fixtures(), ids=lambda f: f["name"])
def test_emit_parse_round_trip_on_reference_fixtures(fx):
    circ = C.Circuit(fx["num_qubits"], fixture_instructions(fx))
    back = qasm.parse(qasm.emit(circ))
    assert back.num_qubits == fx["num_qubits"]
    want = ops(circ)
    got = ops(back)
    # an unlabelled barrier comes back as the whole register
    want = [("barrier",) + tuple(range(fx["num_qubits"])) if w == ("barrier",) else w for w in want]
    assert got == want  # parameters survive exactly (repr round trip)


def test_emit_rejects_what_qasm_cannot_say():
    with pytest.raises(ValueError):
        qasm.emit(C.Circuit(2).add(C.Gate("Iswap"), [0, 1]))
    with pytest.raises(ValueError):
        qasm.emit(C.Circuit(2).add(C.H(), [0], [1]))


def test_counts_format():
    # output.rs tests: zero counts elided, ascending order, header label
    s = frontend.format_counts(frontend.counts_map([0, 0, 3, 3], 2), 4, 2, "seed=0")
    assert s == "counts (4 shots, seed=0):\n  |00⟩  2  (0.5000)\n  |11⟩  2  (0.5000)\n"
    s = frontend.format_counts(frontend.counts_map([3, 3, 0, 0, 1], 2), 5, 2, "seed=7")
    assert s.index("|00⟩") < s.index("|01⟩") < s.index("|11⟩")
    assert frontend.format_counts({}, 0, 2, "seed=7") == "counts (0 shots, seed=7):\n"
    assert frontend.format_counts(frontend.counts_map([0], 1), 1, 1, "seed=entropy").startswith(
        "counts (1 shots, seed=entropy):")
    # qubit 0 is the rightmost character
    assert list(frontend.counts_map([1], 3)) == ["001"]


def test_statevector_and_expectation_format():
    inv = 0.7071067811865476  # FRAC_1_SQRT_2
    s = frontend.format_statevector(np.array([inv, 0, 0, inv], dtype=np.complex128), 2)
    lines = s.splitlines()
    assert lines[0] == "statevector (2 qubits, 4 amplitudes):"
    assert lines[1] == "  |00⟩   +7.0710678118654757e-1 +0.0000000000000000e0i  |a|² = 0.500000"
    assert lines[2] == "  |01⟩   +0.0000000000000000e0 +0.0000000000000000e0i  |a|² = 0.000000"
    assert frontend._rust_exp(-0.125) == "-1.2500000000000000e-1"
    assert frontend._rust_exp(2.0 ** -40) == "+9.0949470177292824e-13"
    assert frontend._rust_exp(123.0) == "+1.2300000000000000e2"
    assert frontend.format_expectation("ZZ", 1.0) == "  ZZ    +1.0000000000000000\n"
    assert frontend.format_expectation("1.5*XX", -0.25) == "  1.5*XX    -0.2500000000000000\n"
    assert frontend.format_duration(1.234) == "1.2s"
    assert frontend.format_duration(0.0123) == "12.3ms"
    assert frontend.format_duration(12.5e-6) == "12.5µs"


def test_pauli_arguments():
    assert frontend.parse_pauli_arg("ZZ") == (1.0, [(0, "Z"), (1, "Z")])
    assert frontend.parse_pauli_arg("1.5*ZZ") == (1.5, [(0, "Z"), (1, "Z")])
    assert frontend.parse_pauli_arg("-0.5*X") == (-0.5, [(0, "X")])
    assert frontend.parse_pauli_arg("IXZI") == (1.0, [(1, "X"), (2, "Z")])
    for bad in ("", "ZZ*1.5", "ZA", "1.5*", "inf*Z"):
        with pytest.raises(ValueError):
            frontend.parse_pauli_arg(bad)


def test_backend_and_precision_names():
    assert frontend.resolve("b200", "auto") == "tc32"
    assert frontend.resolve("cuda", "auto") == "f64"
    assert frontend.resolve("cuda-f32") == "tc32"
    assert frontend.resolve("b200", "f64") == "f64"
    for b, p in (("metal", "auto"), ("stabilizer", "auto"), ("cuda", "f32"), ("b200", "f16")):
        with pytest.raises(ValueError):
            frontend.resolve(b, p)


def test_cli_errors_before_any_device_work(tmp_path, capsys):
    assert cli_main(["run", str(tmp_path / "missing.qasm")]) == 1
    assert "Error: reading QASM file" in capsys.readouterr().err
    bad = tmp_path / "bad.qasm"
    bad.write_text("qubit[2] q;\nh q[5];\n")
    assert cli_main(["run", str(bad)]) == 1
    err = capsys.readouterr().err
    assert f"Error: parsing {bad}" in err and "Caused by:" in err and "error at 2:3:" in err
    big = tmp_path / "big.qasm"
    big.write_text("qubit[11] q; h q[0];\n")
    assert cli_main(["run", str(big), "--statevector"]) == 1
    assert "pass --force-statevector" in capsys.readouterr().err
    ok = tmp_path / "ok.qasm"
    ok.write_text("qubit[2] q; h q[0];\n")
    assert cli_main(["run", str(ok), "--expectation", "ZZZ"]) == 1
    assert "references qubit 2 but circuit has 2 qubits" in capsys.readouterr().err
    assert cli_main(["run", str(ok), "--backend", "mps"]) == 1
    assert "unknown backend" in capsys.readouterr().err


def test_maxcut_pauli_sum_terms():
    """maxcut_pauli_sum (crates/aleph-ir/src/ansatz.rs:105-117): the identity
    at |E|/2 first, then -1/2 Z_i Z_j per edge in edge order; an edge beyond
    the register is an error."""
    from aleph_b200 import workloads

    assert workloads.maxcut_pauli_sum(2, [(0, 1)]) == [(0.5, []), (-0.5, [(0, "Z"), (1, "Z")])]
    h = workloads.maxcut_pauli_sum(4, [(0, 1), (2, 3), (1, 3)])
    assert h[0] == (1.5, []) and [t[1] for t in h[1:]] == [[(0, "Z"), (1, "Z")], [(2, "Z"), (3, "Z")],
                                                              [(1, "Z"), (3, "Z")]]
    # on a basis state the sum is the number of cut edges
    x = 0b0101
    cut = sum(((x >> i) & 1) != ((x >> j) & 1) for i, j in [(0, 1), (2, 3), (1, 3)])
    val = sum(c * math.prod(-1 if (x >> q) & 1 else 1 for q, _ in s) for c, s in h)
    assert val == cut
    with pytest.raises(ValueError):
        workloads.maxcut_pauli_sum(2, [(0, 2)])


def test_pauli_sum_text_format():
    """PauliSum::parse (crates/aleph-core/src/pauli.rs:115-170): comments,
    blanks, trailing identities dropped, the identity term, every error."""
    h = frontend.PauliSum.parse("# H2-like\n\n0.5 ZI\n  0.25 XX  \n-1.5 II\n", 2)
    assert h.num_terms() == 3
    assert h.terms == [(0.5, [(0, "Z")]), (0.25, [(0, "X"), (1, "X")]), (-1.5, [])]
    assert frontend.PauliSum.parse("1e-3 YZ\r\n", 2).terms == [(1e-3, [(0, "Y"), (1, "Z")])]
    bad = {
        "0.5\n": "line 1: expected '<coeff> <pauli>', got \"0.5\"",
        "\n0.5 ZZ X\n": "line 2: expected '<coeff> <pauli>', got \"0.5 ZZ X\"",
        "half ZZ\n": "line 1: coefficient \"half\" is not a finite float",
        "1_0 ZZ\n": "line 1: coefficient \"1_0\" is not a finite float",
        "0.5 ZZZ\n": "line 1: pauli string has 3 chars, expected 2",
        "0.5 ZA\n": "line 1: 'A' is not one of I,X,Y,Z",
        "inf ZZ\n": "line 1: non-finite coefficient",
        "0.5\tZZ\tX\n": "line 1: expected '<coeff> <pauli>', got \"0.5\\tZZ\\tX\"",  # Rust {:?} escapes
        '0.5 Z"\n': "line 1: '\"' is not one of I,X,Y,Z",  # a char's {:?} keeps '"' bare
    }
    for src, msg in bad.items():
        with pytest.raises(frontend.PauliSumError) as e:
            frontend.PauliSum.parse(src, 2)
        assert str(e.value) == msg


def test_pauli_sum_load(tmp_path):
    p = tmp_path / "h.txt"
    p.write_text("0.5 ZZ\n0.5 XQ\n")
    with pytest.raises(ValueError, match=r"^parse .*h\.txt: line 2: 'Q' is not one of I,X,Y,Z$"):
        frontend.PauliSum.load(str(p), 2)
    with pytest.raises(ValueError, match=r"^read .*missing\.txt: "):
        frontend.PauliSum.load(str(tmp_path / "missing.txt"), 2)
    p.write_text("0.5 ZZ\n-0.25 XY\n")
    assert frontend.PauliSum.load(str(p), 2).terms == [(0.5, [(0, "Z"), (1, "Z")]), (-0.25, [(0, "X"), (1, "Y")])]


def test_build_hea_layout():
    """build_hea (crates/aleph-ir/src/ansatz.rs:32-61): Ry layer + CNOT chain
    per entangling layer, a final Ry layer; params[layer * n + q]."""
    from aleph_b200 import workloads

    n, depth = 3, 2
    params = [0.1 * (i + 1) for i in range(n * (depth + 1))]
    c = workloads.build_hea(n, depth, params)
    got = [(g.gate.name, list(g.qubits), g.gate.params) for g in c.instructions]
    want = []
    for layer in range(depth + 1):
        want += [("Ry", [q], (params[layer * n + q],)) for q in range(n)]
        if layer < depth:
            want += [("Cnot", [q, q + 1], ()) for q in range(n - 1)]
    assert got == want
    with pytest.raises(ValueError, match=r"expected 9 params \(n_qubits\*\(depth\+1\)\), got 8"):
        workloads.build_hea(n, depth, params[:-1])
