"""OpenQASM 3 front end: the subset the reference's parser accepts
(crates/aleph-parser/src/parser.rs, lower.rs:123-452, expr.rs), lowered to
this package's circuit records.

Accepted programs:

- an optional ``OPENQASM 3;`` / ``OPENQASM 3.x;`` header (major version 3 only);
- ``include "stdgates.inc";`` (any other include is an unsupported feature);
- declarations ``qubit[n] name;`` and ``bit[n] name;`` before any statement;
- gate statements with the stdgates names of lower.rs:255-283 (``h x y z s
  sdg t tdg rx ry rz p u3 cx cz swap ccx``, plus ``ccz``). Parameters are
  constant expressions of float literals, ``pi``, ``+ - * /``, unary minus
  and parentheses, evaluated when parsed; division by zero and non-finite
  results are errors;
- ``barrier`` over indexed qubits or whole registers;
- ``measure q[i] -> c[j];`` and ``measure q -> c;`` (equal sizes);
- ``reset q[i];`` (lowered to a Reset record, which the engine rejects as
  UnsupportedInstruction, like the reference's state-vector backend).

Whitespace, ``//`` line comments and ``/* */`` block comments are skipped.
Registers map to flat indices in declaration order. Errors are
:class:`QasmError` with the reference's 1-based line/column and message
texts (error.rs:6-118).
"""
from __future__ import annotations

import math
import re
from dataclasses import dataclass

from . import circuit as C

MAX_QUBITS = 65_535  # crates/aleph-ir/src/circuit.rs:22
MAX_CLBITS = 65_535

# qasm name -> (Gate variant, parameter count); lower.rs:255-283
GATES = {
    "h": ("H", 0), "x": ("X", 0), "y": ("Y", 0), "z": ("Z", 0), "s": ("S", 0), "sdg": ("Sdg", 0),
    "t": ("T", 0), "tdg": ("Tdg", 0), "rx": ("Rx", 1), "ry": ("Ry", 1), "rz": ("Rz", 1),
    "p": ("Phase", 1), "u3": ("U3", 3), "cx": ("Cnot", 0), "cz": ("Cz", 0), "swap": ("Swap", 0),
    "ccx": ("Toffoli", 0), "ccz": ("Ccz", 0),
}
GATE_NAMES = {v[0]: k for k, v in GATES.items()}


class QasmError(ValueError):
    """A positioned parse/lowering failure. ``kind`` names the reference's
    ParseErrorKind variant; ``str(err)`` is its display text."""

    def __init__(self, line: int, col: int, kind: str, message: str, snippet: str = ""):
        self.line, self.col, self.kind, self.message, self.snippet = line, col, kind, message, snippet
        super().__init__(f"error at {line}:{col}: {message}")

    def render(self) -> str:
        """Three lines: the message, the source line, a caret under the column."""
        return f"error at {self.line}:{self.col}: {self.message}\n{self.snippet}\n{' ' * max(self.col - 1, 0)}^\n"


@dataclass
class Tok:
    kind: str  # "id", "num", "str", "op", "eof"
    text: str
    line: int
    col: int


_TOKEN = re.compile(
    r"(?P<ws>[ \t\r\n]+)|(?P<lc>//[^\n\r]*)|(?P<bc>/\*.*?\*/)"
    r"|(?P<num>(?:\d+\.\d*|\.\d+|\d+)(?:[eE][+-]?\d+)?)"
    r"|(?P<id>[A-Za-z_][A-Za-z0-9_]*)|(?P<str>\"[^\"\n]*\")"
    r"|(?P<op>->|[\[\]();,+\-*/])",
    re.S)


def _tokenize(src: str) -> list[Tok]:
    toks, pos, line, lstart = [], 0, 1, 0
    while pos < len(src):
        m = _TOKEN.match(src, pos)
        if not m:
            if src.startswith("/*", pos):
                raise QasmError(line, pos - lstart + 1, "UnexpectedToken",
                                "unexpected token: expected end of block comment, found `end of source`",
                                _nth_line(src, line))
            raise QasmError(line, pos - lstart + 1, "UnexpectedToken",
                            f"unexpected token: expected statement, found `{src[pos]}`", _nth_line(src, line))
        kind = m.lastgroup
        text = m.group(kind)
        if kind not in ("ws", "lc", "bc"):
            toks.append(Tok(kind, text, line, pos - lstart + 1))
        nl = text.count("\n")
        if nl:
            line += nl
            lstart = pos + text.rindex("\n") + 1
        pos = m.end()
    toks.append(Tok("eof", "", line, pos - lstart + 1))
    return toks


def _nth_line(src: str, line: int) -> str:
    lines = src.splitlines()
    return lines[line - 1] if 1 <= line <= len(lines) else ""


class _Parser:
    def __init__(self, src: str):
        self.src = src
        self.toks = _tokenize(src)
        self.i = 0

    # ---- token helpers ----
    @property
    def tok(self) -> Tok:
        return self.toks[self.i]

    def err(self, tok: Tok, kind: str, message: str) -> QasmError:
        return QasmError(tok.line, tok.col, kind, message, _nth_line(self.src, tok.line))

    def expect(self, text: str, what: str | None = None) -> Tok:
        t = self.tok
        if t.text != text or t.kind == "str":
            found = "end of source" if t.kind == "eof" else t.text
            raise self.err(t, "UnexpectedToken", f"unexpected token: expected {what or '`' + text + '`'}, found `{found}`")
        self.i += 1
        return t

    def accept(self, text: str) -> bool:
        if self.tok.text == text and self.tok.kind != "str":
            self.i += 1
            return True
        return False

    def ident(self, what: str) -> Tok:
        t = self.tok
        if t.kind != "id":
            found = "end of source" if t.kind == "eof" else t.text
            raise self.err(t, "UnexpectedToken", f"unexpected token: expected {what}, found `{found}`")
        self.i += 1
        return t

    def uint(self, what: str) -> int:
        t = self.tok
        if t.kind != "num" or not t.text.isdigit():
            found = "end of source" if t.kind == "eof" else t.text
            raise self.err(t, "UnexpectedToken", f"unexpected token: expected {what}, found `{found}`")
        self.i += 1
        return int(t.text)

    # ---- expressions (expr.rs: add -> mul -> unary -> atom) ----
    def expr(self) -> float:
        start = self.tok
        v = self._add()
        if not math.isfinite(v):
            raise self.err(start, "BadExpression", f"bad expression: non-finite value {v}")
        return v

    def _add(self) -> float:
        v = self._mul()
        while self.tok.text in ("+", "-") and self.tok.kind == "op":
            op = self.tok.text
            self.i += 1
            r = self._mul()
            v = v + r if op == "+" else v - r
        return v

    def _mul(self) -> float:
        v = self._unary()
        while self.tok.text in ("*", "/") and self.tok.kind == "op":
            op = self.tok
            self.i += 1
            r = self._unary()
            if op.text == "*":
                v = v * r
            else:
                if r == 0.0:
                    raise self.err(op, "BadExpression", "bad expression: division by zero")
                v = v / r
        return v

    def _unary(self) -> float:
        if self.tok.text == "-" and self.tok.kind == "op":
            self.i += 1
            return -self._unary()
        return self._atom()

    def _atom(self) -> float:
        t = self.tok
        if t.kind == "num":
            self.i += 1
            return float(t.text)
        if t.kind == "id" and t.text == "pi":
            self.i += 1
            return math.pi
        if self.accept("("):
            v = self._add()
            self.expect(")")
            return v
        found = "end of source" if t.kind == "eof" else t.text
        raise self.err(t, "UnexpectedToken", f"unexpected token: expected expression, found `{found}`")

    # ---- program ----
    def program(self) -> C.Circuit:
        t = self.tok
        if t.kind == "id" and t.text == "OPENQASM":
            self.i += 1
            vt = self.tok
            if vt.kind != "num" or not re.fullmatch(r"\d+(\.\d+)?", vt.text):
                found = "end of source" if vt.kind == "eof" else vt.text
                raise self.err(vt, "UnexpectedToken", f"unexpected token: expected version number, found `{found}`")
            if int(vt.text.split(".")[0]) != 3:
                raise self.err(vt, "UnsupportedFeature", "unsupported feature: OpenQASM major version other than 3")
            self.i += 1
            self.expect(";")
        while self.tok.kind == "id" and self.tok.text == "include":
            inc = self.tok
            self.i += 1
            p = self.tok
            if p.kind != "str":
                found = "end of source" if p.kind == "eof" else p.text
                raise self.err(p, "UnexpectedToken", f"unexpected token: expected string literal, found `{found}`")
            self.i += 1
            self.expect(";")
            if p.text[1:-1] != "stdgates.inc":
                raise self.err(inc, "UnsupportedFeature", "unsupported feature: non-stdgates include")
        qregs: dict[str, tuple[int, int]] = {}
        cregs: dict[str, tuple[int, int]] = {}
        nq = nc = 0
        while self.tok.kind == "id" and self.tok.text in ("qubit", "bit"):
            d = self.tok
            self.i += 1
            self.expect("[")
            size = self.uint("register size")
            self.expect("]")
            name = self.ident("register name")
            self.expect(";")
            if name.text in qregs or name.text in cregs:
                raise self.err(d, "DuplicateRegister", f"register `{name.text}` is declared more than once")
            if d.text == "qubit":
                if nq + size > MAX_QUBITS:
                    raise self.err(d, "TooManyQubits", f"too many qubits: declared {nq + size}, max {MAX_QUBITS}")
                qregs[name.text] = (nq, size)
                nq += size
            else:
                if nc + size > MAX_CLBITS:
                    raise self.err(d, "TooManyClbits", f"too many clbits: declared {nc + size}, max {MAX_CLBITS}")
                cregs[name.text] = (nc, size)
                nc += size
        self.qregs, self.cregs = qregs, cregs
        circ = C.Circuit(nq, num_clbits=nc)
        while self.tok.kind != "eof":
            t = self.tok
            if t.kind == "id" and t.text in ("qubit", "bit"):
                raise self.err(t, "UnsupportedFeature",
                               "unsupported feature: register declaration after gate statement")
            if t.kind != "id":
                raise self.err(t, "UnexpectedToken", f"unexpected token: expected statement, found `{t.text}`")
            if t.text == "barrier":
                self.i += 1
                qs = []
                while True:
                    qs.extend(self._reg_or_index(qubits=True))
                    if not self.accept(","):
                        break
                self.expect(";")
                circ.instructions.append(C.Barrier(tuple(qs)))
            elif t.text == "measure":
                self.i += 1
                src = self._reg_or_index_ref()
                self.expect("->")
                dst = self._reg_or_index_ref()
                self.expect(";")
                self._lower_measure(circ, t, src, dst)
            elif t.text == "reset":
                self.i += 1
                q = self._indexed(qubits=True)
                self.expect(";")
                circ.instructions.append(C.Reset(q))
            else:
                self._gate(circ)
        return circ

    def _resolve(self, name: Tok, index: int, idx_tok: Tok, qubits: bool) -> int:
        regs = self.qregs if qubits else self.cregs
        if name.text not in regs:
            raise self.err(name, "UnknownRegister", f"undeclared register `{name.text}`")
        base, size = regs[name.text]
        if index >= size:
            raise self.err(name, "IndexOutOfBounds",
                           f"index {index} out of bounds for register `{name.text}` of size {size}")
        return base + index

    def _indexed(self, qubits: bool) -> int:
        name = self.ident("register reference")
        self.expect("[")
        it = self.tok
        idx = self.uint("index")
        self.expect("]")
        return self._resolve(name, idx, it, qubits)

    def _reg_or_index_ref(self):
        name = self.ident("register reference")
        if self.accept("["):
            it = self.tok
            idx = self.uint("index")
            self.expect("]")
            return (name, idx, it)
        return (name, None, None)

    def _reg_or_index(self, qubits: bool) -> list[int]:
        name, idx, it = self._reg_or_index_ref()
        if idx is not None:
            return [self._resolve(name, idx, it, qubits)]
        regs = self.qregs if qubits else self.cregs
        if name.text not in regs:
            raise self.err(name, "UnknownRegister", f"undeclared register `{name.text}`")
        base, size = regs[name.text]
        return list(range(base, base + size))

    def _lower_measure(self, circ, stmt: Tok, src, dst) -> None:
        (qn, qi, qit), (cn, ci, cit) = src, dst
        if qi is not None and ci is not None:
            circ.instructions.append(C.Measure(self._resolve(qn, qi, qit, True), self._resolve(cn, ci, cit, False)))
            return
        if qi is None and ci is None:
            if qn.text not in self.qregs:
                raise self.err(qn, "UnknownRegister", f"undeclared register `{qn.text}`")
            if cn.text not in self.cregs:
                raise self.err(cn, "UnknownRegister", f"undeclared register `{cn.text}`")
            (qb, qs), (cb, cs) = self.qregs[qn.text], self.cregs[cn.text]
            if qs != cs:
                raise self.err(stmt, "SizeMismatch",
                               f"size mismatch: `{qn.text}` has {qs} but `{cn.text}` has {cs}")
            for k in range(qs):
                circ.instructions.append(C.Measure(qb + k, cb + k))
            return
        raise self.err(stmt, "UnsupportedFeature", "unsupported feature: mixed whole-register / indexed measure")

    def _gate(self, circ) -> None:
        name = self.ident("gate name")
        params = []
        if self.accept("("):
            if not self.accept(")"):
                while True:
                    params.append(self.expr())
                    if self.accept(")"):
                        break
                    self.expect(",", "`,` or `)`")
        qs = []
        while True:
            qs.append(self._indexed(qubits=True))
            if not self.accept(","):
                break
        self.expect(";")
        if name.text not in GATES:
            raise self.err(name, "UnknownGate", f"unknown gate `{name.text}`")
        variant, nparams = GATES[name.text]
        if len(params) != nparams:
            raise self.err(name, "UnexpectedToken", "unexpected token: expected param count match, found "
                                                    f"`{len(params)} params (expected {nparams})`")
        seen = set()
        for q in qs:
            if q in seen:
                raise self.err(name, "IrRejected", f"IR rejected this program: duplicate qubit {q}")
            seen.add(q)
        gate = C.Gate(variant, tuple(params))
        if len(qs) != gate.arity():
            raise self.err(name, "IrRejected",
                           f"IR rejected this program: {variant} takes {gate.arity()} qubits, got {len(qs)}")
        circ.instructions.append(C.GateInstance(gate, qs))


def parse(source: str) -> C.Circuit:
    """OpenQASM 3 source -> Circuit (``num_qubits`` and ``num_clbits`` from
    the declarations, in order)."""
    return _Parser(source).program()


def parse_file(path) -> C.Circuit:
    with open(path, encoding="utf-8") as f:
        return parse(f.read())


def emit(circ: C.Circuit) -> str:
    """Circuit -> OpenQASM 3 (one ``q`` and, with measurements, one ``c``
    register): the stdgates subset above, parameters as round-trip float
    literals. Other gate kinds raise ValueError."""
    lines = ["OPENQASM 3.0;", 'include "stdgates.inc";', f"qubit[{circ.num_qubits}] q;"]
    nc = getattr(circ, "num_clbits", 0) or 0
    for inst in circ.instructions:
        if isinstance(inst, C.Measure):
            nc = max(nc, inst.clbit + 1)
    if nc:
        lines.append(f"bit[{nc}] c;")
    for inst in circ.instructions:
        if isinstance(inst, C.GateInstance):
            if inst.controls or inst.gate.name not in GATE_NAMES:
                raise ValueError(f"gate {inst.gate.name} has no OpenQASM 3 standard-subset representation")
            ps = inst.gate.params
            if any(not math.isfinite(p) for p in ps):
                raise ValueError("non-finite parameter cannot be emitted")
            pstr = f"({', '.join(repr(float(p)) for p in ps)})" if ps else ""
            lines.append(f"{GATE_NAMES[inst.gate.name]}{pstr} " + ", ".join(f"q[{q}]" for q in inst.qubits) + ";")
        elif isinstance(inst, C.Measure):
            lines.append(f"measure q[{inst.qubit}] -> c[{inst.clbit}];")
        elif isinstance(inst, C.Barrier):
            args = ", ".join(f"q[{q}]" for q in inst.qubits) if inst.qubits else "q"
            lines.append(f"barrier {args};")
        elif isinstance(inst, C.Reset):
            lines.append(f"reset q[{inst.qubit}];")
        else:
            raise ValueError(f"{type(inst).__name__} has no OpenQASM 3 standard-subset representation")
    return "\n".join(lines) + "\n"
