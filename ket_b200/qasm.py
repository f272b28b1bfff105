"""OpenQASM 2.0 subset: ket's ``from_qasm`` / ``to_qasm`` for the Python mirror.

ket reads and writes a subset of OpenQASM 2.0 (bindings/qasm/qasm.cpp,
declared in include/ket/qasm.hpp:16-20).  This module accepts the same
programs, builds the same circuits and writes the same text:

* statements end at ``;`` outside braces; ``//`` and ``/* */`` comments are
  dropped (qasm.cpp:71-87, 234-258);
* ``qreg`` / ``creg`` declarations share one flat index space per kind, in
  declaration order; ``OPENQASM`` and ``include`` lines are skipped
  (qasm.cpp:165-215, 484-510);
* angle arguments are expressions of numbers, ``pi`` and the parameters of
  the enclosing gate definition with ``+ - * /``, unary signs and
  parentheses (qasm.cpp:89-163);
* gates: h x y z s sdg t tdg id, ch cx cy cz swap ccx cswap, rx ry rz, crx cry
  crz, cp/cu1, cu3/cu (3 angles), U/u/u3, u2(phi, lambda) = U(pi/2, phi,
  lambda), u1/p/phase(lambda) = U(0, 0, lambda), ``measure a -> b``,
  ``barrier`` (whole registers allowed) and user ``gate`` definitions, whose
  calls are appended as composite blocks named after the gate; the first
  definition of a name wins (qasm.cpp:318-477, 512-541);
* ``opaque`` and ``if`` are rejected.

Errors raise ``RuntimeError`` with ket's ``"qasm: ..."`` messages (pybind11
maps ket's std::runtime_error to RuntimeError); a repeated operand or an
index that does not parse as a number raises ``ValueError`` as in ket.

``to_qasm`` writes ket's format (qasm.cpp:546-780): angles that are small
rational multiples of pi as ``k*pi/d`` (d <= 12), others with 15 significant
digits; composite blocks as ``gate`` definitions emitted once per distinct
body, nested ones first, a repeated name with a different body suffixed
``_2``, ``_3``, ...; probes are dropped.
"""
from __future__ import annotations

import math
import re
from typing import Callable, Dict, List, Optional, Sequence, Tuple

from .circuit import Circuit, Gate, GateType

__all__ = ["from_qasm", "to_qasm"]

_SPACE = " \t\n\v\f\r"  # C isspace in the "C" locale


def _fail(msg: str):
    raise RuntimeError("qasm: " + msg)


def _trim(s: str) -> str:
    return s.strip(_SPACE)


def _ident_char(ch: str) -> bool:
    return ch.isascii() and (ch.isalnum() or ch == "_")


def _head(s: str) -> str:
    """The leading identifier of a statement (a keyword or gate name)."""
    i = 0
    while i < len(s) and _ident_char(s[i]):
        i += 1
    return s[:i]


def _pieces(s: str, delim: str) -> List[str]:
    """Split on ``delim``, trim each piece, drop the empty ones."""
    return [t for t in (_trim(x) for x in s.split(delim)) if t]


_COMMENT = re.compile(r"//[^\n]*|/\*.*?(?:\*/|\Z)", re.S)


def _strip_comments(src: str) -> str:
    # a line comment keeps its newline; a block comment (or an unterminated
    # one, to the end of the text) disappears
    return _COMMENT.sub("", src)


def _statements(src: str) -> List[str]:
    """Top-level statements: ``;`` at brace depth 0 ends one, and so does the
    ``}`` that closes a gate body."""
    out, cur, depth = [], [], 0

    def flush():
        t = _trim("".join(cur))
        if t:
            out.append(t)
        cur.clear()

    for ch in src:
        if ch == "{":
            depth += 1
            cur.append(ch)
        elif ch == "}":
            if depth > 0:
                depth -= 1
            cur.append(ch)
            if depth == 0:
                flush()
        elif ch == ";" and depth == 0:
            flush()
        else:
            cur.append(ch)
    flush()
    return out


def _stoul(text: str) -> int:
    """std::stoul on an already trimmed string: the leading decimal digits,
    a minus sign wrapping modulo 2^64 as strtoul does."""
    m = re.match(r"[" + re.escape(_SPACE) + r"]*([+-]?)([0-9]+)", text)
    if not m:
        raise ValueError("stoul")
    v = int(m.group(2))
    if v >= 1 << 64:
        raise IndexError("stoul")  # out of range (std::out_of_range)
    return (-v) % (1 << 64) if m.group(1) == "-" else v


# ---------------------------------------------------------------- angles

_HEX = re.compile(r"0[xX](?:[0-9a-fA-F]+\.?[0-9a-fA-F]*|\.[0-9a-fA-F]+)(?:[pP][+-]?[0-9]+)?")
_DEC = re.compile(r"(?:[0-9]+\.?[0-9]*|\.[0-9]+)(?:[eE][+-]?[0-9]+)?")
_DBL_MIN = 2.2250738585072014e-308


def _number_prefix(s: str, pos: int) -> Optional[Tuple[float, int]]:
    """The longest number std::stod reads at ``pos`` (decimal or hex), as
    (value, length); None where stod would throw, out-of-range results
    included."""
    m = _HEX.match(s, pos)
    if m:
        text = m.group(0)
        mant = text[2:].split("p")[0].split("P")[0]
        v = float.fromhex(text if "p" in text or "P" in text else text + "p0")
        nonzero = any(c not in "0." for c in mant)
    else:
        m = _DEC.match(s, pos)
        if not m:
            return None
        text = m.group(0)
        v = float(text)
        nonzero = any(c in "123456789" for c in re.split(r"[eE]", text)[0])
    if math.isinf(v) or (nonzero and abs(v) < _DBL_MIN):
        return None  # ERANGE: stod throws out_of_range
    return v, len(text)


def _fdiv(a: float, b: float) -> float:
    try:
        return a / b
    except ZeroDivisionError:  # IEEE 754 division, as the C++ parser does it
        if math.isnan(a):
            return a
        if a == 0.0:
            return math.inf - math.inf  # the hardware's default NaN, as 0.0/0.0
        return math.copysign(math.inf, a) * math.copysign(1.0, b)


class _Angle:
    """Recursive-descent evaluation of one angle expression:
    expr = term {(+|-) term}; term = factor {(*|/) factor};
    factor = (+|-) factor | ( expr ) | identifier | number."""

    def __init__(self, text: str, syms: Optional[Dict[str, float]]):
        self.s = text
        self.syms = syms
        self.pos = 0

    def _skip(self):
        while self.pos < len(self.s) and self.s[self.pos] in _SPACE:
            self.pos += 1

    def _eat(self, ch: str) -> bool:
        self._skip()
        if self.pos < len(self.s) and self.s[self.pos] == ch:
            self.pos += 1
            return True
        return False

    def value(self) -> float:
        v = self._expr()
        self._skip()
        if self.pos != len(self.s):
            _fail("bad angle expression: " + self.s)
        return v

    def _expr(self) -> float:
        v = self._term()
        while True:
            if self._eat("+"):
                v += self._term()
            elif self._eat("-"):
                v -= self._term()
            else:
                return v

    def _term(self) -> float:
        v = self._factor()
        while True:
            if self._eat("*"):
                v *= self._factor()
            elif self._eat("/"):
                v = _fdiv(v, self._factor())
            else:
                return v

    def _factor(self) -> float:
        self._skip()
        if self._eat("+"):
            return self._factor()
        if self._eat("-"):
            return -self._factor()
        if self._eat("("):
            v = self._expr()
            if not self._eat(")"):
                _fail("missing ')' in angle: " + self.s)
            return v
        s, p = self.s, self.pos
        if p < len(s) and s[p].isascii() and (s[p].isalpha() or s[p] == "_"):
            e = p
            while e < len(s) and _ident_char(s[e]):
                e += 1
            self.pos = e
            name = s[p:e]
            if name == "pi":
                return math.pi
            if self.syms is not None and name in self.syms:
                return self.syms[name]
            _fail("unknown identifier in angle: " + name)
        got = _number_prefix(s, p)
        if got is None:
            _fail("bad angle: " + s)
        self.pos = p + got[1]
        return got[0]


def _angle(text: str, syms: Dict[str, float]) -> float:
    if not _trim(text):
        _fail("missing angle parameter")
    return _Angle(text, syms).value()


# ---------------------------------------------------------------- registers

class _Registers:
    """Registers of one kind in one flat index space, by declaration order."""

    def __init__(self):
        self.entries: Dict[str, Tuple[int, int]] = {}
        self.total = 0

    def declare(self, name: str, size: int):
        self.entries[name] = (self.total, size)
        self.total += size

    def lookup(self, name: str) -> Tuple[int, int]:
        if name not in self.entries:
            _fail("unknown register: " + name)
        return self.entries[name]

    def index(self, token: str) -> int:
        """``name[i]`` -> flat index."""
        lb, rb = token.find("["), token.find("]")
        if lb < 0 or rb < 0 or rb < lb:
            _fail("expected indexed register, got: " + token)
        i = _stoul(_trim(token[lb + 1:rb]))
        offset, size = self.lookup(_trim(token[:lb]))
        if i >= size:
            _fail("index out of range: " + token)
        return offset + i


def _declare(stmt: str, keyword: str, regs: _Registers):
    rest = _trim(stmt[len(keyword):])
    lb, rb = rest.find("["), rest.find("]")
    if lb < 0 or rb < 0:
        _fail("malformed declaration: " + stmt)
    regs.declare(_trim(rest[:lb]), _stoul(_trim(rest[lb + 1:rb])))


# ---------------------------------------------------------------- gates

class _GateDef:
    __slots__ = ("params", "qubits", "body")

    def __init__(self, params, qubits, body):
        self.params, self.qubits, self.body = params, qubits, body


def _gate_def(stmt: str) -> Tuple[str, _GateDef]:
    """``gate name(p, ...) a, b { body }``."""
    i = len(_head(stmt))
    while i < len(stmt) and stmt[i] in _SPACE:
        i += 1
    j = i
    while j < len(stmt) and _ident_char(stmt[j]):
        j += 1
    name = stmt[i:j]
    if not name:
        _fail("gate: missing name")
    i = j
    while i < len(stmt) and stmt[i] in _SPACE:
        i += 1
    params: List[str] = []
    if i < len(stmt) and stmt[i] == "(":
        close = stmt.find(")", i)
        if close < 0:
            _fail("gate: missing ')' in " + name)
        params = _pieces(stmt[i + 1:close], ",")
        i = close + 1
    brace = stmt.find("{", i)
    if brace < 0:
        _fail("gate: missing '{' in " + name)
    qubits = _pieces(stmt[i:brace], ",")
    if not qubits:
        _fail("gate: " + name + " has no qubit arguments")
    end = stmt.rfind("}")
    if end < 0 or end < brace:
        _fail("gate: missing '}' in " + name)
    return name, _GateDef(params, qubits, _pieces(stmt[brace + 1:end], ";"))


# name -> number of qubits, for the gates without angles
_FIXED = {"h": 1, "x": 1, "y": 1, "z": 1, "s": 1, "sdg": 1, "t": 1, "tdg": 1, "id": 1,
          "ch": 2, "cx": 2, "cy": 2, "cz": 2, "swap": 2, "ccx": 3, "cswap": 3}
# name -> (qubits, Circuit method) for the gates with one angle expression
_ONE_ANGLE = {"rx": (1, "rx"), "ry": (1, "ry"), "rz": (1, "rz"), "crx": (2, "crx"), "cry": (2, "cry"),
              "crz": (2, "crz"), "cp": (2, "cp"), "cu1": (2, "cp")}


def _apply(c: Circuit, stmt: str, qubit: Callable[[str], int], syms: Dict[str, float],
           defs: Dict[str, _GateDef]):
    """Append one gate statement (a built-in gate or a user gate call) to c."""
    name = _head(stmt)
    i = len(name)
    while i < len(stmt) and stmt[i] in _SPACE:
        i += 1
    params = ""
    if i < len(stmt) and stmt[i] == "(":
        close = stmt.find(")", i)
        if close < 0:
            _fail("missing ')' in: " + stmt)
        params = stmt[i + 1:close]
        i = close + 1
    q = [qubit(a) for a in _pieces(_trim(stmt[i:]), ",")]

    def need(n):
        if len(q) != n:
            _fail(f"{name}: expected {n} qubits")

    def angles(count, what):
        a = [_angle(p, syms) for p in _pieces(params, ",")]
        if len(a) != count:
            _fail(what)
        return a

    if name in _FIXED:
        need(_FIXED[name])
        if name != "id":
            getattr(c, name)(*q)
    elif name in _ONE_ANGLE:
        nq, method = _ONE_ANGLE[name]
        need(nq)
        getattr(c, method)(*q, _angle(params, syms))
    elif name in ("cu3", "cu"):
        a = angles(3, name + ": expected 3 angles")
        need(2)
        c.cu(q[0], q[1], *a)
    elif name in ("U", "u", "u3"):
        a = angles(3, name + ": expected 3 angles")
        need(1)
        c.u(q[0], *a)
    elif name == "u2":
        a = angles(2, "u2: expected 2 angles")
        need(1)
        c.u(q[0], math.pi / 2.0, a[0], a[1])
    elif name in ("u1", "p", "phase"):
        a = angles(1, name + ": expected 1 angle")
        need(1)
        c.u(q[0], 0.0, 0.0, a[0])
    else:
        d = defs.get(name)
        if d is None:
            _fail("unsupported gate: " + name)
        a = [] if not params else [_angle(p, syms) for p in _pieces(params, ",")]
        if len(a) != len(d.params):
            _fail(f"{name}: expected {len(d.params)} parameters")
        if len(q) != len(d.qubits):
            _fail(f"{name}: expected {len(d.qubits)} qubits")
        c.append(_instantiate(name, d, a, defs), q, name)


def _instantiate(name: str, d: _GateDef, args: Sequence[float], defs: Dict[str, _GateDef]) -> Circuit:
    """The body of a user gate as a circuit on its formal qubits 0..n-1."""
    sub = Circuit(len(d.qubits), name)
    formal = {}
    for k, qn in enumerate(d.qubits):
        formal[qn] = k

    def qubit(tok: str) -> int:
        t = _trim(tok)
        if t not in formal:
            _fail(name + ": unknown qubit " + tok)
        return formal[t]

    syms = dict(zip(d.params, args))
    for stmt in d.body:
        _apply(sub, stmt, qubit, syms, defs)
    return sub


def from_qasm(source: str) -> Circuit:
    """ket.from_qasm (include/ket/qasm.hpp:16, qasm.cpp:479): parse an
    OpenQASM 2.0 program into a Circuit."""
    stmts = _statements(_strip_comments(source))
    qreg, creg = _Registers(), _Registers()
    defs: Dict[str, _GateDef] = {}
    # declarations and gate definitions first, so sizes and gates are known
    for st in stmts:
        head = _head(st)
        if head == "qreg":
            _declare(st, "qreg", qreg)
        elif head == "creg":
            _declare(st, "creg", creg)
        elif head == "gate":
            name, d = _gate_def(st)
            defs.setdefault(name, d)
    if qreg.total >= 1 << 63:  # a wrapped negative size: ket's vector allocation refuses it
        raise ValueError("cannot create std::vector larger than max_size()")
    c = Circuit(qreg.total)
    for st in stmts:
        head = _head(st)
        if head in ("OPENQASM", "include", "qreg", "creg", "gate"):
            continue
        if head in ("opaque", "if"):
            _fail("unsupported construct: " + head)
        if head == "measure":
            arrow = st.find("->")
            if arrow < 0:
                _fail("measure needs '->': " + st)
            c.measure(qreg.index(_trim(st[7:arrow])), creg.index(_trim(st[arrow + 2:])))
        elif head == "barrier":
            qs: List[int] = []
            for arg in _pieces(_trim(st[7:]), ","):
                if "[" not in arg:
                    offset, size = qreg.lookup(arg)
                    qs.extend(range(offset, offset + size))
                else:
                    qs.append(qreg.index(arg))
            c.barrier(qs)
        else:
            _apply(c, st, qreg.index, {}, defs)
    return c


# ---------------------------------------------------------------- writer

def _angle_text(a: float) -> str:
    """pi multiples k*pi/d (d <= 12) exactly, other angles to 15 digits."""
    if abs(a) < 1e-12:
        return "0"
    ratio = a / math.pi
    for den in range(1, 13):
        scaled = ratio * den
        if not abs(scaled) < 2.0 ** 63:
            break
        num = int(math.copysign(math.floor(abs(scaled) + 0.5), scaled))  # round half away
        if num != 0 and abs(scaled - num) < 1e-9:
            mag = abs(num)
            t = "pi" if mag == 1 else f"{mag}*pi"
            if den != 1:
                t += f"/{den}"
            return "-" + t if num < 0 else t
    if math.isnan(a):  # C's printf shows the sign of a NaN
        return "-nan" if math.copysign(1.0, a) < 0 else "nan"
    return "%.15g" % a


_NAMED = {GateType.H: "h", GateType.X: "x", GateType.Y: "y", GateType.Z: "z", GateType.S: "s",
          GateType.Sdg: "sdg", GateType.T: "t", GateType.Tdg: "tdg", GateType.CH: "ch", GateType.CX: "cx",
          GateType.CY: "cy", GateType.CZ: "cz", GateType.Swap: "swap", GateType.CCX: "ccx",
          GateType.CSwap: "cswap", GateType.Rx: "rx", GateType.Ry: "ry", GateType.Rz: "rz",
          GateType.CRx: "crx", GateType.CRy: "cry", GateType.CRz: "crz", GateType.CP: "cp"}


class _Blocks:
    """``gate`` definitions for composite blocks: one per distinct (name,
    width, body), nested definitions written before their users."""

    def __init__(self):
        self.text: List[str] = []
        self.by_key: Dict[str, str] = {}
        self.names = set()

    def name_of(self, sub: Circuit, wanted: str) -> str:
        body = "".join(_gate_line(g, lambda i: f"q{i}", self) for g in sub.gates)
        key = f"{wanted}#{sub.n_qubits}\x1f{body}"
        if key in self.by_key:
            return self.by_key[key]
        name = wanted or "block"
        if name in self.names:
            k = 2
            while f"{name}_{k}" in self.names:
                k += 1
            name = f"{name}_{k}"
        self.names.add(name)
        self.by_key[key] = name
        head = "gate " + name + "".join((" " if i == 0 else ",") + f"q{i}" for i in range(sub.n_qubits))
        lines = [head + " {\n"] + ["  " + ln + "\n" for ln in body.split("\n") if ln] + ["}\n"]
        self.text.append("".join(lines))
        return name


def _gate_line(g: Gate, ref: Callable[[int], str], blocks: _Blocks) -> str:
    t = g.type
    qs = ",".join(ref(q) for q in g.qubits)
    if t in (GateType.Rx, GateType.Ry, GateType.Rz, GateType.CRx, GateType.CRy, GateType.CRz, GateType.CP):
        return f"{_NAMED[t]}({_angle_text(g.params[0])}) {qs};\n"
    if t in _NAMED:
        return f"{_NAMED[t]} {qs};\n"
    if t == GateType.U:
        return "U(" + ",".join(_angle_text(p) for p in g.params[:3]) + f") {qs};\n"
    if t == GateType.CU:  # the 3-parameter qelib1 spelling
        return "cu3(" + ",".join(_angle_text(p) for p in g.params[:3]) + f") {qs};\n"
    if t == GateType.Measure:
        return f"measure {ref(g.qubits[0])} -> c[{g.clbit}];\n"
    if t == GateType.Barrier:
        return f"barrier {qs};\n"
    if t == GateType.Composite:
        if g.definition is None:
            return ""
        name = blocks.name_of(g.definition, g.label)
        return name + "".join((" " if k == 0 else ",") + ref(q) for k, q in enumerate(g.qubits)) + ";\n"
    return ""  # Probe: no OpenQASM form


def to_qasm(circuit: Circuit) -> str:
    """ket.to_qasm (include/ket/qasm.hpp:20, qasm.cpp:764): the circuit as an
    OpenQASM 2.0 program that from_qasm reads back."""
    blocks = _Blocks()
    body = "".join(_gate_line(g, lambda i: f"q[{i}]", blocks) for g in circuit.gates)
    out = ['OPENQASM 2.0;\ninclude "qelib1.inc";\n', "".join(blocks.text), f"qreg q[{circuit.n_qubits}];\n"]
    if circuit.n_clbits > 0:
        out.append(f"creg c[{circuit.n_clbits}];\n")
    out.append(body)
    return "".join(out)
