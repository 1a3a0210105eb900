"""OpenQASM 2.0 front end: read and write circuits as text.

The reference ships its benchmark circuits as OpenQASM 2.0 files (circuits/qasm/*.qasm, written by
circuits/generators.py) and loads them through Qiskit. This reader needs no Qiskit: it covers the
OpenQASM 2.0 statements those files and typical qelib1 circuits use --

  OPENQASM 2.0;  include "qelib1.inc";  qreg / creg declarations (several registers are laid out one after
  another in declaration order);  gate applications with parameter expressions (pi, + - * / ^, unary
  minus, parentheses, sin cos tan exp ln sqrt);  whole-register arguments (broadcast);  user gate
  definitions (gate name(params) args { body }, expanded in place);  barrier and measure (kept as such;
  the runtime drops final measurements);  opaque and reset are rejected.

Gate names are the qelib1 names, which are also this package's Circuit names (u3 and U become u, u2(a, b)
becomes u(pi/2, a, b), u1 becomes p); anything else must be defined in the file with a gate block.
"""
import ast
import math
import operator
import re

from .circuit import Circuit

# qelib1 gates understood natively: name -> (number of parameters, number of qubits)
_NATIVE = {
    "id": (0, 1), "x": (0, 1), "y": (0, 1), "z": (0, 1), "h": (0, 1), "s": (0, 1), "sdg": (0, 1),
    "t": (0, 1), "tdg": (0, 1), "sx": (0, 1), "sxdg": (0, 1),
    "rx": (1, 1), "ry": (1, 1), "rz": (1, 1), "p": (1, 1), "u1": (1, 1), "u2": (2, 1), "u3": (3, 1),
    "u": (3, 1), "U": (3, 1), "r": (2, 1),
    "cx": (0, 2), "CX": (0, 2), "cy": (0, 2), "cz": (0, 2), "ch": (0, 2), "csx": (0, 2), "swap": (0, 2),
    "iswap": (0, 2), "ecr": (0, 2), "dcx": (0, 2), "cs": (0, 2), "csdg": (0, 2),
    "cp": (1, 2), "cu1": (1, 2), "crx": (1, 2), "cry": (1, 2), "crz": (1, 2), "cu3": (3, 2), "cu": (4, 2),
    "rxx": (1, 2), "ryy": (1, 2), "rzz": (1, 2), "rzx": (1, 2),
    "ccx": (0, 3), "ccz": (0, 3), "cswap": (0, 3), "c3x": (0, 4), "c4x": (0, 5),
    "rccx": (0, 3), "rc3x": (0, 4), "c3sqrtx": (0, 4),
}
# qelib1 names -> this package's (Qiskit's) names, and back for export
_RENAME = {"u3": "u", "U": "u", "u1": "p", "CX": "cx", "rc3x": "rcccx", "c3sqrtx": "c3sx"}
_EXPORT = {"u": "u3", "rcccx": "rc3x", "c3sx": "c3sqrtx"}

_BINOPS = {ast.Add: operator.add, ast.Sub: operator.sub, ast.Mult: operator.mul, ast.Div: operator.truediv,
           ast.Pow: operator.pow}
_FUNCS = {"sin": math.sin, "cos": math.cos, "tan": math.tan, "exp": math.exp, "ln": math.log, "sqrt": math.sqrt}


class QasmError(ValueError):
    pass


def _eval(expr, env):
    """Value of an OpenQASM parameter expression (no names other than pi, gate parameters and the
    functions above)."""
    try:
        # OpenQASM's ^ is exponentiation, binding tighter than unary minus: Python's **
        node = ast.parse(expr.strip().replace("^", "**"), mode="eval").body
    except SyntaxError as e:
        raise QasmError(f"bad expression {expr!r}") from e

    def ev(n):
        if isinstance(n, ast.Constant) and isinstance(n.value, (int, float)):
            return float(n.value)
        if isinstance(n, ast.Name):
            if n.id == "pi":
                return math.pi
            if n.id in env:
                return env[n.id]
            raise QasmError(f"unknown name {n.id!r} in {expr!r}")
        if isinstance(n, ast.UnaryOp) and isinstance(n.op, (ast.USub, ast.UAdd)):
            v = ev(n.operand)
            return -v if isinstance(n.op, ast.USub) else v
        if isinstance(n, ast.BinOp) and type(n.op) in _BINOPS:
            return _BINOPS[type(n.op)](ev(n.left), ev(n.right))
        if isinstance(n, ast.Call) and isinstance(n.func, ast.Name) and n.func.id in _FUNCS and len(n.args) == 1:
            return _FUNCS[n.func.id](ev(n.args[0]))
        raise QasmError(f"unsupported expression {expr!r}")

    return ev(node)


def _split_args(s):
    """Split a comma-separated list at the top level (commas inside parentheses stay)."""
    out, depth, cur = [], 0, []
    for ch in s:
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        if ch == "," and depth == 0:
            out.append("".join(cur).strip())
            cur = []
        else:
            cur.append(ch)
    if "".join(cur).strip():
        out.append("".join(cur).strip())
    return out


_APPLY = re.compile(r"^([A-Za-z_][A-Za-z0-9_]*)\s*(\((.*)\))?\s*(.*)$", re.S)


def from_qasm(text, name="qasm"):
    """Circuit of an OpenQASM 2.0 program (a string, or a path ending in .qasm)."""
    if "\n" not in text and text.endswith(".qasm"):
        name = text.rsplit("/", 1)[-1][:-5]
        with open(text) as f:
            text = f.read()
    text = re.sub(r"//[^\n]*", "", text)
    # gate definitions: name(params) args { body }
    defs = {}
    for m in re.finditer(r"gate\s+([A-Za-z_][A-Za-z0-9_]*)\s*(\(([^)]*)\))?\s*([^{]*)\{([^}]*)\}", text):
        params = [p.strip() for p in (m.group(3) or "").split(",") if p.strip()]
        args = [a.strip() for a in m.group(4).split(",") if a.strip()]
        defs[m.group(1)] = (params, args, [st.strip() for st in m.group(5).split(";") if st.strip()])
    text = re.sub(r"gate\s+[A-Za-z_][A-Za-z0-9_]*\s*(\([^)]*\))?\s*[^{]*\{[^}]*\}", "", text)
    stmts = [s.strip() for s in text.split(";") if s.strip()]
    regs, nq = {}, 0
    body = []
    for st in stmts:
        if st.startswith("OPENQASM"):
            if not st.split()[1].startswith("2"):
                raise QasmError(f"only OpenQASM 2 is read, not {st!r}")
        elif st.startswith("include"):
            continue
        elif st.startswith("qreg"):
            m = re.match(r"qreg\s+([A-Za-z_][A-Za-z0-9_]*)\s*\[\s*(\d+)\s*\]$", st)
            if not m:
                raise QasmError(f"bad declaration {st!r}")
            regs[m.group(1)] = (nq, int(m.group(2)))
            nq += int(m.group(2))
        elif st.startswith("creg"):
            continue
        elif st.startswith(("opaque", "reset", "if")):
            raise QasmError(f"unsupported statement {st!r}")
        else:
            body.append(st)
    qc = Circuit(nq, name=name)

    def qubits_of(arg):
        m = re.match(r"([A-Za-z_][A-Za-z0-9_]*)\s*(\[\s*(\d+)\s*\])?$", arg)
        if not m or m.group(1) not in regs:
            raise QasmError(f"unknown qubit argument {arg!r}")
        base, size = regs[m.group(1)]
        if m.group(3) is None:
            return list(range(base, base + size))
        i = int(m.group(3))
        if i >= size:
            raise QasmError(f"{arg!r} is outside its register of {size}")
        return [base + i]

    def apply(gname, params, qubits, depth=0):
        if depth > 32:
            raise QasmError("gate definitions nest too deeply")
        if gname in defs:
            pnames, anames, stmts_ = defs[gname]
            if len(pnames) != len(params) or len(anames) != len(qubits):
                raise QasmError(f"gate {gname} takes {len(pnames)} parameters and {len(anames)} qubits")
            env = dict(zip(pnames, params))
            amap = dict(zip(anames, qubits))
            for s in stmts_:
                m = _APPLY.match(s)
                sub = [_eval(e, env) for e in _split_args(m.group(3))] if m.group(2) else []
                qa = [amap[a.strip()] for a in _split_args(m.group(4))]
                if m.group(1) == "barrier":
                    continue
                apply(m.group(1), sub, qa, depth + 1)
            return
        if gname not in _NATIVE:
            raise QasmError(f"unknown gate {gname!r}")
        npar, nqb = _NATIVE[gname]
        if len(params) != npar or len(qubits) != nqb:
            raise QasmError(f"{gname} takes {npar} parameters and {nqb} qubits, got {len(params)} and {len(qubits)}")
        if gname == "u2":
            qc.append("u", qubits, (math.pi / 2, params[0], params[1]))
            return
        qc.append(_RENAME.get(gname, gname), qubits, params)

    for st in body:
        m = _APPLY.match(st)
        if not m:
            raise QasmError(f"cannot read {st!r}")
        gname = m.group(1)
        if gname == "measure":
            for q in qubits_of(st.split()[1].split("->")[0].strip()):
                qc.append("measure", (q,))
            continue
        params = [_eval(e, {}) for e in _split_args(m.group(3))] if m.group(2) else []
        args = [qubits_of(a) for a in _split_args(m.group(4))]
        if gname == "barrier":
            qc.append("barrier", tuple(q for a in args for q in a))
            continue
        width = max(len(a) for a in args) if args else 0
        if any(len(a) not in (1, width) for a in args):
            raise QasmError(f"register arguments of different sizes in {st!r}")
        for i in range(width):            # broadcast over whole-register arguments
            apply(gname, params, [a[0] if len(a) == 1 else a[i] for a in args])
    return qc


def to_qasm(qc):
    """OpenQASM 2.0 text of a Circuit (one register q; parameters printed exactly, repr of the float)."""
    lines = ["OPENQASM 2.0;", 'include "qelib1.inc";', f"qreg q[{qc.num_qubits}];"]
    for ins in qc.data:
        name = ins.name
        if name in ("mcx", "mcp"):
            raise QasmError(f"{name} has no qelib1 form; decompose it first")
        qs = ",".join(f"q[{q}]" for q in ins.qubits)
        if name == "measure":
            continue
        if name == "barrier":
            lines.append(f"barrier {qs};")
            continue
        ps = "(" + ",".join(repr(float(p)) for p in ins.params) + ")" if ins.params else ""
        lines.append(f"{_EXPORT.get(name, name)}{ps} {qs};")
    return "\n".join(lines) + "\n"
