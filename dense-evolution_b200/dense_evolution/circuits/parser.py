"""OpenQASM 2/3 front end with the behaviour of the reference's
``dense_evolution/circuits/parser.py:13-695`` (host code, not on the device path).

Pipeline of ``QASMParser.parse``:
comments stripped -> ``gate`` definitions lifted out -> ``for`` loops with
integer bounds unrolled (inclusive end), ``if``/``while``/``def`` blocks and
unresolvable loops dropped -> statements split on ``;`` -> calls of defined
gates expanded recursively -> declarations (qreg/creg, qubit/bit) and gate
applications.  Parameters are evaluated by an AST whitelist (numbers, + - * /
** %, unary +/-, the constants pi/tau/euler and a fixed set of functions);
anything else raises ValueError.  Qubit arguments: ``q[i]``, bare ``q``
(= q[0]), ``q[a:b]`` (exclusive), bare integers.  Single-qubit gates given
several qubits are expanded into one op per qubit.
"""
from __future__ import annotations

import ast
import operator
import re
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np

__all__ = ['QASMCircuit', 'QASMParser']


@dataclass
class QASMCircuit:
    """n_qubits / n_cbits declared or inferred; ops = [{'type': 'gate', 'name',
    'qubits': [int], 'params': [float]}]."""
    n_qubits: int = 0
    n_cbits: int = 0
    ops: List[Dict] = field(default_factory=list)

    def to_tuples(self) -> List[Tuple]:
        """(name, *qubits, *params) per op -- the run_circuit tuple format."""
        return [(op['name'], *op['qubits'], *op['params']) for op in self.ops]

    def __iter__(self):
        return iter(self.to_tuples())


_ALIAS = {'cu1': 'cp', 'u1': 'p', 'toffoli': 'ccx', 'fredkin': 'cswap', 'cnot': 'cx', 'not': 'x', 'id': 'i'}
_SINGLE_QUBIT = frozenset(('h', 'x', 'y', 'z', 's', 'sdg', 't', 'tdg', 'sx', 'id', 'rx', 'ry', 'rz', 'p', 'u1',
                           'u2', 'u3'))
_SKIP = frozenset(('openqasm', 'include', 'barrier', 'measure', 'reset', 'gate', 'def', 'if', 'for', 'while'))
_ENV = {
    'pi': np.pi, 'tau': 2.0 * np.pi, 'euler': np.e,
    'sin': np.sin, 'cos': np.cos, 'tan': np.tan, 'sqrt': np.sqrt, 'exp': np.exp, 'log': np.log,
    'asin': np.arcsin, 'acos': np.arccos, 'atan': np.arctan,
    'arcsin': np.arcsin, 'arccos': np.arccos, 'arctan': np.arctan,
    'abs': abs, 'round': round,
}
_BIN = {ast.Add: operator.add, ast.Sub: operator.sub, ast.Mult: operator.mul, ast.Div: operator.truediv,
        ast.Pow: operator.pow, ast.Mod: operator.mod}
_UN = {ast.UAdd: operator.pos, ast.USub: operator.neg}

_BLOCK_CMT = re.compile(r'/\*.*?\*/', re.DOTALL)
_LINE_CMT = re.compile(r'//[^\n]*')
_BLOCK_HEAD = re.compile(r'\b(for|if|while|def|gate)\b[^{]*\{')
_FOR_HEAD = re.compile(r'for\s+(?:\w+\s+)?(\w+)\s+in\s*\[\s*([^\]]+?)\s*:\s*([^\]]+?)\s*\]\s*\{')
_INT_DECL = re.compile(r'(?:const\s+)?int(?:\s*\[\d+\])?\s+(\w+)\s*=\s*(-?\d+)\s*;')
_GATE_DEF = re.compile(r'\bgate\s+([a-zA-Z_]\w*)\s*(?:\(([^)]*)\))?\s*([^{]*)\{')
_QREG2 = re.compile(r'^qreg\s+([a-zA-Z_]\w*)\s*\[(\d+)\]')
_CREG2 = re.compile(r'^creg\s+([a-zA-Z_]\w*)\s*\[(\d+)\]')
_QREG3 = re.compile(r'^qubit(?:\s*\[(\d+)\])?\s+([a-zA-Z_]\w*)')
_CREG3 = re.compile(r'^bit(?:\s*\[(\d+)\])?\s+([a-zA-Z_]\w*)')
_RANGE = re.compile(r'^([a-zA-Z_]\w*)\[(\d+):(\d+)\]$')
_INDEX = re.compile(r'\[(\d+)\]')
_WS = re.compile(r'\s+')


def _eval(node, env):
    if isinstance(node, ast.Expression):
        return _eval(node.body, env)
    if isinstance(node, ast.Constant) and isinstance(node.value, (int, float)):
        return node.value
    if isinstance(node, ast.BinOp) and type(node.op) in _BIN:
        return _BIN[type(node.op)](_eval(node.left, env), _eval(node.right, env))
    if isinstance(node, ast.UnaryOp) and type(node.op) in _UN:
        return _UN[type(node.op)](_eval(node.operand, env))
    if isinstance(node, ast.Name) and node.id in env and not callable(env[node.id]):
        return env[node.id]
    if (isinstance(node, ast.Call) and isinstance(node.func, ast.Name) and node.func.id in env
            and callable(env[node.func.id]) and not node.keywords):
        return env[node.func.id](*[_eval(a, env) for a in node.args])
    raise ValueError(f"disallowed expression node: {type(node).__name__}")


def _matching_brace(s: str, i: int) -> Optional[int]:
    depth = 0
    for k in range(i, len(s)):
        ch = s[k]
        if ch == '{':
            depth += 1
        elif ch == '}':
            depth -= 1
            if depth == 0:
                return k
    return None


def _split_params(s: str) -> List[str]:
    out, cur, depth = [], [], 0
    for ch in s:
        if ch == ',' and depth == 0:
            out.append(''.join(cur).strip())
            cur = []
            continue
        depth += (ch == '(') - (ch == ')')
        cur.append(ch)
    if cur:
        out.append(''.join(cur).strip())
    return [t for t in out if t]


class QASMParser:
    """OpenQASM 2.0 / 3.0 parser producing :class:`QASMCircuit`."""

    _ALIAS = _ALIAS
    _SINGLE_QUBIT_GATES = _SINGLE_QUBIT
    _SKIP = _SKIP
    _MATH_ENV = _ENV

    # ------------------------------------------------------------ preprocessing
    @staticmethod
    def _int_expr(expr: str, decls: Dict[str, int]) -> Optional[int]:
        expr = expr.strip()
        for name, val in decls.items():
            expr = re.sub(r'\b' + re.escape(name) + r'\b', str(val), expr)
        try:
            return int(_eval(ast.parse(expr, mode='eval'), {}))
        except Exception:
            return None

    def _process_block_constructs(self, s: str) -> str:
        decls = {name: int(v) for name, v in _INT_DECL.findall(s)}
        while True:
            m = _BLOCK_HEAD.search(s)
            if not m:
                return s
            open_i = m.end() - 1
            close_i = _matching_brace(s, open_i)
            if close_i is None:
                return s
            repl = ''
            if m.group(1).lower() == 'for':
                fm = _FOR_HEAD.search(s[m.start():open_i] + '{')
                if fm:
                    lo, hi = self._int_expr(fm.group(2), decls), self._int_expr(fm.group(3), decls)
                    if lo is not None and hi is not None:
                        var = re.compile(r'\b' + re.escape(fm.group(1)) + r'\b')
                        body = s[open_i + 1:close_i]
                        repl = ' '.join(var.sub(str(i), body) for i in range(lo, hi + 1))
            s = s[:m.start()] + repl + s[close_i + 1:]

    def _extract_gate_definitions(self, s: str):
        defs: Dict[str, Tuple[List[str], List[str], str]] = {}
        while True:
            m = _GATE_DEF.search(s)
            if not m:
                return s, defs
            close_i = _matching_brace(s, m.end() - 1)
            if close_i is None:
                return s, defs
            params = [p.strip() for p in (m.group(2) or '').split(',') if p.strip()]
            args = [a.strip() for a in m.group(3).split(',') if a.strip()]
            defs[m.group(1).lower()] = (params, args, s[m.end():close_i])
            s = s[:m.start()] + s[close_i + 1:]

    def _expand_gate_call(self, instr: str, defs: Dict, depth: int = 0) -> List[str]:
        instr = _WS.sub(' ', instr).strip()
        head = re.split(r'[\s(]', instr, 1)[0].lower()
        if head not in defs:
            return [instr]
        if depth > 64:
            raise ValueError(f"gate definitions nested too deeply at '{head}'")
        params, args, body = defs[head]
        rest = instr[len(head):].strip()
        actual_params: List[str] = []
        if rest.startswith('('):
            depth_p, close = 0, -1
            for k, ch in enumerate(rest):
                depth_p += (ch == '(') - (ch == ')')
                if depth_p == 0:
                    close = k
                    break
            actual_params = [t.strip() for t in _split_params(rest[1:close])]
            rest = rest[close + 1:]
        actual_args = [a.strip() for a in rest.split(',') if a.strip()]
        if len(actual_args) != len(args) or len(actual_params) != len(params):
            raise ValueError(f"gate '{head}' expects {len(params)} parameters and {len(args)} qubits, got '{instr}'")
        table = dict(zip(args, actual_args))
        table.update({p: f'({v})' for p, v in zip(params, actual_params)})
        if table:
            rx = re.compile(r'\b(' + '|'.join(re.escape(k) for k in table) + r')\b')
            body = rx.sub(lambda mm: table[mm.group(1)], body)
        out: List[str] = []
        for st in body.split(';'):
            if st.strip():
                out.extend(self._expand_gate_call(st, defs, depth + 1))
        return out

    # ------------------------------------------------------------ parse
    def parse(self, qasm_str: str) -> QASMCircuit:
        qmap: Dict[str, int] = {}
        n_q = n_c = 0
        ops: List[Dict] = []
        src = _LINE_CMT.sub(' ', _BLOCK_CMT.sub(' ', qasm_str))
        src, defs = self._extract_gate_definitions(src)
        src = self._process_block_constructs(src)
        stmts = [e for st in (x.strip() for x in src.split(';')) if st for e in self._expand_gate_call(st, defs)]
        for instr in stmts:
            instr = _WS.sub(' ', instr).strip()
            if not instr:
                continue
            if re.split(r'[\s(]', instr)[0].lower() in _SKIP:
                continue
            m = _QREG2.match(instr) or _QREG3.match(instr)
            if m:
                if m.re is _QREG2:
                    name, size = m.group(1), int(m.group(2))
                else:
                    name, size = m.group(2), int(m.group(1)) if m.group(1) else 1
                for i in range(size):
                    qmap[f'{name}[{i}]'] = n_q + i
                qmap[name] = n_q
                n_q += size
                continue
            m = _CREG2.match(instr) or _CREG3.match(instr)
            if m:
                size = int(m.group(2)) if m.re is _CREG2 else (int(m.group(1)) if m.group(1) else 1)
                n_c += size
                continue
            op = self._parse_gate(instr, qmap)
            if op is None:
                continue
            if op['name'] in _SINGLE_QUBIT and len(op['qubits']) > 1:
                for q in op['qubits']:
                    ops.append({'type': op['type'], 'name': op['name'], 'qubits': [q], 'params': list(op['params'])})
                    n_q = max(n_q, q + 1)
            else:
                ops.append(op)
                if op['qubits']:
                    n_q = max(n_q, max(op['qubits']) + 1)
        return QASMCircuit(n_q, n_c, ops)

    def validate(self, circ: QASMCircuit) -> Tuple[bool, str]:
        """Structural checks only (qubit count, non-empty, qubit ranges)."""
        if circ.n_qubits <= 0:
            return False, 'n_qubits must be > 0.'
        if not circ.ops:
            return False, 'No gate operations found in circuit.'
        for i, op in enumerate(circ.ops):
            for q in op.get('qubits', []):
                if not 0 <= q < circ.n_qubits:
                    return False, (f"Gate '{op['name']}' at op[{i}] references qubit {q} but "
                                   f"n_qubits={circ.n_qubits}.")
        return True, 'OK'

    # ------------------------------------------------------------ statements
    def _parse_gate(self, instr: str, qmap: Dict[str, int]) -> Optional[Dict]:
        instr = instr.strip()
        po = instr.find('(')
        params_s = ''
        if po != -1:
            depth, pc = 0, -1
            for k in range(po, len(instr)):
                if instr[k] == '(':
                    depth += 1
                elif instr[k] == ')':
                    depth -= 1
                    if depth == 0:
                        pc = k
                        break
            if pc == -1:
                return None
            params_s = instr[po + 1:pc].strip()
            head, qpart = instr[:po].strip(), instr[pc + 1:].strip()
        else:
            parts = instr.split(None, 1)
            head, qpart = parts[0], parts[1] if len(parts) > 1 else ''
        raw = head.strip().lower()
        if not raw:
            return None
        name = _ALIAS.get(raw, raw)
        params = [self._eval_param(t.strip()) for t in _split_params(params_s) if t.strip()] if params_s else []
        qubits = self._resolve_qubits(qpart.replace(' ', ''), qmap)
        if not qubits:
            return None
        return {'type': 'gate', 'name': name, 'qubits': qubits, 'params': params}

    def _eval_param(self, tok: str) -> float:
        try:
            return float(_eval(ast.parse(tok, mode='eval'), _ENV))
        except Exception as e:
            raise ValueError(f"Invalid gate parameter expression '{tok}': {e}") from e

    @staticmethod
    def _split_params(s: str) -> List[str]:
        return _split_params(s)

    def _resolve_qubits(self, s: str, qmap: Dict[str, int]) -> List[int]:
        out: List[int] = []
        for tok in (t.strip() for t in s.split(',')):
            if not tok:
                continue
            m = _RANGE.match(tok)
            if m:
                for i in range(int(m.group(2)), int(m.group(3))):
                    key = f'{m.group(1)}[{i}]'
                    if key in qmap:
                        out.append(qmap[key])
                continue
            if tok in qmap:
                out.append(qmap[tok])
                continue
            b = _INDEX.search(tok)
            if b:
                key = f"{tok[:tok.index('[')]}[{b.group(1)}]"
                out.append(qmap[key] if key in qmap else int(b.group(1)))
                continue
            digits = re.findall(r'\d+', tok)
            if digits and not re.search(r'[a-zA-Z_]', tok):
                out.append(int(digits[-1]))
        return out
