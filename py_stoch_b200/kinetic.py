"""General kinetic laws: the hazard strings of ``SPN.h`` compiled to a
postfix program the kernels evaluate per reaction and step.

The reference pastes each hazard into its kernels as C source,
``a[j] = <law>;`` with ``species_i`` -> ``x[i]`` (int) and ``parameter_k``
-> ``d_c[k]`` (double) (``mod/parser/parser.py:32-55``), so a law is
evaluated with C's typing: integer subexpressions (species, integer
literals) stay integer, and ``/`` of two integers truncates.  Laws of the
mass-action form ``k * prod (x_i - m)`` take the engine's factor path
(``model.analyse_hazard``); every other law is compiled here.  Evaluation
is FP64 with explicitly rounded operations (integer subexpressions are
exact in FP64 below 2^53), the result rounded once to the FP32 propensity.

Grammar (the infix form ``formulaToL3String`` writes): numbers, names,
``+ - * / ^``, unary minus, parentheses, and the functions ``exp``,
``ln``, ``log10``, ``sqrt``, ``abs``, ``floor``, ``ceil``/``ceiling`` and
``pow``.  ``^`` and ``pow`` with a small non-negative integer literal
exponent become repeated multiplication; other powers are
``exp(b * ln(a))``.

Program words: ``op << 24 | arg``; constants (parameter values and
literals) in an FP64 pool.
"""

import math
import re

import numpy as np

OP_X, OP_C, OP_ADD, OP_SUB, OP_MUL, OP_DIV, OP_IDIV, OP_NEG = 1, 2, 3, 4, 5, 6, 7, 8
OP_EXP, OP_LN, OP_SQRT, OP_ABS, OP_FLOOR, OP_CEIL, OP_DUP = 10, 11, 12, 13, 14, 15, 16

MAX_STACK = 8  # evaluation stack of the kernels (registers / local array)
MAX_INT_POW = 8


class KineticLawError(ValueError):
    pass


_TOKEN = re.compile(r'\s*(?:(?P<num>(?:\d+\.\d*|\.\d+|\d+)(?:[eE][+-]?\d+)?)'
                    r'|(?P<name>[A-Za-z_][A-Za-z_0-9]*)'
                    r'|(?P<op>[-+*/^(),]))')


def _tokens(text):
    pos, out = 0, []
    text = text.strip()
    while pos < len(text):
        m = _TOKEN.match(text, pos)
        if not m or m.end() == pos:
            raise KineticLawError('cannot read kinetic law %r at %r'
                                  % (text, text[pos:pos + 10]))
        pos = m.end()
        if m.group('num') is not None:
            s = m.group('num')
            is_int = re.fullmatch(r'\d+', s) is not None
            out.append(('num', int(s) if is_int else float(s), is_int))
        elif m.group('name') is not None:
            out.append(('name', m.group('name'), None))
        else:
            out.append(('op', m.group('op'), None))
    out.append(('end', None, None))
    return out


class _Parser(object):
    """Recursive descent to nodes (kind, value, children, is_int)."""

    FUNCS = {'exp', 'ln', 'log10', 'sqrt', 'abs', 'floor', 'ceil', 'ceiling',
             'pow'}

    def __init__(self, text, n_species, n_params):
        self.t = _tokens(text)
        self.i = 0
        self.text = text
        self.S = n_species
        self.P = n_params

    def peek(self):
        return self.t[self.i]

    def take(self, kind=None, val=None):
        tok = self.t[self.i]
        if (kind and tok[0] != kind) or (val is not None and tok[1] != val):
            raise KineticLawError('unexpected %r in kinetic law %r'
                                  % (tok[1], self.text))
        self.i += 1
        return tok

    def parse(self):
        node = self.expr()
        self.take('end')
        return node

    def expr(self):
        node = self.term()
        while self.peek()[0] == 'op' and self.peek()[1] in '+-':
            op = self.take()[1]
            rhs = self.term()
            node = (op, None, [node, rhs], node[3] and rhs[3])
        return node

    def term(self):
        node = self.unary()
        while self.peek()[0] == 'op' and self.peek()[1] in '*/':
            op = self.take()[1]
            rhs = self.unary()
            node = (op, None, [node, rhs], node[3] and rhs[3])
        return node

    def unary(self):
        if self.peek()[0] == 'op' and self.peek()[1] in '+-':
            op = self.take()[1]
            node = self.unary()
            return node if op == '+' else ('neg', None, [node], node[3])
        return self.power()

    def power(self):
        base = self.atom()
        if self.peek()[0] == 'op' and self.peek()[1] == '^':
            self.take()
            exp = self.unary()  # right associative
            return ('pow', None, [base, exp], False)
        return base

    def atom(self):
        tok = self.take()
        if tok[0] == 'num':
            return ('num', tok[1], [], tok[2])
        if tok[0] == 'op' and tok[1] == '(':
            node = self.expr()
            self.take('op', ')')
            return node
        if tok[0] == 'name':
            name = tok[1]
            if self.peek()[0] == 'op' and self.peek()[1] == '(':
                if name not in self.FUNCS:
                    raise KineticLawError('unsupported function %r in %r'
                                          % (name, self.text))
                self.take()
                args = [self.expr()]
                while self.peek()[0] == 'op' and self.peek()[1] == ',':
                    self.take()
                    args.append(self.expr())
                self.take('op', ')')
                want = 2 if name == 'pow' else 1
                if len(args) != want:
                    raise KineticLawError('%s takes %d argument(s) in %r'
                                          % (name, want, self.text))
                if name == 'pow':
                    return ('pow', None, args, False)
                is_int = name == 'abs' and args[0][3]
                return ('fn', name, args, is_int)
            m = re.fullmatch(r'species_(\d+)', name)
            if m and int(m.group(1)) < self.S:
                return ('x', int(m.group(1)), [], True)
            m = re.fullmatch(r'parameter_(\d+)', name)
            if m and int(m.group(1)) < self.P:
                return ('p', int(m.group(1)), [], False)
            raise KineticLawError('unknown name %r in kinetic law %r'
                                  % (name, self.text))
        raise KineticLawError('unexpected %r in kinetic law %r'
                              % (tok[1], self.text))


def compile_law(text, n_species, params):
    """(code words [np.uint32], constants [np.float64], species used) of
    one hazard string; ``params`` are the values of ``parameter_k``."""
    node = _Parser(text, n_species, len(params)).parse()
    code, consts, used = [], [], set()
    depth = [0, 0]  # current, max

    def push(n=1):
        depth[0] += n
        depth[1] = max(depth[1], depth[0])

    def const(v):
        v = float(v)
        for k, c in enumerate(consts):
            if c == v and math.copysign(1.0, c) == math.copysign(1.0, v):
                return k
        consts.append(v)
        return len(consts) - 1

    def emit(op, arg=0, pops=0, pushes=0):
        code.append((op << 24) | arg)
        depth[0] -= pops
        push(pushes)

    def gen(n):
        kind = n[0]
        if kind == 'num':
            emit(OP_C, const(n[1]), 0, 1)
        elif kind == 'x':
            used.add(n[1])
            emit(OP_X, n[1], 0, 1)
        elif kind == 'p':
            emit(OP_C, const(params[n[1]]), 0, 1)
        elif kind == 'neg':
            gen(n[2][0])
            emit(OP_NEG, 0, 1, 1)
        elif kind in '+-*/':
            gen(n[2][0])
            gen(n[2][1])
            if kind == '/':
                op = OP_IDIV if n[3] else OP_DIV
            else:
                op = {'+': OP_ADD, '-': OP_SUB, '*': OP_MUL}[kind]
            emit(op, 0, 2, 1)
        elif kind == 'pow':
            base, ex = n[2]
            if (ex[0] == 'num' and ex[3] and 0 <= ex[1] <= MAX_INT_POW):
                k = ex[1]
                if k == 0:
                    emit(OP_C, const(1.0), 0, 1)
                    return
                gen(base)
                for _ in range(k - 1):
                    emit(OP_DUP, 0, 0, 1)
                for _ in range(k - 1):
                    emit(OP_MUL, 0, 2, 1)
                return
            # a^b = exp(b * ln a)
            gen(ex)
            gen(base)
            emit(OP_LN, 0, 1, 1)
            emit(OP_MUL, 0, 2, 1)
            emit(OP_EXP, 0, 1, 1)
        elif kind == 'fn':
            name = n[1]
            gen(n[2][0])
            if name == 'log10':
                emit(OP_LN, 0, 1, 1)
                emit(OP_C, const(1.0 / math.log(10.0)), 0, 1)
                emit(OP_MUL, 0, 2, 1)
                return
            op = {'exp': OP_EXP, 'ln': OP_LN, 'sqrt': OP_SQRT,
                  'abs': OP_ABS, 'floor': OP_FLOOR, 'ceil': OP_CEIL,
                  'ceiling': OP_CEIL}[name]
            emit(op, 0, 1, 1)
        else:  # pragma: no cover - parser produces no other kinds
            raise KineticLawError('internal: node %r' % (kind,))

    gen(node)
    if depth[1] > MAX_STACK:
        raise KineticLawError('kinetic law %r needs a stack of %d (limit %d)'
                              % (text, depth[1], MAX_STACK))
    if len(consts) >= (1 << 24):
        raise KineticLawError('too many constants')
    return (np.asarray(code, dtype=np.uint32),
            np.asarray(consts, dtype=np.float64), sorted(used))


def has_int_division(text, n_species, n_params):
    """True when the law divides two integer-typed subexpressions, which C
    (and so the reference) truncates; such laws are compiled even when
    their real-valued form is mass action."""
    def walk(n):
        if n[0] == '/' and n[3]:
            return True
        return any(walk(c) for c in n[2])
    try:
        return walk(_Parser(text, n_species, n_params).parse())
    except KineticLawError:
        return False


def evaluate(code, consts, x):
    """Reference evaluation of a compiled program in Python floats (FP64
    per operation; for tests of the compiler)."""
    st = []
    for w in np.asarray(code, dtype=np.uint64):
        op, arg = int(w) >> 24, int(w) & 0xFFFFFF
        if op == OP_X:
            st.append(float(x[arg]))
        elif op == OP_C:
            st.append(float(consts[arg]))
        elif op == OP_DUP:
            st.append(st[-1])
        elif op in (OP_ADD, OP_SUB, OP_MUL, OP_DIV, OP_IDIV):
            b, a = st.pop(), st.pop()
            if op == OP_ADD:
                st.append(a + b)
            elif op == OP_SUB:
                st.append(a - b)
            elif op == OP_MUL:
                st.append(a * b)
            elif op == OP_DIV:
                st.append(a / b if b != 0 else math.copysign(math.inf, a)
                          if a != 0 else math.nan)
            else:
                st.append(float(math.trunc(a / b)) if b != 0 else math.nan)
        elif op == OP_NEG:
            st.append(-st.pop())
        elif op == OP_EXP:
            v = st.pop()
            st.append(math.exp(v) if v < 709.0 else math.inf)
        elif op == OP_LN:
            v = st.pop()
            st.append(math.log(v) if v > 0 else (-math.inf if v == 0
                                                 else math.nan))
        elif op == OP_SQRT:
            v = st.pop()
            st.append(math.sqrt(v) if v >= 0 else math.nan)
        elif op == OP_ABS:
            st.append(abs(st.pop()))
        elif op == OP_FLOOR:
            st.append(float(math.floor(st.pop())))
        elif op == OP_CEIL:
            st.append(float(math.ceil(st.pop())))
        else:
            raise KineticLawError('bad opcode %d' % op)
    return st[-1]
