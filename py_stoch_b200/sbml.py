"""Minimal SBML Level 2 reader exposing the subset of the libsbml API that the
stochastic Petri net builder uses.

The reference builds its Petri net from a ``libsbml`` model object
(``mod/petri_net/SPN.py:17-150``) and prints kinetic laws with
``libsbml.formulaToL3String`` (``SPN.py:115``).  libsbml is not a dependency
here, so this module reads the XML with ``xml.etree`` and offers the same
method names (``getListOfSpecies``, ``getKineticLaw().getMath()``, ``AST_NAME``,
``formulaToL3String`` ...).  Any object with that API -- including a real
libsbml model -- can be passed to :class:`py_stoch_b200.petri_net.SPN`.

Only the MathML needed by kinetic laws is supported: ``apply`` with
times/divide/plus/minus/power/root/exp/ln/log/abs/floor/ceiling, ``ci``,
``cn`` (integer, real, e-notation, rational) and the constants ``pi`` and
``exponentiale``.  Anything else raises ``ValueError``.
"""

import math
import xml.etree.ElementTree as ET

# AST node types (names follow libsbml; the integer values are private).
AST_PLUS = 1
AST_MINUS = 2
AST_TIMES = 3
AST_DIVIDE = 4
AST_POWER = 5
AST_INTEGER = 10
AST_REAL = 11
AST_RATIONAL = 12
AST_NAME = 20
AST_CONSTANT_PI = 30
AST_CONSTANT_E = 31
AST_FUNCTION = 40          # unary built-in function, name in .fname

_OPS = {'plus': AST_PLUS, 'minus': AST_MINUS, 'times': AST_TIMES,
        'divide': AST_DIVIDE, 'power': AST_POWER}
_FUNCS = {'exp', 'ln', 'log', 'abs', 'floor', 'ceiling', 'root'}


def _local(tag):
    return tag.rsplit('}', 1)[-1]


class ASTNode(object):
    """A MathML expression node with the libsbml ASTNode accessors."""

    def __init__(self, node_type, name=None, value=None, children=None,
                 fname=None):
        self._type = node_type
        self._name = name
        self.value = value
        self.fname = fname
        self._children = list(children or [])

    def getType(self):
        return self._type

    def getName(self):
        return self._name

    def setName(self, name):
        self._name = name

    def getNumChildren(self):
        return len(self._children)

    def getChild(self, i):
        return self._children[i]

    def isName(self):
        return self._type == AST_NAME


def _parse_cn(el):
    kind = el.get('type', 'real')
    parts = [p.strip() for p in el.itertext()]
    parts = [p for p in parts if p]
    if kind == 'integer':
        return ASTNode(AST_INTEGER, value=int(parts[0]))
    if kind == 'e-notation':
        return ASTNode(AST_REAL, value=float(parts[0]) * 10.0 ** int(parts[1]))
    if kind == 'rational':
        return ASTNode(AST_RATIONAL, value=(int(parts[0]), int(parts[1])))
    return ASTNode(AST_REAL, value=float(parts[0]))


def _parse_math(el):
    tag = _local(el.tag)
    if tag == 'math':
        kids = list(el)
        if len(kids) != 1:
            raise ValueError('math element must have exactly one child')
        return _parse_math(kids[0])
    if tag == 'ci':
        return ASTNode(AST_NAME, name=''.join(el.itertext()).strip())
    if tag == 'cn':
        return _parse_cn(el)
    if tag == 'pi':
        return ASTNode(AST_CONSTANT_PI)
    if tag == 'exponentiale':
        return ASTNode(AST_CONSTANT_E)
    if tag == 'apply':
        kids = list(el)
        op = _local(kids[0].tag)
        args = []
        degree = None
        logbase = None
        for k in kids[1:]:
            kt = _local(k.tag)
            if kt == 'degree':
                degree = _parse_math(list(k)[0])
            elif kt == 'logbase':
                logbase = _parse_math(list(k)[0])
            else:
                args.append(_parse_math(k))
        if op in _OPS:
            return ASTNode(_OPS[op], children=args)
        if op in _FUNCS:
            if op == 'root':
                # root(n, x) -> x^(1/n); default square root
                n = degree if degree is not None else ASTNode(AST_INTEGER,
                                                             value=2)
                inv = ASTNode(AST_DIVIDE,
                              children=[ASTNode(AST_INTEGER, value=1), n])
                return ASTNode(AST_POWER, children=[args[0], inv])
            if op == 'log':
                base = logbase if logbase is not None else ASTNode(
                    AST_INTEGER, value=10)
                return ASTNode(AST_DIVIDE, children=[
                    ASTNode(AST_FUNCTION, fname='ln', children=args),
                    ASTNode(AST_FUNCTION, fname='ln', children=[base])])
            return ASTNode(AST_FUNCTION, fname=op, children=args)
        raise ValueError('unsupported MathML operator: %s' % op)
    raise ValueError('unsupported MathML element: %s' % tag)


# --- infix printing ---------------------------------------------------------

_PREC = {AST_PLUS: 1, AST_MINUS: 1, AST_TIMES: 2, AST_DIVIDE: 2,
         AST_POWER: 4}
_SYM = {AST_PLUS: '+', AST_MINUS: '-', AST_TIMES: '*', AST_DIVIDE: '/',
        AST_POWER: '^'}


def _fmt_real(v):
    if v == int(v) and abs(v) < 1e15:
        return str(int(v))
    r = repr(float(v))
    return r


def _prec(node):
    t = node.getType()
    if t in _PREC:
        if t == AST_MINUS and node.getNumChildren() == 1:
            return 3
        return _PREC[t]
    if t in (AST_INTEGER, AST_REAL) and node.value < 0:
        return 3
    return 5


def formulaToL3String(node):
    """Print an expression tree as an infix string.

    Mirrors the role of ``libsbml.formulaToL3String`` (used at
    ``SPN.py:115``): binary operators are separated by single spaces,
    powers use ``^``, function calls use ``name(arg)`` and parentheses are
    emitted only where precedence requires them.
    """
    t = node.getType()
    if t == AST_NAME:
        return node.getName()
    if t == AST_INTEGER:
        return str(node.value)
    if t == AST_REAL:
        return _fmt_real(node.value)
    if t == AST_RATIONAL:
        return '(%d / %d)' % node.value
    if t == AST_CONSTANT_PI:
        return 'pi'
    if t == AST_CONSTANT_E:
        return 'exponentiale'
    if t == AST_FUNCTION:
        return '%s(%s)' % (node.fname, ', '.join(
            formulaToL3String(c) for c in node._children))
    if t in _SYM:
        kids = node._children
        if t == AST_MINUS and len(kids) == 1:
            inner = formulaToL3String(kids[0])
            if _prec(kids[0]) < 5:
                inner = '(' + inner + ')'
            return '-' + inner
        if len(kids) == 0:
            return '0' if t in (AST_PLUS, AST_MINUS) else '1'
        if len(kids) == 1:
            return formulaToL3String(kids[0])
        p = _PREC[t]
        out = []
        for i, c in enumerate(kids):
            s = formulaToL3String(c)
            cp = _prec(c)
            need = cp < p
            if i > 0 and cp == p and t in (AST_MINUS, AST_DIVIDE):
                need = True
            if t == AST_POWER and i == 0 and cp <= p:
                need = True
            if need:
                s = '(' + s + ')'
            out.append(s)
        return (' %s ' % _SYM[t]).join(out)
    raise ValueError('cannot print node type %r' % t)


# --- model objects ----------------------------------------------------------

class _ListOf(list):
    def size(self):
        return len(self)

    def get(self, i):
        return self[i]


def _bool_attr(el, name, default=False):
    v = el.get(name)
    if v is None:
        return default
    return v.strip().lower() in ('true', '1')


class Species(object):
    def __init__(self, el):
        self._id = el.get('id')
        self._name = el.get('name', self._id)
        amt = el.get('initialAmount')
        if amt is None:
            amt = el.get('initialConcentration')
        self._amount = float(amt) if amt is not None else float('nan')
        self._constant = _bool_attr(el, 'constant', False)
        self._boundary = _bool_attr(el, 'boundaryCondition', False)

    def getId(self):
        return self._id

    def getName(self):
        return self._name

    def getInitialAmount(self):
        return self._amount

    def getConstant(self):
        return self._constant

    def getBoundaryCondition(self):
        return self._boundary


class Parameter(object):
    def __init__(self, el):
        self._id = el.get('id')
        self._name = el.get('name', self._id)
        v = el.get('value')
        self._value = float(v) if v is not None else float('nan')

    def getId(self):
        return self._id

    def getName(self):
        return self._name

    def getValue(self):
        return self._value


class SpeciesReference(object):
    def __init__(self, el):
        self._species = el.get('species')
        st = el.get('stoichiometry')
        # SBML Level 2 default stoichiometry is 1.
        self._stoich = float(st) if st is not None else 1.0

    def getSpecies(self):
        return self._species

    def getStoichiometry(self):
        return self._stoich


class KineticLaw(object):
    def __init__(self, el):
        math_el = None
        for k in el:
            if _local(k.tag) == 'math':
                math_el = k
        if math_el is None:
            raise ValueError('kineticLaw without math')
        self._math = _parse_math(math_el)
        self._params = _ListOf()
        for k in el:
            if _local(k.tag) in ('listOfParameters', 'listOfLocalParameters'):
                for p in k:
                    self._params.append(Parameter(p))

    def getMath(self):
        return self._math

    def getListOfParameters(self):
        return self._params


class Reaction(object):
    def __init__(self, el):
        self._id = el.get('id')
        self._name = el.get('name', self._id)
        self._reversible = _bool_attr(el, 'reversible', True)
        self._reactants = _ListOf()
        self._products = _ListOf()
        self._law = None
        for k in el:
            t = _local(k.tag)
            if t == 'listOfReactants':
                self._reactants.extend(SpeciesReference(s) for s in k)
            elif t == 'listOfProducts':
                self._products.extend(SpeciesReference(s) for s in k)
            elif t == 'kineticLaw':
                self._law = KineticLaw(k)

    def getId(self):
        return self._id

    def getName(self):
        return self._name

    def getReversible(self):
        return self._reversible

    def getListOfReactants(self):
        return self._reactants

    def getListOfProducts(self):
        return self._products

    def getKineticLaw(self):
        return self._law


class Model(object):
    def __init__(self, el):
        self._id = el.get('id', el.get('name', ''))
        self._name = el.get('name', self._id)
        self._species = _ListOf()
        self._params = _ListOf()
        self._reactions = _ListOf()
        for k in el:
            t = _local(k.tag)
            if t == 'listOfSpecies':
                self._species.extend(Species(s) for s in k)
            elif t == 'listOfParameters':
                self._params.extend(Parameter(p) for p in k)
            elif t == 'listOfReactions':
                self._reactions.extend(Reaction(r) for r in k)

    def getId(self):
        return self._id

    def getName(self):
        return self._name

    def getListOfSpecies(self):
        return self._species

    def getListOfParameters(self):
        return self._params

    def getListOfReactions(self):
        return self._reactions

    def getNumSpecies(self):
        return len(self._species)

    def getNumReactions(self):
        return len(self._reactions)


class SBMLDocument(object):
    def __init__(self, model, errors):
        self._model = model
        self._errors = errors

    def getNumErrors(self):
        return len(self._errors)

    def getError(self, i):
        return self._errors[i]

    def getModel(self):
        return self._model


def _document_from_root(root):
    errors = []
    model = None
    for k in root:
        if _local(k.tag) == 'model':
            try:
                model = Model(k)
            except ValueError as e:
                errors.append(str(e))
    if model is None:
        errors.append('no model element')
    return SBMLDocument(model, errors)


class SBMLReader(object):
    """``libsbml.SBMLReader`` look-alike: ``readSBML(path)``."""

    def readSBML(self, path):
        try:
            root = ET.parse(path).getroot()
        except (ET.ParseError, IOError, OSError) as e:
            return SBMLDocument(None, [str(e)])
        return _document_from_root(root)

    def readSBMLFromString(self, text):
        try:
            root = ET.fromstring(text)
        except ET.ParseError as e:
            return SBMLDocument(None, [str(e)])
        return _document_from_root(root)


def read_sbml(path):
    """Read an SBML file and return its model; raise on any error.

    Same check as the reference example scripts (``PL_sim.py:17-20``): a
    non-zero error count raises ``UserWarning``.
    """
    doc = SBMLReader().readSBML(path)
    if doc.getNumErrors() > 0:
        raise UserWarning('%d errors in SBML file: %s'
                          % (doc.getNumErrors(), path))
    return doc.getModel()


def evaluate(node, env):
    """Numerically evaluate an expression tree with names bound in ``env``."""
    t = node.getType()
    if t == AST_NAME:
        return float(env[node.getName()])
    if t in (AST_INTEGER, AST_REAL):
        return float(node.value)
    if t == AST_RATIONAL:
        return node.value[0] / float(node.value[1])
    if t == AST_CONSTANT_PI:
        return math.pi
    if t == AST_CONSTANT_E:
        return math.e
    vals = [evaluate(c, env) for c in node._children]
    if t == AST_PLUS:
        return sum(vals)
    if t == AST_MINUS:
        return -vals[0] if len(vals) == 1 else vals[0] - sum(vals[1:])
    if t == AST_TIMES:
        p = 1.0
        for v in vals:
            p *= v
        return p
    if t == AST_DIVIDE:
        return vals[0] / vals[1]
    if t == AST_POWER:
        return vals[0] ** vals[1]
    if t == AST_FUNCTION:
        f = {'exp': math.exp, 'ln': math.log, 'abs': abs,
             'floor': math.floor, 'ceiling': math.ceil}[node.fname]
        return f(vals[0])
    raise ValueError('cannot evaluate node type %r' % t)


# --- writing ----------------------------------------------------------------

def write_sbml(model_id, species, parameters, reactions):
    """SBML Level 2 Version 4 text of a small model.

    ``species``: list of (id, initial_amount) or (id, amount, constant);
    ``parameters``: list of (id, value); ``reactions``: list of
    (id, reactants, products, kinetic_law) with reactants / products lists
    of (species_id, stoichiometry) and the law an infix string over species
    and parameter ids using + - * / ( ) and numbers.
    """
    import re
    from xml.sax.saxutils import quoteattr

    def mathml(expr):
        toks = re.findall(r'\d+\.\d*(?:[eE][-+]?\d+)?|\d+(?:[eE][-+]?\d+)?'
                          r'|[A-Za-z_]\w*|[-+*/()^]', expr)
        pos = [0]

        def peek():
            return toks[pos[0]] if pos[0] < len(toks) else None

        def take():
            t = toks[pos[0]]
            pos[0] += 1
            return t

        def atom():
            t = take()
            if t == '(':
                e = add()
                take()
                return e
            if t == '-':
                return '<apply><minus/>%s</apply>' % atom()
            if re.match(r'\d', t):
                return '<cn>%s</cn>' % t
            return '<ci>%s</ci>' % t

        def power():
            b = atom()
            if peek() == '^':
                take()
                return '<apply><power/>%s%s</apply>' % (b, power())
            return b

        def mul():
            e = power()
            while peek() in ('*', '/'):
                op = 'times' if take() == '*' else 'divide'
                e = '<apply><%s/>%s%s</apply>' % (op, e, power())
            return e

        def add():
            e = mul()
            while peek() in ('+', '-'):
                op = 'plus' if take() == '+' else 'minus'
                e = '<apply><%s/>%s%s</apply>' % (op, e, mul())
            return e

        body = add()
        return ('<math xmlns="http://www.w3.org/1998/Math/MathML">%s</math>'
                % body)

    lines = ['<?xml version="1.0" encoding="UTF-8"?>',
             '<sbml xmlns="http://www.sbml.org/sbml/level2/version4" '
             'level="2" version="4">',
             '<model id=%s name=%s>' % (quoteattr(model_id),
                                        quoteattr(model_id)),
             '<listOfCompartments><compartment id="cell" size="1"/>'
             '</listOfCompartments>', '<listOfSpecies>']
    for sp in species:
        sid, amt = sp[0], sp[1]
        const = len(sp) > 2 and sp[2]
        lines.append('<species id=%s compartment="cell" initialAmount="%r"%s/>'
                     % (quoteattr(sid), float(amt),
                        ' constant="true"' if const else ''))
    lines.append('</listOfSpecies><listOfParameters>')
    for pid, val in parameters:
        lines.append('<parameter id=%s value="%r"/>' % (quoteattr(pid),
                                                        float(val)))
    lines.append('</listOfParameters><listOfReactions>')
    for rid, reactants, products, law in reactions:
        lines.append('<reaction id=%s reversible="false">' % quoteattr(rid))
        for tag, lst in (('listOfReactants', reactants),
                         ('listOfProducts', products)):
            if lst:
                lines.append('<%s>' % tag)
                for s, st in lst:
                    lines.append('<speciesReference species=%s '
                                 'stoichiometry="%d"/>' % (quoteattr(s), st))
                lines.append('</%s>' % tag)
        lines.append('<kineticLaw>%s</kineticLaw></reaction>' % mathml(law))
    lines.append('</listOfReactions></model></sbml>')
    return '\n'.join(lines)


def read_sbml_string(text):
    doc = SBMLReader().readSBMLFromString(text)
    if doc.getNumErrors() > 0:
        raise UserWarning('%d errors in SBML text' % doc.getNumErrors())
    return doc.getModel()


def lotka_volterra_sbml():
    """SBML text of the Lotka-Volterra network (species x, y, catalyst a)."""
    return write_sbml(
        'lotka_volterra', [('x', 1000), ('y', 1000), ('a', 1)],
        [('c1', 10), ('c2', 0.01), ('c3', 10)],
        [('reaction1', [('a', 1), ('x', 1)], [('a', 1), ('x', 2)],
          'c1 * x * a'),
         ('reaction2', [('x', 1), ('y', 1)], [('y', 2)], 'c2 * x * y'),
         ('reaction3', [('y', 1)], [], 'c3 * y')])


def schlogl_sbml():
    """SBML text of the Schlogl network with buffered A, B as parameters."""
    return write_sbml(
        'schlogl', [('X', 250)],
        [('c1', 3e-7), ('c2', 1e-4), ('c3', 1e-3), ('c4', 3.5), ('a', 1e5),
         ('b', 2e5)],
        [('reaction1', [('X', 2)], [('X', 3)], 'c1 / 2 * a * X * (X - 1)'),
         ('reaction2', [('X', 3)], [('X', 2)],
          'c2 / 6 * X * (X - 1) * (X - 2)'),
         ('reaction3', [], [('X', 1)], 'c3 * b'),
         ('reaction4', [('X', 1)], [], 'c4 * X')])
