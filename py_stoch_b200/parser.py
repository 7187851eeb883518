"""Simulation argument bags and the parser that fills them.

Python 3 restatement of ``mod/parser/parser.py``, ``mod/parser/tl_parser.py``
and ``mod/parser/g_parser.py`` (reference).  ``TlArgs`` keeps every field the
reference defines (``tl_parser.py:8-47``) with the same meaning and dtype, so
code written against the reference's ``TlArgs`` reads the same values here.

Three fields are added for the B200 engine, which does not compile the
generated CUDA source string: ``pre_matrix``/``post_matrix`` (dense ``Pre`` and
``Post``) and ``hazard_exprs`` (the kinetic-law strings ``SPN.h``).  The
sparse ``char4`` encodings (``A``, ``V``, ``V_t``, ``V_bar``) keep the
reference's int8/uint8 limits (``parser.py:58-71``); for a model beyond them
the fields are ``None`` while the engine still runs it from the dense fields.
"""

import re
import xml.etree.ElementTree as ET

import numpy
import sympy


class EncodingLimitError(ValueError):
    """A matrix does not fit the reference's int8 index / uint8 count format."""


class Parser(object):
    @staticmethod
    def parse_settings(settings_file, args_obj):
        """Read output species, duration, sample count and trajectory count
        from a settings XML file (``parser.py:8-29``)."""
        root = ET.parse(settings_file).getroot()
        out_species = root.find('output_species')
        args_obj.E = numpy.array(
            [int(s.get('idx')) for s in out_species.findall('species')]
        ).astype(numpy.int32)
        args_obj.t_max = float(root.find('duration').text)
        args_obj.ita = int(root.find('num_output_time_points').text)
        args_obj.U = int(root.find('num_simulations').text)

    @staticmethod
    def define_hazards(spn):
        """CUDA source of ``UpdatePropensities`` for the model (``parser.py:32-55``).

        One ``a[j] = <kinetic law>;`` line per reaction with ``species_i``
        replaced by ``x[i]`` and ``parameter_k`` by ``d_c[k]``, highest index
        first so ``species_1`` never clobbers ``species_10``.  The B200 engine
        does not compile this string; it is kept for API compatibility.
        """
        lines = ['    a[%d] = %s;' % (j, h) for j, h in enumerate(spn.h)]
        code = ('\n__device__ void UpdatePropensities(double* __restrict__ a, '
                'int* __restrict__ x)\n{\n' + '\n'.join(lines) + '\n}\n')
        for i in range(len(spn.P), 0, -1):
            code = code.replace('species_%d' % (i - 1), 'x[%d]' % (i - 1))
        for k in range(len(spn.c), 0, -1):
            code = code.replace('parameter_%d' % (k - 1), 'd_c[%d]' % (k - 1))
        return code

    @staticmethod
    def flatten_matrix(matrix):
        """Row-major list of nonzeros as ``(int8 row, int8 col, int8 value, 0)``
        plus the count as ``uint8`` (``parser.py:58-71``).

        Raises :class:`EncodingLimitError` where the reference's int8/uint8
        types cannot hold an index, value or count.
        """
        matrix = numpy.asarray(matrix)
        entries = []
        for i in range(matrix.shape[0]):
            for j in range(matrix.shape[1]):
                v = matrix[i][j]
                if v != 0:
                    if not (-128 <= i <= 127 and -128 <= j <= 127
                            and -128 <= v <= 127):
                        raise EncodingLimitError(
                            'entry (%d, %d, %r) exceeds int8' % (i, j, v))
                    entries.append(numpy.array(
                        [numpy.int8(i), numpy.int8(j), numpy.int8(int(v)),
                         numpy.int8(0)]))
        if len(entries) > 255:
            raise EncodingLimitError('%d nonzeros exceed uint8'
                                     % len(entries))
        return numpy.array(entries), numpy.uint8(len(entries))


class TlArgs(object):
    """Parameter bag of one cuTauLeaping / Gillespie run (``tl_parser.py:8-47``)."""

    def __init__(self):
        self.c = []
        self.x_0 = []
        self.A = []
        self.V = []
        self.V_t = []
        self.V_bar = []
        self.M = 0
        self.N = 0
        self.A_size = 0
        self.V_size = 0
        self.V_t_size = 0
        self.V_bar_size = 0
        self.hazards = []
        self.H = []
        self.H_type = []
        self.E = numpy.array([0]).astype(numpy.int32)
        self.t_max = 1
        self.ita = 11
        self.U = 128
        self.kappa = len(self.E)
        self.I = numpy.array([])
        self.n_c = 10
        self.eta = 0.03
        self.gillespie = 0
        # engine inputs (dense matrices and kinetic-law strings)
        self.pre_matrix = None
        self.post_matrix = None
        self.hazard_exprs = None


def _flatten_or_none(matrix):
    try:
        return Parser.flatten_matrix(matrix)
    except EncodingLimitError:
        return None, int(numpy.count_nonzero(matrix))


class TlParser(Parser):
    @staticmethod
    def parse(args_out, stochastic_petri_net):
        """Fill ``args_out`` from a Petri net (``tl_parser.py:51-78``)."""
        spn = stochastic_petri_net
        args_out.c = numpy.array(spn.c).astype(numpy.float64)
        args_out.x_0 = numpy.array(spn.M).astype(numpy.int32)

        ma = numpy.asarray(spn.Pre)
        mb = numpy.asarray(spn.Post)
        mv = mb - ma
        mv_t = mv.transpose()
        mv_bar = abs(mv * numpy.asarray(spn.StoichMConst))

        args_out.A, args_out.A_size = _flatten_or_none(ma)
        args_out.V, args_out.V_size = _flatten_or_none(mv)
        args_out.V_t, args_out.V_t_size = _flatten_or_none(mv_t)
        args_out.V_bar, args_out.V_bar_size = _flatten_or_none(mv_bar)

        args_out.M = len(spn.T)
        args_out.N = len(spn.P)
        args_out.H, args_out.H_type = TlParser.get_hors(spn)
        args_out.hazards = TlParser.define_hazards(spn)
        args_out.kappa = len(args_out.E)
        args_out.I = numpy.linspace(0, args_out.t_max,
                                    num=args_out.ita).astype(numpy.float32)

        args_out.pre_matrix = ma.copy()
        args_out.post_matrix = mb.copy()
        args_out.hazard_exprs = list(spn.h)
        return args_out

    @staticmethod
    def get_reaction_orders(hazards, species, pre=None):
        """Total polynomial degree of each hazard in the species symbols
        (``tl_parser.py:81-95``).  The reference raises for a law that is
        not a polynomial in the species (e.g. Michaelis-Menten); given the
        Pre matrix, such a reaction's order here is its number of reactant
        molecules instead."""
        orders = []
        syms = sympy.symbols(list(species.keys()))
        for j, hazard in enumerate(hazards):
            expr = sympy.expand(hazard.replace('^', '**'))
            try:
                poly = sympy.poly(expr, *syms) if syms else None
            except sympy.PolynomialError:
                if pre is None:
                    raise
                orders.append(int(numpy.asarray(pre)[:, j].sum()))
                continue
            orders.append(int(poly.total_degree()) if poly is not None else 0)
        return orders

    @staticmethod
    def get_hors(spn):
        """Highest order of reaction (``H``) per species and the largest
        reactant stoichiometry of that species (``H_type``) over the
        reactions whose hazard mentions it (``tl_parser.py:98-120``)."""
        hors = numpy.zeros(len(spn.P))
        hors_type = numpy.zeros(len(spn.P))
        pre = numpy.asarray(spn.Pre)
        orders = TlParser.get_reaction_orders(spn.h, spn.P, pre)
        for reaction, j in spn.T.items():
            for species, i in spn.P.items():
                hazard = spn.h[j]
                if re.search('(?<![a-zA-Z0-9_])' + species +
                             '(?![a-zA-Z0-9_])', hazard) is not None:
                    if hors[i] <= orders[j]:
                        hors[i] = orders[j]
                    stoich = pre[i][j]
                    if stoich > hors_type[i]:
                        hors_type[i] = int(stoich)
        return (numpy.array(hors).astype(numpy.int32),
                numpy.array(hors_type).astype(numpy.int32))


class GArgs(object):
    """SSA-only parameter bag (``g_parser.py:5-28``)."""

    def __init__(self):
        self.c = []
        self.x_0 = []
        self.V = []
        self.M = 0
        self.N = 0
        self.V_size = 0
        self.hazards = []
        self.E = numpy.array([0]).astype(numpy.int32)
        self.t_max = 1
        self.ita = 11
        self.U = 128
        self.kappa = len(self.E)
        self.I = numpy.array([])
        self.gillespie = 1
        self.pre_matrix = None
        self.post_matrix = None
        self.hazard_exprs = None


class GParser(Parser):
    @staticmethod
    def parse(args_out, stochastic_petri_net):
        """Fill a :class:`GArgs` (``g_parser.py:32-52``)."""
        spn = stochastic_petri_net
        args_out.c = numpy.array(spn.c).astype(numpy.float64)
        args_out.x_0 = numpy.array(spn.M).astype(numpy.int32)
        ma = numpy.asarray(spn.Pre)
        mb = numpy.asarray(spn.Post)
        args_out.V, args_out.V_size = _flatten_or_none(mb - ma)
        args_out.M = len(spn.T)
        args_out.N = len(spn.P)
        args_out.hazards = GParser.define_hazards(spn)
        args_out.kappa = len(args_out.E)
        args_out.I = numpy.linspace(0, args_out.t_max,
                                    num=args_out.ita).astype(numpy.float32)
        args_out.pre_matrix = ma.copy()
        args_out.post_matrix = mb.copy()
        args_out.hazard_exprs = list(spn.h)
        return args_out
