"""Engine model: a mass-action reaction network in dense form, and its
packing into the device blob.

The reference evaluates each kinetic law as generated C code
(``Parser.define_hazards``, ``mod/parser/parser.py:32-55``).  The engine
instead evaluates every propensity in one generic form,

    a_j(x) = k_j * prod_i prod_{m < n_ij} (x_i - m * falling_ij)     (FP32)

and :func:`analyse_hazard` finds ``k_j``, ``n_ij`` and ``falling_ij`` for a
kinetic-law string by symbolic division (SymPy): the law must equal
``k_j`` (free of species) times a falling-factorial or power product of
species.  All six SBML fixtures of the reference reduce to this form
(``c1/2*a*X*(X-1)`` -> k = c1*a/2 with X of falling order 2).  Other laws
raise :class:`UnsupportedKineticLaw`.
"""

import functools
import math

import numpy as np
import sympy

from . import _lib


class UnsupportedKineticLaw(ValueError):
    pass


_SYMPY_LOCALS = {'exponentiale': sympy.E, 'pi': sympy.pi, 'ln': sympy.log,
                 'exp': sympy.exp, 'abs': sympy.Abs, 'floor': sympy.floor,
                 'ceiling': sympy.ceiling}


@functools.lru_cache(maxsize=4096)
def analyse_hazard(hazard, pre_col, n_species):
    """Split a kinetic-law string into (orders, falling, rate expression).

    ``hazard`` uses the ``species_i`` / ``parameter_k`` names of
    ``SPN.h``; ``pre_col`` is the reaction's column of ``Pre``.  Returns
    ``(orders tuple, falling tuple, sympy rate expression in parameter_k)``.
    """
    sp = [sympy.Symbol('species_%d' % i) for i in range(n_species)]
    loc = dict(_SYMPY_LOCALS)
    loc.update({str(s): s for s in sp})
    try:
        expr = sympy.sympify(hazard.replace('^', '**'), locals=loc)
    except (sympy.SympifyError, SyntaxError, TypeError) as e:
        raise UnsupportedKineticLaw('cannot parse kinetic law %r: %s'
                                    % (hazard, e))
    present = [i for i in range(n_species) if sp[i] in expr.free_symbols]
    spset = set(sp)
    candidates = []
    pre_orders = tuple(int(v) for v in pre_col)
    candidates.append((pre_orders, True))
    degs = [0] * n_species
    poly_ok = True
    for i in present:
        try:
            degs[i] = int(sympy.degree(expr, sp[i]))
        except (sympy.PolynomialError, ValueError, TypeError):
            poly_ok = False
    if poly_ok:
        candidates.append((tuple(degs), True))
        candidates.append((tuple(degs), False))
    for orders, falling in candidates:
        ff = sympy.Integer(1)
        for i, n in enumerate(orders):
            for m in range(n):
                ff = ff * (sp[i] - m if falling else sp[i])
        ratio = sympy.cancel(expr / ff)
        if not (ratio.free_symbols & spset):
            return (orders, tuple([1 if falling else 0] * n_species), ratio)
    raise UnsupportedKineticLaw(
        'kinetic law %r is not of mass-action form k * prod(x_i falling or '
        'power orders)' % hazard)


def _eval_rate(ratio, c):
    subs = {sympy.Symbol('parameter_%d' % k): float(v)
            for k, v in enumerate(c)}
    val = ratio.subs(subs)
    free = val.free_symbols
    if free:
        raise UnsupportedKineticLaw('kinetic law refers to unknown names %s'
                                    % sorted(str(s) for s in free))
    return float(val)


class Model(object):
    """Dense model (the fields of ``pyst_model_desc``).

    Arrays: order/falling/pre/net [S, R]; rate [R] (float64, rounded to
    FP32 by the packer); x0, hor, hor_type [S]; sample_times [ita] float32;
    out_species [kappa].  ``laws``: None, or per reaction None (mass action)
    or the (code, constants) program of a general kinetic law
    (:func:`py_stoch_b200.kinetic.compile_law`); a reaction with a law
    ignores its order column and rate.
    """

    def __init__(self, order, pre, net, rate, x0, sample_times, out_species,
                 hor=None, hor_type=None, falling=None, t_max=None, eta=0.03,
                 n_c=10, name='', laws=None):
        self.order = np.ascontiguousarray(order, dtype=np.int32)
        S, R = self.order.shape
        self.pre = np.ascontiguousarray(pre, dtype=np.int32).reshape(S, R)
        self.net = np.ascontiguousarray(net, dtype=np.int32).reshape(S, R)
        self.falling = (np.ones((S, R), np.uint8) if falling is None else
                        np.ascontiguousarray(falling, np.uint8).reshape(S, R))
        self.rate = np.ascontiguousarray(rate, dtype=np.float64).reshape(R)
        self.x0 = np.ascontiguousarray(x0, dtype=np.int32).reshape(S)
        self.sample_times = np.ascontiguousarray(sample_times,
                                                 dtype=np.float32).ravel()
        self.out_species = np.ascontiguousarray(out_species,
                                                dtype=np.int32).ravel()
        self.laws = None
        if laws is not None and any(l is not None for l in laws):
            if len(laws) != R:
                raise ValueError('laws must have one entry per reaction')
            self.laws = list(laws)
        if hor is None or hor_type is None:
            order_h = self.order.copy()
            for j in self.law_reactions():
                order_h[:, j] = self.pre[:, j]
            hor, hor_type = derive_hors(self.pre, order_h)
        self.hor = np.ascontiguousarray(hor, dtype=np.int32).reshape(S)
        self.hor_type = np.ascontiguousarray(hor_type,
                                             dtype=np.int32).reshape(S)
        self.t_max = (float(self.sample_times[-1]) if t_max is None
                      else float(t_max))
        self.eta = float(eta)
        self.n_c = int(n_c)
        self.name = name
        self._blob = None

    def law_reactions(self):
        """Indices of the reactions with a general kinetic law."""
        if self.laws is None:
            return []
        return [j for j, l in enumerate(self.laws) if l is not None]

    @property
    def has_laws(self):
        return self.laws is not None

    @property
    def n_species(self):
        return self.order.shape[0]

    @property
    def n_reactions(self):
        return self.order.shape[1]

    @property
    def kappa(self):
        return len(self.out_species)

    @property
    def ita(self):
        return len(self.sample_times)

    # ---- constructors ---------------------------------------------------
    @classmethod
    def from_tl_args(cls, args):
        """Engine model of a parsed :class:`~py_stoch_b200.parser.TlArgs`
        (or ``GArgs``)."""
        if args.pre_matrix is None or args.hazard_exprs is None:
            raise ValueError('args were not produced by TlParser.parse / '
                             'GParser.parse of this package')
        pre = np.asarray(args.pre_matrix, dtype=np.int64)
        post = np.asarray(args.post_matrix, dtype=np.int64)
        S, R = pre.shape
        order = np.zeros((S, R), np.int32)
        falling = np.ones((S, R), np.uint8)
        rate = np.zeros(R, np.float64)
        laws = [None] * R
        from .kinetic import has_int_division
        n_par = len(np.ravel(args.c))
        for j, hz in enumerate(args.hazard_exprs):
            try:
                if has_int_division(hz, S, n_par):
                    raise UnsupportedKineticLaw('integer division')
                o, fl, ratio = analyse_hazard(
                    hz, tuple(int(v) for v in pre[:, j]), S)
                r = _eval_rate(ratio, args.c)
            except UnsupportedKineticLaw:
                # not k * prod(x_i falling or power): compile the law as
                # the reference would evaluate it (C typing, FP64)
                from .kinetic import compile_law, KineticLawError
                try:
                    code, consts, _ = compile_law(
                        hz, S, [float(v) for v in np.ravel(args.c)])
                except KineticLawError as e:
                    raise UnsupportedKineticLaw(str(e))
                laws[j] = (code, consts)
                continue
            order[:, j] = o
            falling[:, j] = fl
            rate[j] = r
        hor = getattr(args, 'H', None)
        hor_type = getattr(args, 'H_type', None)
        if hor is None or len(hor) != S:
            hor, hor_type = derive_hors(pre, order)
        return cls(order, pre, post - pre, rate, args.x_0, args.I, args.E,
                   hor=hor, hor_type=hor_type, falling=falling,
                   t_max=args.t_max, eta=getattr(args, 'eta', 0.03),
                   n_c=getattr(args, 'n_c', 10), laws=laws)

    @classmethod
    def mass_action(cls, pre, post, k, x0, sample_times, out_species=None,
                    combinatorial=True, **kw):
        """Network with propensity k_j * prod_i C(x_i, pre_ij) (the usual
        stochastic mass action; ``combinatorial=False`` drops the 1/n!)."""
        pre = np.asarray(pre, dtype=np.int64)
        post = np.asarray(post, dtype=np.int64)
        S, R = pre.shape
        k = np.asarray(k, dtype=np.float64).reshape(R)
        if combinatorial:
            if pre.max(initial=0) > 20:
                raise ValueError('stoichiometry above 20')
            fact = np.array([math.factorial(n) for n in range(21)],
                            dtype=np.float64)
            k = k / fact[pre].prod(axis=0)
        if out_species is None:
            out_species = np.arange(S)
        return cls(pre, pre, post - pre, k, x0, sample_times, out_species,
                   **kw)

    # ---- packing --------------------------------------------------------
    def desc(self):
        """``pyst_model_desc`` pointing into this model's arrays."""
        import ctypes as C
        d = _lib.ModelDesc()
        d.n_species = self.n_species
        d.n_reactions = self.n_reactions
        d.order = self.order.ctypes.data
        d.falling = self.falling.ctypes.data
        d.pre = self.pre.ctypes.data
        d.net_change = self.net.ctypes.data
        d.rate = self.rate.ctypes.data
        d.x0 = self.x0.ctypes.data
        d.hor = self.hor.ctypes.data
        d.hor_type = self.hor_type.ctypes.data
        d.sample_times = self.sample_times.ctypes.data
        d.n_samples = self.ita
        d.out_species = self.out_species.ctypes.data
        d.n_out = self.kappa
        d.t_max = self.t_max
        d.eta = C.c_float(self.eta).value
        d.n_c = self.n_c
        if self.laws is not None:
            ptr, code, consts = self.law_arrays()
            d.law_ptr = ptr.ctypes.data
            d.law_code = code.ctypes.data if code.size else None
            d.law_const = consts.ctypes.data if consts.size else None
            d.n_law_const = int(consts.size)
        return d

    def law_arrays(self):
        """(law_ptr int32 [R+1], law_code uint32, law_const float64) of the
        kinetic-law programs, constants pooled (kept alive on the model)."""
        if getattr(self, '_law_arrays', None) is None:
            from .kinetic import OP_C
            ptr, code, consts = [0], [], []
            for law in (self.laws or [None] * self.n_reactions):
                if law is not None:
                    c, k = law
                    base = len(consts)
                    for wd in np.asarray(c, dtype=np.uint32):
                        wd = int(wd)
                        if wd >> 24 == OP_C:
                            wd = (OP_C << 24) | ((wd & 0xFFFFFF) + base)
                        code.append(wd)
                    consts.extend(float(v) for v in np.ravel(k))
                ptr.append(len(code))
            self._law_arrays = (np.asarray(ptr, dtype=np.int32),
                                np.asarray(code, dtype=np.uint32),
                                np.asarray(consts, dtype=np.float64))
        return self._law_arrays

    def blob(self):
        """Packed device blob (np.uint32, length a multiple of 4)."""
        if self._blob is None:
            import ctypes as C
            L = _lib.lib()
            d = self.desc()
            n = C.c_int64(0)
            _lib.check(L.pyst_model_blob_words(C.byref(d), C.byref(n)),
                       'pyst_model_blob_words')
            out = np.zeros(n.value, dtype=np.uint32)
            _lib.check(L.pyst_model_build(C.byref(d), out.ctypes.data,
                                          n.value), 'pyst_model_build')
            self._blob = out
        return self._blob

    def with_rates(self, rate):
        """Copy of the model with other rate constants."""
        m = Model(self.order, self.pre, self.net, rate, self.x0,
                  self.sample_times, self.out_species, hor=self.hor,
                  hor_type=self.hor_type, falling=self.falling,
                  t_max=self.t_max, eta=self.eta, n_c=self.n_c,
                  name=self.name, laws=self.laws)
        return m

    def with_x0(self, x0):
        return Model(self.order, self.pre, self.net, self.rate, x0,
                     self.sample_times, self.out_species, hor=self.hor,
                     hor_type=self.hor_type, falling=self.falling,
                     t_max=self.t_max, eta=self.eta, n_c=self.n_c,
                     name=self.name, laws=self.laws)


def derive_hors(pre, order):
    """H (highest total order of a reaction the species takes part in as a
    reactant) and H_type (its largest reactant stoichiometry), the quantities
    of ``TlParser.get_hors`` (``mod/parser/tl_parser.py:98-120``) for a law
    that mentions exactly its reactants."""
    pre = np.asarray(pre)
    order = np.asarray(order)
    tot = order.sum(axis=0)
    mask = order > 0
    hor = np.where(mask, tot[None, :], 0).max(axis=1, initial=0)
    hty = np.where(mask, pre, 0).max(axis=1, initial=0)
    return hor.astype(np.int32), hty.astype(np.int32)
