"""Stochastic Petri net built from an SBML model.

Python 3 restatement of ``mod/petri_net/SPN.py`` (reference).  Produces the
same fields with the same meaning:

* ``Pre`` / ``Post``: float arrays [species][reaction] of reactant / product
  stoichiometries (``SPN.py:72-97``);
* ``StoichMConst``: 1 where the species is declared constant (``SPN.py:93-94``);
* ``M``: initial amounts (``SPN.py:100-104``), ``c``: parameter values
  (``SPN.py:145-150``);
* ``P``: ``{"species_i": i}``, ``T``: ``{reaction_id: j}`` (``SPN.py:47-62``);
* ``h``: kinetic-law strings with species ids rewritten to ``species_i`` and
  global parameter ids to ``parameter_k`` (``SPN.py:107-142``).

The SBML model may be a :mod:`py_stoch_b200.sbml` model, a real libsbml model,
or a path to an SBML file.
"""

import copy

import numpy as np

from . import sbml as _sbml


class SPN(object):
    def __init__(self):
        self.Pre = []
        self.Post = []
        self.M = []
        self.h = []
        self.c = []
        self.P = {}
        self.T = {}
        self.StoichMConst = []

    def sbml_2_stochastic_petri_net(self, sbml_model):
        """Fill every field from ``sbml_model`` (``SPN.py:17-45``)."""
        if isinstance(sbml_model, str):
            sbml_model = _sbml.read_sbml(sbml_model)
        self.Pre, self.Post, self.StoichMConst = self.get_stoichiometries(
            sbml_model)
        self.M = self.get_initial_state_vector(sbml_model)
        self.c = self.get_rate_constants_vector(sbml_model)
        constants = self.get_rate_constants(sbml_model)
        self.P = self.get_species_vector(sbml_model)
        self.T = self.get_reactions_vector(sbml_model)
        self.h = self.get_hazards_vector(sbml_model, self.P, constants)
        return self

    @staticmethod
    def get_species_vector(sbml_model):
        return {'species_%d' % i: i
                for i, _ in enumerate(sbml_model.getListOfSpecies())}

    @staticmethod
    def get_reactions_vector(sbml_model):
        return {r.getId(): j
                for j, r in enumerate(sbml_model.getListOfReactions())}

    @staticmethod
    def get_rate_constants(sbml_model):
        return {p.getId(): k
                for k, p in enumerate(sbml_model.getListOfParameters())}

    @staticmethod
    def get_stoichiometries(sbml_model):
        species = list(sbml_model.getListOfSpecies())
        reactions = list(sbml_model.getListOfReactions())
        pre = np.zeros([len(species), len(reactions)])
        post = np.zeros_like(pre)
        const = np.zeros_like(pre)
        for j, reaction in enumerate(reactions):
            # a species listed twice keeps its last stoichiometry, as the
            # dict comprehension at SPN.py:78-81 does
            reactants = {r.getSpecies(): r.getStoichiometry()
                         for r in reaction.getListOfReactants()}
            products = {p.getSpecies(): p.getStoichiometry()
                        for p in reaction.getListOfProducts()}
            for i, sp in enumerate(species):
                sid = sp.getId()
                if sid in reactants:
                    pre[i, j] = int(reactants.get(sid, 0))
                if sid in products:
                    post[i, j] = int(products.get(sid, 0))
                if sp.getConstant():
                    const[i, j] = 1
        return pre, post, const

    @staticmethod
    def get_initial_state_vector(sbml_model):
        return [sp.getInitialAmount() for sp in sbml_model.getListOfSpecies()]

    @staticmethod
    def get_hazards_vector(sbml_model, species_dict, param_dict):
        h = []
        for reaction in sbml_model.getListOfReactions():
            math = reaction.getKineticLaw().getMath()
            math = (math.deepCopy() if hasattr(math, 'deepCopy')
                    else copy.deepcopy(math))
            math = SPN.replace_hazard_species(math, sbml_model)
            math = SPN.replace_hazard_parameter(math, param_dict)
            h.append(_to_string(math))
        return h

    @staticmethod
    def replace_hazard_species(mathml, sbml_model):
        """Rename species ids to ``species_i`` (post-order, ``SPN.py:120-130``)."""
        for i in range(mathml.getNumChildren()):
            SPN.replace_hazard_species(mathml.getChild(i), sbml_model)
        if mathml.getType() == _name_type(mathml):
            for idx, sp in enumerate(sbml_model.getListOfSpecies()):
                if sp.getId() == mathml.getName():
                    mathml.setName('species_%d' % idx)
                    break
        return mathml

    @staticmethod
    def replace_hazard_parameter(mathml, params_dict):
        """Rename global parameter ids to ``parameter_k`` (``SPN.py:133-142``)."""
        for i in range(mathml.getNumChildren()):
            SPN.replace_hazard_parameter(mathml.getChild(i), params_dict)
        if mathml.getType() == _name_type(mathml):
            for param, idx in params_dict.items():
                if param == mathml.getName():
                    mathml.setName('parameter_%d' % idx)
                    break
        return mathml

    @staticmethod
    def get_rate_constants_vector(sbml_model):
        return [p.getValue() for p in sbml_model.getListOfParameters()]


def _name_type(node):
    """AST_NAME of whichever library built ``node``."""
    if isinstance(node, _sbml.ASTNode):
        return _sbml.AST_NAME
    import libsbml  # a real libsbml tree
    return libsbml.AST_NAME


def _to_string(node):
    if isinstance(node, _sbml.ASTNode):
        return _sbml.formulaToL3String(node)
    import libsbml
    return libsbml.formulaToL3String(node)
