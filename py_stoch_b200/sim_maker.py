"""Sweep builder: one :class:`~py_stoch_b200.parser.TlArgs` per combination
of initial states and parameter values.

Python 3 restatement of the reference's ``sim_maker.py``.  Same call
signature and the same ordering of combinations (initial-state lists outer,
parameter lists inner, ``sim_maker.py:13-23``), so ``make_list(...)[i]``
is the same sweep point in both.  Unlike the reference, the SBML model is
turned into a Petri net once and copied per combination instead of being
re-read (``sim_maker.py:25-27``); the resulting fields are identical.
"""

import copy

import numpy

from .parser import TlArgs, TlParser
from .petri_net import SPN


class TLArgsList(object):
    @staticmethod
    def make_list(sbml_model, sweep_species_init, sweep_params,
                  output_species, duration, num_output_time_points,
                  num_simulations, gillespie=0):
        """Cartesian product of the sweeps (``sim_maker.py:7-43``)."""
        species_init_lists = rest_list(sweep_species_init)
        param_lists = rest_list(sweep_params)

        sim_objects = []
        for species_init_list in species_init_lists:
            for param_list in param_lists:
                obj = SimObj()
                obj.species_init = species_init_list
                obj.params = param_list
                sim_objects.append(obj)

        base = SPN()
        base.sbml_2_stochastic_petri_net(sbml_model)

        tl_args_list = []
        for obj in sim_objects:
            spn = copy.deepcopy(base)
            spn.M = numpy.array(obj.species_init).astype(numpy.int32)
            spn.c = numpy.array(obj.params).astype(numpy.float64)

            tl_args = TlArgs()
            tl_args.E = numpy.array(output_species).astype(numpy.int32)
            tl_args.t_max = duration
            tl_args.ita = num_output_time_points
            tl_args.U = num_simulations
            tl_args.gillespie = gillespie
            tl_args = TlParser.parse(tl_args, spn)
            tl_args_list.append(tl_args)
        return tl_args_list


def rest_list(list_in, index=0):
    """Recursive Cartesian product of a list of value lists
    (``sim_maker.py:46-64``).

    As in the reference, the innermost level returns the last value list
    itself, so a single-species sweep yields bare values rather than
    one-element lists.
    """
    if index == len(list_in) - 1:
        return list_in[index]
    sub_lists = rest_list(list_in, index + 1)
    out = []
    for head in list_in[index]:
        for sub in sub_lists:
            out.append([head] + sub if isinstance(sub, list)
                       else [head] + [sub])
    return out


class SimObj(object):
    def __init__(self):
        self.species_init = []
        self.params = []
