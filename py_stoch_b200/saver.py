"""Writing simulation results to disk.

The reference writes one text file per output species with
``numpy.savetxt`` (``mod/utils/saver.py:6-52``): directory
``<cwd>/<sim_name>/x-<x0...>_c-<c...>/``, file name
``<sim_type>_species<k>_<Y-M-D-H-M>``, ``fmt='%1u'``, and a header naming
the output species, duration, time points, trajectories, initial state and
parameters (``make_header``, ``saver.py:55-65``).

:func:`save_results` keeps that directory layout, file naming and header.
``fmt='text'`` writes the reference's text files; the default
``fmt='npz'`` writes the same content as one binary ``.npz`` per call
(int32 ``samples [kappa, ita, U]`` plus the header fields as arrays),
which is exact, a fraction of the size and loads back with
:func:`load_results`.  :func:`save_batch` writes a whole batched run -- the
item table and, per item, the on-device summary statistics and Jacobians
(and, if kept, the samples and per-trajectory status / event counts) -- so
a sweep never needs its trajectories turned into text.
"""

import os
from datetime import datetime

import numpy


def _dir_name(arg_obj):
    """``x-<x0...>_c-<c...>`` (the reference's ``saver.py:19-33``)."""
    x0 = 'x'
    try:
        for v in arg_obj.x_0:
            x0 += '-' + str(v)
    except TypeError:
        x0 += '-' + str(arg_obj.x_0)
    c = '_c'
    try:
        for v in arg_obj.c:
            c += '-' + str(v).rstrip('.0')
    except TypeError:
        c += '-' + str(arg_obj.c).rstrip('.0')
    return x0 + c


def make_header(args):
    """The reference's text header (``saver.py:55-65``)."""
    return ('\noutput_species: {0}\nduration: {1}\nnum_output_time_points: '
            '{2}\nnum_simulations: {3}\nspecies_init: {4}\nparameters:{5}\n'
            ).format(str(args.E), str(args.t_max), str(args.ita),
                     str(args.U), str(args.x_0), str(args.c))


def _stamp(now=None):
    now = now or datetime.now()
    return '{0}-{1}-{2}-{3}-{4}'.format(now.year, now.month, now.day,
                                        now.hour, now.minute)


def save_results(sim_result, arg_obj, sim_name, sim_type='TL', fmt='npz',
                 root=None, now=None):
    """Write ``sim_result`` ([kappa, ita, U] int32, the layout ``run(args)``
    returns) for the sweep point ``arg_obj``; returns the written paths.

    ``fmt='text'``: one ``numpy.savetxt`` file per species, as the
    reference.  ``fmt='npz'``: one ``<sim_type>_<stamp>.npz``.  ``root``
    defaults to the current directory and ``now`` to the current time (the
    file-name stamp)."""
    out_dir = os.path.join(root or os.getcwd(), sim_name,
                           _dir_name(arg_obj))
    os.makedirs(out_dir, exist_ok=True)
    dt = _stamp(now)
    res = numpy.asarray(sim_result)
    paths = []
    if fmt == 'text':
        header = make_header(arg_obj)
        rows = res if res.ndim == 3 else numpy.moveaxis(res, 1, 0)
        for k in range(len(rows)):
            p = os.path.join(out_dir, '%s_species%d_%s' % (sim_type, k, dt))
            numpy.savetxt(p, rows[k], fmt='%1u', header=header)
            paths.append(p)
        return paths
    if fmt != 'npz':
        raise ValueError("fmt must be 'npz' or 'text'")
    p = os.path.join(out_dir, '%s_%s.npz' % (sim_type, dt))
    numpy.savez_compressed(
        p, samples=res.astype(numpy.int32, copy=False),
        output_species=numpy.asarray(arg_obj.E, numpy.int32),
        duration=numpy.float64(arg_obj.t_max),
        num_output_time_points=numpy.int64(arg_obj.ita),
        num_simulations=numpy.int64(arg_obj.U),
        species_init=numpy.asarray(arg_obj.x_0),
        parameters=numpy.asarray(arg_obj.c, numpy.float64))
    return [p]


def load_results(path):
    """Dict of the arrays :func:`save_results` (npz) or :func:`save_batch`
    wrote."""
    with numpy.load(path, allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


def save_batch(batch, path, samples=False):
    """Write a finished :class:`py_stoch_b200.batch.Batch` to ``path``
    (``.npz``): per item ``item<i>_stats`` [kappa, ita, 3] (mean, variance,
    lag-1 correlation), ``item<i>_jacobian`` [2, kappa, ita, R] when the
    batch computed them, ``item<i>_status`` / ``item<i>_events``, and with
    ``samples=True`` ``item<i>_samples`` [kappa, ita, n_traj]; plus the item
    table (``n_traj``, ``method``, ``mapping``, ``traj_id_base``,
    ``kappa``, ``ita``, ``n_reactions``)."""
    import torch
    torch.cuda.synchronize(batch.device)
    arrays = {'n_traj': batch.n_traj, 'method': batch.methods,
              'mapping': batch.mappings, 'traj_id_base': batch.traj_id_base,
              'kappa': batch.kappa, 'ita': batch.ita,
              'n_reactions': batch.R}
    out = batch.out
    for i in range(len(batch.models)):
        if 'stats' in out:
            arrays['item%d_stats' % i] = batch.stats(i).cpu().numpy()
        if 'jacobian' in out:
            arrays['item%d_jacobian' % i] = batch.jacobian(i).cpu().numpy()
        for k in ('status', 'events'):
            if k in out:
                arrays['item%d_%s' % (i, k)] = batch.per_traj(k, i).cpu(
                ).numpy()
        if samples:
            arrays['item%d_samples' % i] = batch.samples(i).cpu().numpy()
    numpy.savez_compressed(path, **arrays)
    return path
