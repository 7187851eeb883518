"""Exact first and second moments of first-order (linear) reaction networks
(test infrastructure: an FP64 reference for means, variances and their
gradients in log rate constants).

For propensities a_j(x) = c_j * x_{i_j} (or c_j for zero order) with net
change v_j, the moments close:

    dm/dt   = sum_j v_j E[a_j]
    dM2/dt  = sum_j E[a_j (v_j x^T + x v_j^T)] + v_j v_j^T E[a_j]

with E[a_j x] = c_j M2[:, i_j] (first order) or c_j m (zero order).
Integrated with scipy's solve_ivp at tight tolerances; gradients by central
differences of the ODE solution in log c (FP64, h = 1e-5).
"""

import numpy as np
from scipy.integrate import solve_ivp


def _linear_structure(model):
    S, R = model.order.shape
    reactant = np.full(R, -1)
    for j in range(R):
        tot = int(model.order[:, j].sum())
        if tot > 1:
            raise ValueError('reaction %d is not first order' % j)
        if tot == 1:
            reactant[j] = int(np.argmax(model.order[:, j]))
    return reactant


def moments(model, rates=None, times=None):
    """(mean [S, T], var [S, T]) at `times` (default: the sample times)."""
    c = np.asarray(model.rate if rates is None else rates, np.float64)
    times = np.asarray(model.sample_times if times is None else times,
                       np.float64)
    S, R = model.order.shape
    V = model.net.astype(np.float64)
    reactant = _linear_structure(model)

    def rhs(_, y):
        m = y[:S]
        M2 = y[S:].reshape(S, S)
        dm = np.zeros(S)
        dM = np.zeros((S, S))
        for j in range(R):
            v = V[:, j]
            if reactant[j] >= 0:
                i = reactant[j]
                Ea = c[j] * m[i]
                Eax = c[j] * M2[:, i]
            else:
                Ea = c[j]
                Eax = c[j] * m
            dm += v * Ea
            dM += np.outer(v, Eax) + np.outer(Eax, v) + np.outer(v, v) * Ea
        return np.concatenate([dm, dM.ravel()])

    x0 = model.x0.astype(np.float64)
    y0 = np.concatenate([x0, np.outer(x0, x0).ravel()])
    sol = solve_ivp(rhs, (0.0, float(times[-1])), y0, t_eval=times,
                    method='LSODA', rtol=1e-11, atol=1e-9)
    if not sol.success:
        raise RuntimeError(sol.message)
    m = sol.y[:S]
    M2 = sol.y[S:].reshape(S, S, -1)
    var = np.stack([M2[i, i] for i in range(S)]) - m * m
    return m, var


def moment_gradients(model, h=1e-5):
    """d mean / d log c_j and d var / d log c_j: arrays [R, S, T]."""
    c = model.rate.astype(np.float64)
    R = len(c)
    gm, gv = [], []
    for j in range(R):
        up = c.copy()
        dn = c.copy()
        up[j] *= np.exp(h)
        dn[j] *= np.exp(-h)
        mu, vu = moments(model, up)
        md, vd = moments(model, dn)
        gm.append((mu - md) / (2 * h))
        gv.append((vu - vd) / (2 * h))
    return np.array(gm), np.array(gv)
