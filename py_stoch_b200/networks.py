"""Reaction networks of the benchmark workloads, built directly as engine
models (no SBML file needed), plus the seeded generator of uneven synthetic
networks for batched runs.

* :func:`lotka_volterra` -- the network of ``examples/lotkaVoltera_sbml.xml``
  (species x, y and a catalyst a fixed at 1): a + x -> a + 2x (k1 x a),
  x + y -> 2y (k2 x y), y -> 0 (k3 y).
* :func:`schlogl` -- the network of ``examples/schlogl_sbmlv2.xml`` with the
  buffered species A, B folded into the rates: 2X -> 3X (c1/2 A X(X-1)),
  3X -> 2X (c2/6 X(X-1)(X-2)), 0 -> X (c3 B), X -> 0 (c4 X).
* :func:`telegraph` -- two-state gene expression (G_off, G_on, mRNA,
  protein).
* :func:`synthetic_networks` -- S ~ U[5,64], R ~ U[8,256] mass-action
  networks with 0-2 reactants / products of stoichiometry 1-2, rate
  constants log-uniform in [1e-3, 1e1], x0 ~ U{0..1000}, t_end log-uniform
  in [1, 100].
"""

import numpy as np

from .model import Model


def _times(t_end, n):
    return np.linspace(0, t_end, num=n).astype(np.float32)


def lotka_volterra(k1=10.0, k2=0.01, k3=10.0, x0=(1000, 1000, 1), t_end=10.0,
                   n_samples=100, out_species=(0, 1)):
    pre = np.array([[1, 1, 0],
                    [0, 1, 1],
                    [1, 0, 0]])
    post = np.array([[2, 0, 0],
                     [0, 2, 0],
                     [1, 0, 0]])
    m = Model.mass_action(pre, post, [k1, k2, k3], x0, _times(t_end, n_samples),
                          out_species, t_max=t_end)
    m.name = 'lotka_volterra'
    return m


SCHLOGL_NOMINAL = dict(c1=3e-7, c2=1e-4, c3=1e-3, c4=3.5, A=1e5, B=2e5)


def schlogl(c1=3e-7, c2=1e-4, c3=1e-3, c4=3.5, A=1e5, B=2e5, x0=250,
            t_end=5.0, n_samples=200):
    pre = np.array([[2, 3, 0, 1]])
    post = np.array([[3, 2, 1, 0]])
    # propensities c1/2 A X(X-1), c2/6 X(X-1)(X-2), c3 B, c4 X
    rate = [c1 * A / 2.0, c2 / 6.0, c3 * B, c4]
    m = Model(pre, pre, post - pre, rate, [x0], _times(t_end, n_samples), [0],
              hor=[3], hor_type=[3], t_max=t_end)
    m.name = 'schlogl'
    return m


TELEGRAPH_NOMINAL = (0.5, 0.2, 20.0, 1.0, 5.0, 0.1)


def telegraph(k=TELEGRAPH_NOMINAL, t_end=50.0, n_samples=20,
              out_species=(3,)):
    """Species (G_off, G_on, mRNA, protein), x0 = (1, 0, 0, 0); reactions
    off->on, on->off, on->on+mRNA, mRNA->0, mRNA->mRNA+protein,
    protein->0."""
    pre = np.array([[1, 0, 0, 0, 0, 0],
                    [0, 1, 1, 0, 0, 0],
                    [0, 0, 0, 1, 1, 0],
                    [0, 0, 0, 0, 0, 1]])
    post = np.array([[0, 1, 0, 0, 0, 0],
                     [1, 0, 1, 0, 0, 0],
                     [0, 0, 1, 0, 1, 0],
                     [0, 0, 0, 0, 1, 0]])
    m = Model.mass_action(pre, post, k, [1, 0, 0, 0], _times(t_end, n_samples),
                          out_species, t_max=t_end)
    m.name = 'telegraph'
    return m


def synthetic_networks(n_networks, seed=0, s_range=(5, 64), r_range=(8, 256),
                       n_samples=50, k_range=(1e-3, 1e1), x0_max=1000,
                       t_range=(1.0, 100.0)):
    """Seeded uneven mass-action networks (list of :class:`Model`).

    Per network: S ~ U{s_range}, R ~ U{r_range}; each reaction draws 0-2
    distinct reactant species and 0-2 distinct product species, each with
    stoichiometry 1 or 2; rate constants log-uniform in k_range (stochastic
    mass action k * prod C(x_i, n_i)); x0 ~ U{0..x0_max}; t_end log-uniform
    in t_range; all species recorded at n_samples times."""
    rng = np.random.default_rng(seed)
    lk0, lk1 = np.log(k_range[0]), np.log(k_range[1])
    lt0, lt1 = np.log(t_range[0]), np.log(t_range[1])
    out = []
    for _ in range(n_networks):
        S = int(rng.integers(s_range[0], s_range[1] + 1))
        R = int(rng.integers(r_range[0], r_range[1] + 1))
        mats = []
        for _side in range(2):
            n = rng.integers(0, 3, R)                      # species per side
            order = np.argsort(rng.random((R, S)), axis=1)[:, :2]
            st = rng.integers(1, 3, (R, 2))
            mat = np.zeros((S, R), np.int64)
            cols = np.arange(R)
            for q in range(2):
                use = n > q
                mat[order[use, q], cols[use]] = st[use, q]
            mats.append(mat)
        pre, post = mats
        k = np.exp(rng.uniform(lk0, lk1, R))
        x0 = rng.integers(0, x0_max + 1, S)
        t_end = float(np.exp(rng.uniform(lt0, lt1)))
        m = Model.mass_action(pre, post, k, x0, _times(t_end, n_samples),
                              np.arange(S), t_max=t_end)
        m.name = 'synthetic'
        out.append(m)
    return out


LV_NOMINAL = (10.0, 0.01, 10.0)


def parameter_sweep(n_sets, seed=1, n_samples=50, lv_t_end=10.0,
                    schlogl_t_end=5.0):
    """Parameter sets drawn log-uniformly within one decade of the
    Lotka-Volterra (k1, k2, k3) and Schlogl (c1..c4; A, B fixed) nominal
    values, half of each (Lotka-Volterra first), as engine models with
    n_samples sample times up to t_end = 10 (Lotka-Volterra) / 5 (Schlogl).
    Returns (models, log_factors): log_factors[i] is the log of the
    set's rates relative to the nominal ones."""
    rng = np.random.default_rng(seed)
    n_lv = n_sets // 2
    out, logf = [], []
    for i in range(n_sets):
        if i < n_lv:
            f = rng.uniform(-np.log(10), np.log(10), 3)
            k = np.array(LV_NOMINAL) * np.exp(f)
            m = lotka_volterra(k1=k[0], k2=k[1], k3=k[2], t_end=lv_t_end,
                               n_samples=n_samples)
        else:
            f = rng.uniform(-np.log(10), np.log(10), 4)
            c = np.array([SCHLOGL_NOMINAL[n] for n in ('c1', 'c2', 'c3', 'c4')
                          ]) * np.exp(f)
            m = schlogl(c1=c[0], c2=c[1], c3=c[2], c4=c[3],
                        t_end=schlogl_t_end, n_samples=n_samples)
        out.append(m)
        logf.append(f)
    return out, logf
