"""Seeded synthetic choice data: the workloads this library is measured and tested on.

Every generator draws from ``numpy.random.default_rng(seed)`` in a fixed order, so an instance
is reproducible from its arguments alone.

mixture_instance   menus of the subset lattice kept with probability ``density``; p(a | M) from a
                   Dirichlet(1)-weighted mixture of K uniformly random linear orders (the weight of
                   the orders whose top member of M is a); every menu resampled as
                   Multinomial(N, p(. | M)) / N, one row per member (zero rows kept).
panel_instance     a respondent panel: R respondents each answer ``per_respondent`` distinct
                   menus drawn uniformly from the kept menus, each choosing with one order drawn
                   from the mixture; rows are counted from the panel.
dsr_instance       ``n_menus`` distinct random menus that all contain alternative 0, sizes uniform
                   on 2..n; R respondents answer every menu; only alternative 0 is observed.

Rows are ``(menu bitmask, chosen alternative, p_hat)``, menus ascending and members ascending
within a menu, as the reference's data generators and ``cells_from_panel`` order them
(data/gen_instances.py:79-106, solver/inference/draws.py:104-126).
"""
import numpy as np

__all__ = ["mixture_instance", "panel_instance", "dsr_instance", "rows_of", "top_of_orders",
           "cells_from_panel", "CONFIGS", "config_instance"]


def _popcount(a):
    a = np.asarray(a, dtype=np.uint64)
    c = np.zeros(a.shape, dtype=np.int64)
    for b in range(64):
        c += ((a >> np.uint64(b)) & np.uint64(1)).astype(np.int64)
        if not (a >> np.uint64(b + 1)).any():
            break
    return c


def top_of_orders(n, menus, orders):
    """(U, K) array: the top member of each menu under each order (orders: (K, n) permutations,
    best first)."""
    menus = np.asarray(menus, dtype=np.int64)
    memb = ((menus[:, None] >> np.arange(n)[None, :]) & 1).astype(bool)          # (U, n)
    pos = np.empty_like(orders)
    K = orders.shape[0]
    pos[np.arange(K)[:, None], orders] = np.arange(n)[None, :]                   # rank of each alt
    big = np.where(memb[:, None, :], pos[None, :, :], n + 1)                     # (U, K, n)
    return np.argmin(big, axis=2)


def _mixture(rng, n, K):
    orders = np.stack([rng.permutation(n) for _ in range(K)])
    weights = rng.dirichlet(np.ones(K))
    return orders, weights


def rows_of(n, menus, p_menu):
    """Rows (menu, member, p) for every menu and member, members ascending."""
    menus = np.asarray(menus, dtype=np.int64)
    memb = ((menus[:, None] >> np.arange(n)[None, :]) & 1).astype(bool)
    j, a = np.nonzero(memb)
    return menus[j], a.astype(np.int64), np.asarray(p_menu)[j, a]


def mixture_instance(n, density, K, N, seed=0, min_size=2):
    """(menu, alternative, p_hat) of the mixture-of-orders generator; see the module docstring.

    density = 1 keeps every menu with at least ``min_size`` members."""
    rng = np.random.default_rng(seed)
    masks = np.arange(1 << n, dtype=np.int64)
    size = _popcount(masks)
    keep = size >= min_size
    if density < 1.0:
        keep &= rng.random(masks.size) < density
    menus = masks[keep]
    orders, weights = _mixture(rng, n, K)
    top = top_of_orders(n, menus, orders)                                       # (U, K)
    p = np.zeros((menus.size, n))
    np.add.at(p, (np.repeat(np.arange(menus.size), K), top.reshape(-1)), np.tile(weights, menus.size))
    p /= p.sum(axis=1, keepdims=True)
    counts = rng.multinomial(N, p)
    return rows_of(n, menus, counts / float(N))


def cells_from_panel(n, menu, chosen, alternatives=None):
    """Rows counted from one row per choice: p_hat(D, a) = #(D, a) / #D, menus ascending and
    alternatives ascending within a menu; alternatives restricts the observed members
    (solver/inference/draws.py:104-126)."""
    menu = np.asarray(menu, dtype=np.int64)
    chosen = np.asarray(chosen, dtype=np.int64)
    menus, inv, den = np.unique(menu, return_inverse=True, return_counts=True)
    alts = np.arange(n) if alternatives is None else np.unique(np.asarray(alternatives, dtype=np.int64))
    j, k = np.nonzero((menus[:, None] >> alts[None, :]) & 1)
    num = np.bincount(inv * n + chosen, minlength=menus.size * n)
    return menus[j], alts[k], num[j * n + alts[k]] / den[j]


def panel_instance(n, density, respondents, per_respondent, K, seed=0):
    """A respondent panel over the menus of ``density``: returns (panel dict with columns
    respondent, menu, chosen; (menu, alternative, p_hat) rows counted from it)."""
    rng = np.random.default_rng(seed)
    masks = np.arange(1 << n, dtype=np.int64)
    keep = (_popcount(masks) >= 2) & (rng.random(masks.size) < density)
    pool = masks[keep]
    orders, weights = _mixture(rng, n, K)
    resp, menu, chosen = [], [], []
    for i in range(respondents):
        ms = pool[rng.choice(pool.size, size=per_respondent, replace=False)]
        k = rng.choice(K, p=weights)
        top = top_of_orders(n, ms, orders[k:k + 1])[:, 0]
        resp.append(np.full(per_respondent, i))
        menu.append(ms)
        chosen.append(top)
    panel = dict(respondent=np.concatenate(resp), menu=np.concatenate(menu), chosen=np.concatenate(chosen))
    return panel, cells_from_panel(n, panel["menu"], panel["chosen"])


def dsr_instance(n, n_menus, respondents, K, seed=0):
    """The alternative-0 panel: ``n_menus`` distinct menus containing 0, sizes uniform on 2..n,
    every respondent answers every menu; rows observe alternative 0 only."""
    rng = np.random.default_rng(seed)
    seen, menus = set(), []
    while len(menus) < n_menus:
        s = int(rng.integers(2, n + 1))
        others = rng.choice(np.arange(1, n), size=s - 1, replace=False)
        m = 1 | int(np.sum(np.int64(1) << others.astype(np.int64)))
        if m not in seen:
            seen.add(m)
            menus.append(m)
    menus = np.array(sorted(menus), dtype=np.int64)
    orders, weights = _mixture(rng, n, K)
    which = rng.choice(K, size=respondents, p=weights)
    top = top_of_orders(n, menus, orders)                                       # (U, K)
    resp = np.repeat(np.arange(respondents), menus.size)
    menu = np.tile(menus, respondents)
    chosen = top[np.tile(np.arange(menus.size), respondents), np.repeat(which, menus.size)]
    panel = dict(respondent=resp, menu=menu, chosen=chosen)
    return panel, cells_from_panel(n, menu, chosen, alternatives=[0])


# The measured workloads, by what they are.
CONFIGS = {
    "n10_all_k20": dict(kind="mixture", n=10, density=1.0, K=20, N=200),
    "n18_d1pct_k50": dict(kind="mixture", n=18, density=0.01, K=50, N=500),
    "n18_d05pct_k50": dict(kind="mixture", n=18, density=0.005, K=50, N=500),
    "n20_d1pct_panel520": dict(kind="panel", n=20, density=0.01, respondents=520, per_respondent=30, K=30),
    "n25_dsr301_panel520": dict(kind="dsr", n=25, n_menus=301, respondents=520, K=40),
}


def config_instance(name, seed=0):
    """(n, menu, alternative, p_hat[, panel]) of a named workload."""
    c = dict(CONFIGS[name])
    kind = c.pop("kind")
    n = c["n"]
    if kind == "mixture":
        return (n,) + mixture_instance(seed=seed, **c)
    if kind == "panel":
        panel, rows = panel_instance(seed=seed, **c)
        return (n,) + rows + (panel,)
    panel, rows = dsr_instance(seed=seed, **c)
    return (n,) + rows + (panel,)
