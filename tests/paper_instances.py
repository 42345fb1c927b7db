"""The reference's paper instances, regenerated for the tests (data/gen_instances.py:37-152).

The reference certified distance brackets on these exact instances (data/opt_refs.json); the
generators are restated here so that the same bytes come out (legacy RandomState streams, which
numpy keeps stable), and the tests check every regenerated instance against the sha256
fingerprint the reference stores for it."""
import hashlib

import numpy as np


def gen_pairwise(n, phat_seed=100):
    rng = np.random.RandomState(phat_seed)
    rows = []
    for i in range(n):
        for j in range(i + 1, n):
            g = rng.rand(2)
            g = g / g.sum()
            mask = (1 << i) | (1 << j)
            rows.append((mask, i, float(g[0])))
            rows.append((mask, j, float(g[1])))
    cd = np.array(rows, dtype=np.float64)
    return cd, len(rows)


def gen_medium(n, mult=20, menu_seed=42, phat_seed=100):
    target = mult * n * (n - 1)
    rng = np.random.RandomState(menu_seed)
    seen, menus, mp = set(), [], 0
    while mp < target:
        m = int(rng.randint(0, 1 << n))
        if m in seen:
            continue
        k = bin(m).count("1")
        if k < 2:
            continue
        seen.add(m)
        menus.append(m)
        mp += k
    prng = np.random.RandomState(phat_seed)
    rows = []
    for m in menus:
        items = [i for i in range(n) if (m >> i) & 1]
        g = prng.rand(len(items))
        g = g / g.sum()
        for kk, x in enumerate(items):
            rows.append((m, x, float(g[kk])))
    cd = np.array(rows, dtype=np.float64)
    return cd, len(rows)


def p_inside(cd):
    cd = np.array(cd, dtype=np.float64, copy=True)
    sizes = np.array([bin(int(m)).count("1") for m in cd[:, 0]], dtype=np.float64)
    cd[:, 2] = 1.0 / sizes
    return cd


def get_instance(n, cat):
    if cat == "sparse":
        return gen_pairwise(n)
    if cat == "medium":
        return gen_medium(n, mult=20)
    if cat == "d1pct":
        m2 = n * (1 << (n - 1))
        return gen_medium(n, mult=round(0.01 * m2 / (n * (n - 1))))
    if cat.startswith("m") and cat[1:].isdigit():
        return gen_medium(n, mult=int(cat[1:]))
    if "_lam" in cat:
        base, k = cat.split("_lam")
        cd, mp = get_instance(n, base)
        lam = int(k) / 10.0
        out = cd.copy()
        out[:, 2] = lam * p_inside(cd)[:, 2] + (1.0 - lam) * cd[:, 2]
        return out, mp
    raise ValueError(cat)


def fingerprint(cd):
    a = np.ascontiguousarray(cd, dtype=np.float64)
    return hashlib.sha256(a.tobytes()).hexdigest()[:16]
