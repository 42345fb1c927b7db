"""Generates the golden fixtures in this folder by running the reference's own CPU code.

    PYTHONPATH=<reference root>:<reference root>/data python tests/golden/make_golden.py <reference root>

It imports mingxiz/rum-testing-gpu from the path given (read-only, never copied) and writes small
.npz / .json files next to this script. The tests compare the oracle (oracle/) and the library
against these files; nothing at test time reads the reference itself.

Fixtures:
  certificate.npz   push_flow, zeta_rows, fw_lb_rows, _best_ranking, slab_index on seeded inputs
                    (solver/common/certificate.py:27-139)
  qp.npz            solve_qp_native / project_simplex on seeded simplex QPs (solver/common/qp_native.py)
  lattice.npz       Gosper layers and colex ranks (solver/common/layers.py:9-31,
                    solver/flow_cg/pricing_stream.py:254-264), binom_table (solver/flow_cg/cg_core.py:53-60)
  columns.npz       map_ranking_to_choice on seeded rankings (solver/flow_cg/cg_core.py:63-80)
  refs.json         certified [lb, opt] brackets and sha256 fingerprints of paper instances
                    (data/opt_refs.json, data/gen_instances.py:196-199), plus the fingerprints of the
                    instances regenerated by get_instance here
  pricer.npz        the reference's BM-ADMM defaults (beta rule) on sample mp values
                    (solver/params.py:52-54)
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root):
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/numba_cache_golden")
    sys.path.insert(0, ref_root)
    sys.path.insert(0, os.path.join(ref_root, "data"))
    # The reference's CPU helpers live in modules that also build CuPy kernels at import time;
    # CuPy is not installed here, so a do-nothing stand-in lets those modules import. Only
    # functions that never touch CuPy are called below.
    from unittest import mock
    sys.modules.setdefault("cupy", mock.MagicMock(name="cupy"))
    from solver.common import certificate as C
    from solver.common import qp_native as QN
    from solver.flow_cg import cg_core  # noqa: E402
    from solver import params
    import gen_instances as G

    rng = np.random.default_rng(20240601)
    out = {}
    for n in (3, 4, 5, 6, 8, 10):
        m2 = n << (n - 1)
        q = rng.standard_normal(m2)
        out["push_q_%d" % n] = q
        out["push_rf_%d" % n] = C.push_flow(n, q)
        g = rng.standard_normal(m2)
        out["bestrank_g_%d" % n] = g
        out["bestrank_v_%d" % n] = np.array([C._best_ranking(n, g.copy())])
        obs = np.sort(rng.choice(m2, size=min(40, m2), replace=False)).astype(np.int64)
        out["zeta_obs_%d" % n] = obs
        out["zeta_rows_%d" % n] = C.zeta_rows(n, q, obs)
        y = rng.random(obs.size)
        ph = rng.random(obs.size)
        out["fwlb_y_%d" % n] = y
        out["fwlb_p_%d" % n] = ph
        out["fwlb_v_%d" % n] = np.array(C.fw_lb_rows(n, obs, y, ph)[:3])
        # slab_index on random (menu, alt) rows
        menus = rng.integers(1, 1 << n, size=30, dtype=np.int64)
        menus = menus[np.array([bin(int(m)).count("1") >= 1 for m in menus])]
        alts = np.array([int(rng.choice([a for a in range(n) if (int(m) >> a) & 1])) for m in menus], dtype=np.int64)
        out["slab_menu_%d" % n] = menus
        out["slab_alt_%d" % n] = alts
        out["slab_idx_%d" % n] = C.slab_index(n, menus, alts)
    np.savez_compressed(os.path.join(HERE, "certificate.npz"), **out)

    out = {}
    for t, K in enumerate((3, 8, 20, 40)):
        V = (rng.random((60, K)) < 0.5).astype(np.float64)
        ph = rng.random(60)
        Q = V.T @ V
        h = V.T @ ph
        lam, A = QN.solve_qp_native(Q, h)
        out["Q_%d" % t], out["h_%d" % t], out["lam_%d" % t] = Q, h, lam
        out["A_%d" % t] = np.array(A, dtype=np.int64)
        y = rng.standard_normal(K)
        out["ps_y_%d" % t], out["ps_x_%d" % t] = y, QN.project_simplex(y)
    np.savez_compressed(os.path.join(HERE, "qp.npz"), **out)

    from solver.common import layers as LY
    out = {}
    for n in (5, 9, 12):
        for k in range(0, n + 1):
            lay = np.empty(0, dtype=np.int32)
            if k > 0:
                import math
                lay = np.empty(math.comb(n, k), dtype=np.int32)
                LY._gosper_fill(lay, n, k)
            out["layer_%d_%d" % (n, k)] = lay
        out["binom_%d" % n] = cg_core.binom_table(n)
        from solver.flow_cg.pricing_stream import colex_rank
        allm = np.arange(1 << n, dtype=np.int64)
        out["colex_%d" % n] = np.array([colex_rank(int(m)) for m in allm], dtype=np.int64)
    np.savez_compressed(os.path.join(HERE, "lattice.npz"), **out)

    out = {}
    cd, mp = G.get_instance(18, "m4")
    menus = cd[:, 0].astype(np.int64).astype(np.uint32)
    alts = cd[:, 1].astype(np.int32)
    out["menus"], out["alts"] = menus, alts
    for t in range(5):
        rank = rng.permutation(18).astype(np.int32)
        out["rank_%d" % t] = rank
        out["col_%d" % t] = cg_core.map_ranking_to_choice(menus, alts, rank, 18)
    np.savez_compressed(os.path.join(HERE, "columns.npz"), **out)

    refs = json.load(open(os.path.join(ref_root, "data", "opt_refs.json")))
    keep = {}
    for key in ("n18_sparse", "n18_m2", "n18_m4", "n18_m8", "n18_medium", "n18_d1pct", "n18_m39",
                "n18_sparse_lam5", "n19_sparse", "n20_sparse", "n20_d1pct"):
        r = refs[key]
        n = int(key.split("_")[0][1:])
        cat = key.split("_", 1)[1]
        cd, mp = G.get_instance(n, cat)
        keep[key] = dict(opt=r["opt"], lb=r["lb"], mp=r["mp"], cd_hash=r["cd_hash"], regenerated_hash=G.fingerprint(cd),
                         regenerated_mp=int(mp))
    beta = {str(m): params.bm_beta_default(m) for m in (10, 306, 5110, 23568, 81188, 104885, 2359278)}
    json.dump(dict(refs=keep, beta_default=beta), open(os.path.join(HERE, "refs.json"), "w"), indent=1, sort_keys=True)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "baseline"))
    import build_ref
    root = sys.argv[1] if len(sys.argv) > 1 else build_ref.reference_root()
    if root is None:
        raise SystemExit("the reference's source tree was not found (give it as the argument, or RUM_REFERENCE_ROOT)")
    main(root)
