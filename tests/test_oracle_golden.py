"""The oracle pinned against the reference: golden vectors produced by the reference's own CPU
code (tests/golden/make_golden.py), the reference's own pricer test properties
(validation/feasibility/test_stream_pricer.py:49-84) and an exact small-n distance."""
import itertools
import json
import math
import os

import numpy as np
import pytest

import oracle as O
import paper_instances as PI

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    return np.load(os.path.join(GOLD, name))


@pytest.mark.parametrize("n", [3, 4, 5, 6, 8, 10])
def test_certificate_pieces_match_reference(n):
    g = _load("certificate.npz")
    # push (make_r_feasible in float64) vs certificate.push_flow
    rf = O.make_feasible64(n, g["push_q_%d" % n])
    np.testing.assert_allclose(rf, g["push_rf_%d" % n], rtol=1e-12, atol=1e-15)
    # best ranking = subset-sum butterfly + longest path
    gs = O.butterfly(n, g["bestrank_g_%d" % n], 1.0, 0.0, 1.0, 1.0)
    assert abs(O.longest_path64(n, gs) - g["bestrank_v_%d" % n][0]) <= 1e-12 * max(1.0, abs(g["bestrank_v_%d" % n][0]))
    # zeta at rows
    z = O.butterfly(n, g["push_q_%d" % n], 1.0, 1.0, 0.0, 1.0)[g["zeta_obs_%d" % n]]
    np.testing.assert_allclose(z, g["zeta_rows_%d" % n], rtol=1e-12, atol=1e-13)
    # Frank-Wolfe lower bound
    lb = O.fw_lb64(n, g["zeta_obs_%d" % n], g["fwlb_y_%d" % n], g["fwlb_p_%d" % n])
    assert abs(lb - g["fwlb_v_%d" % n][0]) <= 1e-11 * max(1.0, lb)
    # slab positions
    idx = O.slab_index(n, g["slab_menu_%d" % n], g["slab_alt_%d" % n])
    np.testing.assert_array_equal(idx, g["slab_idx_%d" % n])


@pytest.mark.parametrize("n", [3, 4, 5, 6, 8, 10])
def test_oracle_two_layer_bound_matches_reference(n):
    """fw_lb_stream64 (the float64 max sweep, two layers live) gives the reference's slab-based
    Frank-Wolfe bound at the golden points."""
    g = _load("certificate.npz")
    idx = np.asarray(g["zeta_obs_%d" % n], dtype=np.int64)
    x = idx >> (n - 1)
    rest = idx & ((1 << (n - 1)) - 1)
    menu = ((rest >> x) << (x + 1)) | (rest & ((1 << x) - 1)) | (1 << x)
    lb = O.fw_lb_stream64(n, menu, x, g["fwlb_y_%d" % n], g["fwlb_p_%d" % n])
    assert abs(lb - g["fwlb_v_%d" % n][0]) <= 1e-11 * max(1.0, lb)


@pytest.mark.parametrize("n", [4, 6, 7])
def test_oracle_max_sweep_is_the_best_ranking(n):
    """V[full] of the float64 max sweep is the largest summed score over all n! rankings."""
    rng = np.random.default_rng(n)
    menus_all = [m for m in range(1, 1 << n) if bin(m).count("1") >= 2]
    rows = [(m, x) for m in menus_all if rng.random() < 0.6 for x in range(n) if (m >> x) & 1]
    menu = np.array([r[0] for r in rows], dtype=np.int64)
    alt = np.array([r[1] for r in rows], dtype=np.int64)
    menus, alts, _, offsets, perm = O.cg_layout(n, menu, alt, np.zeros(len(rows)))
    scores = rng.standard_normal(len(rows))
    best = -np.inf
    for order in itertools.permutations(range(n)):
        rank = np.empty(n, dtype=np.int32)
        rank[list(order)] = np.arange(n)
        col = O.ranking_column(n, menus, alts, rank)
        best = max(best, float(scores[col > 0].sum()))
    v = O.sweep_max64(n, menus, scores, offsets)
    assert abs(v - best) <= 1e-12 * max(1.0, abs(best))


def test_master_qp_matches_reference():
    g = _load("qp.npz")
    for t in range(4):
        lam, A = O.qp_native(g["Q_%d" % t], g["h_%d" % t])
        np.testing.assert_allclose(lam, g["lam_%d" % t], rtol=0, atol=1e-12)
        np.testing.assert_allclose(O.project_simplex(g["ps_y_%d" % t]), g["ps_x_%d" % t], atol=1e-15)


def test_lattice_layers_and_colex():
    g = _load("lattice.npz")
    for n in (5, 9, 12):
        order, bounds = O.layers(n)
        for k in range(1, n + 1):
            np.testing.assert_array_equal(order[bounds[k]:bounds[k + 1]], g["layer_%d_%d" % (n, k)])
        colex = np.array([O.lib().ora_colex_rank(int(m)) for m in range(1 << n)])
        np.testing.assert_array_equal(colex, g["colex_%d" % n])


def test_ranking_columns_match_reference():
    g = _load("columns.npz")
    for t in range(5):
        col = O.ranking_column(18, g["menus"], g["alts"], g["rank_%d" % t])
        np.testing.assert_array_equal(col, g["col_%d" % t])


def test_paper_instances_regenerate_bit_for_bit():
    refs = json.load(open(os.path.join(GOLD, "refs.json")))["refs"]
    for key in ("n18_sparse", "n18_m2", "n18_m4", "n18_m8", "n18_sparse_lam5", "n19_sparse", "n20_sparse"):
        n = int(key.split("_")[0][1:])
        cd, mp = PI.get_instance(n, key.split("_", 1)[1])
        assert PI.fingerprint(cd) == refs[key]["cd_hash"], key
        assert mp == refs[key]["mp"]


def test_beta_rule_matches_reference():
    beta = json.load(open(os.path.join(GOLD, "refs.json")))["beta_default"]
    for mp, b in beta.items():
        assert O.beta_default(int(mp)) == b


def _exact_distance(n, menu, alt, p):
    """min ||V lam - p|| over the mixtures of all n! rankings (independent of BM-ADMM)."""
    cols = []
    for perm in itertools.permutations(range(n)):
        rank = np.empty(n, dtype=np.int32)
        rank[list(perm)] = np.arange(n)
        cols.append(O.ranking_column(n, menu.astype(np.uint64), alt.astype(np.int32), rank).astype(np.float64))
    V = np.stack(cols, axis=1)
    Q = V.T @ V
    h = V.T @ p
    lam, _ = O.qp_native(Q, h, max_outer=2000)
    return float(np.linalg.norm(V @ lam - p))


@pytest.mark.parametrize("seed", [0, 1])
def test_oracle_bm_admm_brackets_exact_distance(seed):
    from rumb.instances import mixture_instance
    n = 5
    menu, alt, p = mixture_instance(n, 1.0, K=3, N=30, seed=seed)
    d = _exact_distance(n, menu, alt, p)
    bm = O.BMOracle(n, menu, alt, p)
    r = bm.solve(check=25, abs_tol=1e-7, rel_tol=None, max_iter=200000)
    assert r["stop"] == "gap_abs"
    assert r["lb"] - 1e-9 <= d <= r["ub"] + 1e-9


def test_oracle_float32_iteration_tracks_float64():
    from rumb.instances import mixture_instance
    n = 8
    menu, alt, p = mixture_instance(n, 1.0, K=5, N=100, seed=3)
    a = O.BMOracle(n, menu, alt, p, dtype=np.float64)
    b = O.BMOracle(n, menu, alt, p, dtype=np.float32)
    a.iterate(30)
    b.iterate(30)
    assert np.max(np.abs(a.x2 - b.x2)) < 1e-3


# ---------------------------------------------------------------- pricer: the reference's own checks
def _brute(n, menus, alts, scores):
    best = -1e30
    for perm in itertools.permutations(range(n)):
        rank = np.empty(n, dtype=np.int32)
        rank[list(perm)] = np.arange(n)
        col = O.ranking_column(n, menus, alts, rank)
        best = max(best, float(np.sum(scores.astype(np.float64)[col > 0])))
    return best


def _col_value(n, menus, alts, scores, rank):
    col = O.ranking_column(n, menus, alts, rank)
    return float(np.sum(scores.astype(np.float64)[col > 0]))


@pytest.mark.parametrize("n,gen", [(6, "pair"), (8, "pair"), (12, "med"), (14, "pair")])
def test_oracle_stream_pricer_properties(n, gen):
    cd, mp = PI.gen_pairwise(n) if gen == "pair" else PI.gen_medium(n, mult=3)
    menus, alts, _p32, offsets, _ = O.cg_layout(n, cd[:, 0], cd[:, 1], cd[:, 2])
    rng = np.random.RandomState(1)
    for trial in range(3):
        scores = (rng.randn(mp) * (2.0 if trial == 0 else 0.3)).astype(np.float32)
        vm, rm = O.price_mask(n, menus, scores, offsets)
        vf, rf, mf, _ = O.price_stream(n, menus, scores, offsets, "f32", k_pred=max(1, n - 4))
        assert vf == vm and np.array_equal(rf, rm), "f32 stream must equal the mask sweep bit for bit"
        for mode in ("u16", "u24"):
            vu, ru, mu, _ = O.price_stream(n, menus, scores, offsets, mode, k_pred=max(1, n - 4))
            assert abs(vu - vm) <= mu + 1e-5
            assert abs(_col_value(n, menus, alts, scores, ru) - vm) <= mu + 1e-4
        if n <= 8 and trial == 0:
            assert abs(_brute(n, menus, alts, scores) - vm) < 1e-4


def test_oracle_cg_loop_closes_small_instance():
    cd, mp = PI.gen_medium(8, mult=3)
    r = O.cg_solve(8, cd[:, 0], cd[:, 1], cd[:, 2], mode="u24", max_iters=300, gap_abs_tol=1e-6)
    assert r["stop"] == "gap_abs"
    assert r["lb"] <= r["ub"] + 1e-12


REPLAY = os.path.join(GOLD, "pricer_replay.npz")


@pytest.mark.skipif(not os.path.exists(REPLAY), reason="reference kernel outputs not recorded")
def test_oracle_pricer_matches_recorded_reference_kernels():
    """The oracle's stream pricers (fma decode) and mask sweep against the outputs the reference's
    own kernels gave on a B200 (tests/golden/make_replay_golden.py), bit for bit; the n = 18 case is
    left to the GPU test (minutes of oracle time)."""
    import make_replay_golden as MR
    g = np.load(REPLAY)
    for name, n, m, a, p in MR.cases():
        if n > 16:
            continue
        menus, alts, p32, offsets, _ = O.cg_layout(n, m, a, p)
        for trial in range(2):
            key = "%s_t%d" % (name, trial)
            s = g[key + "_scores"]
            np.testing.assert_array_equal(s, MR.scores_for(name, menus.size, trial))
            for mode in ("f32", "u16", "u24"):
                v, r, mg, steps = O.price_stream(n, menus, s, offsets, mode=mode)
                assert np.float32(v) == g["%s_%s_vmax" % (key, mode)], (key, mode)
                np.testing.assert_array_equal(r, g["%s_%s_rank" % (key, mode)])
                np.testing.assert_array_equal(np.asarray(steps, np.float32), g["%s_%s_steps" % (key, mode)])
                assert abs(mg - float(g["%s_%s_margin" % (key, mode)])) <= 1e-6 * max(1.0, mg)
            v, r = O.price_mask(n, menus, s, offsets)
            assert np.float32(v) == g[key + "_mask_vmax"]
            np.testing.assert_array_equal(r, g[key + "_mask_rank"])
