"""The library against the reference's own kernels, JIT-compiled by NVRTC from the reference's
source strings and replayed (baseline/build_ref.py, baseline/ref_replay.py): Flow-CG pricing must
agree bit for bit (values, rankings, per-layer steps). Skipped where baseline/_ref was not built
(it needs the reference's source tree at build time)."""
import os

import numpy as np
import pytest

import oracle as O
import paper_instances as PI
import ref_replay
from rumb import _lib
from rumb.instances import config_instance

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_replay.available(), reason="baseline/_ref not built")]


def _cases():
    yield "pair8", PI.gen_pairwise(8)[0], 8
    yield "med12", PI.gen_medium(12, mult=3)[0], 12
    yield "pair16", PI.gen_pairwise(16)[0], 16
    n, m, a, p = config_instance("n18_d05pct_k50")
    yield "n18_d05pct", np.column_stack([m, a, p]).astype(np.float64), n


CASES = list(_cases())


@pytest.mark.parametrize("name,cd,n", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("mode", ["f32", "f32_stream", "u16", "u24"])
def test_stream_pricer_matches_reference_kernels(ctx, name, cd, n, mode):
    """f32: the lattice by mask where it fits (the tile sweep); f32_stream: two rank-indexed layers."""
    menus, alts, p32, offsets, _ = O.cg_layout(n, cd[:, 0], cd[:, 1], cd[:, 2])
    stream = mode == "f32_stream"
    mode = "f32" if stream else mode
    pr = _lib.Pricer(ctx, n, menus, offsets, mode=mode, stream=stream)
    rng = np.random.RandomState(11)
    for trial in range(2):
        scores = (rng.randn(menus.size) * (1.0 if trial == 0 else 0.02)).astype(np.float32)
        v_ref, r_ref, m_ref, steps_ref = ref_replay.price_stream(menus, alts, scores, offsets, n, mode=mode)
        v, r, m, steps = pr.price(scores, want_steps=True)
        assert v == v_ref, (v, v_ref)
        np.testing.assert_array_equal(r, r_ref)
        np.testing.assert_array_equal(steps, steps_ref)
        assert abs(m - m_ref) <= 1e-6 * max(1.0, m_ref)      # the reference sums the steps in float32
    pr.close()


@pytest.mark.parametrize("name,cd,n", CASES[:3], ids=[c[0] for c in CASES[:3]])
def test_mask_pricer_matches_reference_kernel(ctx, name, cd, n):
    menus, alts, p32, offsets, _ = O.cg_layout(n, cd[:, 0], cd[:, 1], cd[:, 2])
    pr = _lib.Pricer(ctx, n, menus, offsets, mode="mask")
    scores = np.random.RandomState(5).randn(menus.size).astype(np.float32)
    v_ref, r_ref = ref_replay.price_mask(menus, scores, offsets, n)
    v, r, _ = pr.price(scores)
    assert v == v_ref and np.array_equal(r, r_ref)


# ------------------------------------------------------------------ BM-ADMM against the reference
def _bm_instance(case):
    if case == "n14_mix":
        from rumb.instances import mixture_instance
        m, a, p = mixture_instance(14, 0.05, K=20, N=300, seed=14)
        return 14, m, a, p
    return config_instance(case)[:4]


BM_CASES = ["n10_all_k20", "n14_mix", "n18_d1pct_k50"]
# float64 iterates after 1, 10 and 100 iterations, relative to the largest entry: the library
# contracts multiply-adds and runs some transforms high bits first, the reference's kernels follow
# their own stage plan, so the two round differently by a few ulps per iteration
ITER_TOL = {1: 1e-11, 10: 1e-10, 100: 1e-9}


def _max_rel(a, b):
    return float(np.max(np.abs(a - b))) / max(1.0, float(np.max(np.abs(b))))


@pytest.mark.parametrize("case", BM_CASES)
def test_bm_iterates_match_reference_kernels(ctx, case):
    """rumb_bm_iterate and the reference's own float64 iteration (solve_kadmm_v2's one_iter with
    its kernels and calibrated butterfly plan, solver/bm_admm/solver.py:240-254) from the same cold
    start (solver/bm_admm/solver.py:263-267): x2, s, y, z after 1, 10 and 100 iterations."""
    n, menu, alt, p = _bm_instance(case)
    beta = O.beta_default(p.size)
    ref = ref_replay.BMReplay(n, menu, alt, p, beta)
    prob = ctx.bm_problem(n, menu, alt, p)
    par = ctx.bm_params(beta, dtype="float64")
    st = ctx.bm_iterate(prob, par, None, 0, cold_start=True)
    r = ref.state()
    assert _max_rel(st["x2"], r["x2"]) <= 1e-12
    total = 0
    for k in (1, 9, 90):
        st = ctx.bm_iterate(prob, par, st, k)
        ref.iterate(k)
        total += k
        r = ref.state()
        for name in ("x2", "s", "y", "z"):
            d = _max_rel(st[name], r[name])
            assert d <= ITER_TOL[total], (case, name, total, d)


@pytest.mark.parametrize("case", BM_CASES)
def test_oracle_iterates_match_reference_kernels(case):
    """The oracle's float64 iteration (oracle/rum_oracle.c, the CPU restatement every other
    BM-ADMM test checks the library against) pinned to the reference's own kernels the same way."""
    n, menu, alt, p = _bm_instance(case)
    beta = O.beta_default(p.size)
    ref = ref_replay.BMReplay(n, menu, alt, p, beta)
    O.set_threads(0)
    bm = O.BMOracle(n, menu, alt, p, beta=beta)
    assert _max_rel(bm.x2, ref.state()["x2"]) <= 1e-12
    total = 0
    for k in (1, 9, 90):
        bm.iterate(k)
        ref.iterate(k)
        total += k
        r = ref.state()
        for name in ("x2", "s", "y", "z"):
            d = _max_rel(getattr(bm, name), r[name])
            assert d <= ITER_TOL[total], (case, name, total, d)


_REF_SOLVES = {}


def _reference_bracket(case):
    """The reference's certified float64 bracket of a workload at abs 1e-5, check 50 (its kernels,
    replayed with the runner's hooks); one run per session."""
    if case not in _REF_SOLVES:
        n, menu, alt, p = _bm_instance(case)
        ref = ref_replay.BMReplay(n, menu, alt, p, O.beta_default(p.size))
        _REF_SOLVES[case] = ref.solve(abs_tol=1e-5, check=50, lb_every=1)
    return _REF_SOLVES[case]


@pytest.mark.parametrize("dtype", ["float64", "mixed"])
@pytest.mark.parametrize("case", ["n10_all_k20", "n18_d1pct_k50"])
def test_certified_bracket_matches_reference_float64(ctx, case, dtype):
    """The certified bracket at abs 1e-5 (n18_d1pct_k50 is the benchmark workload: n = 18, 1 %
    menus, K = 50, N = 500) against the reference's float64 bm_admm run with its own kernels: both
    certified and overlapping, each bound within 1e-6 of the reference's in float64 (the library
    follows the reference's trajectory and stops at the same check) and, for mixed (float32 until
    the float32 bracket stalls, then float64), on the benchmark workload; elsewhere mixed reaches
    its own point of the certified bracket, within the 1e-5 tolerance."""
    n, menu, alt, p = _bm_instance(case)
    ref = _reference_bracket(case)
    assert ref["stop_reason"] == "gap_abs" and ref["ub"] - ref["lb"] <= 1e-5
    res, _, _ = ctx.bm_solve(ctx.bm_problem(n, menu, alt, p),
                             ctx.bm_params(O.beta_default(p.size), check=50, abs_tol=1e-5, rel_tol=None,
                                           dtype=dtype, time_limit=600))
    assert res["stop_reason"] == "gap_abs", res
    assert res["lb"] <= res["ub"] and res["ub"] - res["lb"] <= 1e-5
    # two certified brackets of one distance overlap
    assert res["lb"] <= ref["ub"] + 1e-12 and ref["lb"] <= res["ub"] + 1e-12
    # float64 follows the reference's trajectory, and on the benchmark workload so does mixed's
    # float64 finish, to 1e-6; at n = 10 the float32 start leads mixed to another point of the
    # same 1e-5 bracket (measured 8e-6 from the reference's upper bound)
    tol = 1e-6 if (dtype == "float64" or case == "n18_d1pct_k50") else 1e-5
    assert abs(res["ub"] - ref["ub"]) <= tol, (res["ub"], ref["ub"])
    assert abs(res["lb"] - ref["lb"]) <= tol, (res["lb"], ref["lb"])
    if dtype == "float64":
        assert res["iters"] == ref["iters"], (res["iters"], ref["iters"])


# ------------------------------------------------------------------ Flow-CG n18_d05pct_k50, every column
# uint16's block quantization margin enters the Frank-Wolfe bound, and at this density it keeps the
# bracket above abs 1e-5 (the run reaches 4,000 columns without certifying): uint16 runs a fixed
# number of columns instead
CG3_MAX = {"u24": 4000, "u16": 1000}


def _config3_run(ctx, mode, check_reference):
    """The library's CG loop on n18_d05pct_k50 (n = 18, 0.5 % menus, K = 50, N = 500) to abs 1e-5
    in `mode` (uint16: CG3_MAX columns); at every iteration the residual it priced is priced again
    by the reference's own stream kernels (when check_reference) and by the library's pricer
    directly."""
    from rumb import flow_cg
    n, m, a, p = config_instance("n18_d05pct_k50")
    prob = flow_cg.CGProblem(ctx, n, m, a, mode)
    menus, alts, _, offsets, _ = O.cg_layout(n, m, a, p)
    bad = []

    def on_price(it, scores, vmax, rank_pos, margin):
        v2, r2, m2 = prob.pricer.price(scores)           # the residual read back is the one priced
        if not (v2 == vmax and np.array_equal(r2, rank_pos)):
            bad.append(("library", it))
        if check_reference:
            v_ref, r_ref, m_ref, _ = ref_replay.price_stream(menus, alts, scores, offsets, n, mode=mode)
            if not (v_ref == vmax and np.array_equal(r_ref, rank_pos)):
                bad.append(("reference", it, v_ref, vmax))

    res = flow_cg.solve_cg(prob, p, max_iters=CG3_MAX[mode], gap_abs_tol=1e-5, record_columns=True,
                           on_price=on_price)
    return res, bad


@pytest.mark.parametrize("mode", ["u24", "u16"])
def test_config3_columns_match_reference_kernels_every_iteration(ctx, mode):
    """The n18_d05pct_k50 workload's check: Flow-CG at n = 18, 0.5 % density, run to abs 1e-5 (uint24; uint16
    for 1,000 columns, see CG3_MAX), and the column
    (the ranking) the library prices at every CG iteration is the one the reference's own
    bf_stream_u24 / bf_stream_u16 kernels and backtrace pick on the same residual
    (solver/flow_cg/pricing_stream.py:61-181,302-412, solver/flow_cg/solver.py:131-243)."""
    res, bad = _config3_run(ctx, mode, check_reference=True)
    assert res["stop_reason"] == ("gap_abs" if mode == "u24" else "max_iters"), res["stop_reason"]
    assert not bad, bad[:5]
    gold = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cg_config3.npz")
    if os.path.exists(gold):
        g = np.load(gold)
        np.testing.assert_array_equal(np.array(res["picked"]), g["picked_" + mode])


# ------------------------------------------------------------------ large lattices (n = 28)
@pytest.mark.parametrize("mode", ["f32", "f32_stream", "u16", "u24"])
def test_stream_pricer_at_n28_matches_reference_kernels(ctx, mode):
    """The stream pricer at n = 28 (pairwise menus, 756 rows; 2^28 subsets, rows scanned per
    subset as the lists are not built above n = 26) against the reference's own stream kernels:
    the same Vmax, ranking, per-layer steps and margin (solver/flow_cg/pricing_stream.py:61-181,
    302-412; the reference's large-n pricing path, solver/flow_cg/MEMORY.md:59-74)."""
    n = 28
    cd, _ = PI.gen_pairwise(n)
    menus, alts, p32, offsets, _ = O.cg_layout(n, cd[:, 0], cd[:, 1], cd[:, 2])
    stream = mode == "f32_stream"
    mode = "f32" if stream else mode
    pr = _lib.Pricer(ctx, n, menus, offsets, mode=mode, stream=stream)
    scores = (np.random.RandomState(28).randn(menus.size)).astype(np.float32)
    v_ref, r_ref, m_ref, steps_ref = ref_replay.price_stream(menus, alts, scores, offsets, n, mode=mode)
    v, r, m, steps = pr.price(scores, want_steps=True)
    assert v == v_ref, (v, v_ref)
    np.testing.assert_array_equal(r, r_ref)
    np.testing.assert_array_equal(steps, steps_ref)
    assert abs(m - m_ref) <= 1e-6 * max(1.0, m_ref)
    pr.close()


def test_max64_at_n28_matches_reference_kernels(ctx):
    """The float64 max sweep at n = 28 (pairwise menus, rows scanned: the group form) against the
    reference's own bf_stream_max64 kernel (solver/flow_cg/pricing_stream.py:190-249), bit for bit."""
    if "max64" not in ref_replay._mods():
        pytest.skip("the reference's max64 kernel is not built")
    n = 28
    cd, _ = PI.gen_pairwise(n)
    menus, alts, p32, offsets, _ = O.cg_layout(n, cd[:, 0], cd[:, 1], cd[:, 2])
    s = np.random.RandomState(281).randn(menus.size)
    pr = _lib.Pricer(ctx, n, menus, offsets, mode="u16")
    v = pr.max64(s)
    pr.close()
    assert v == ref_replay.sweep_max64(menus, s, offsets, n)
