"""Batched draws (rumb_bm_solve_batch) against one-at-a-time solves of the same draws: identical
float64 trajectories, float32 brackets that still contain the distance, thresholds, and slot
refilling when there are more draws than slots."""
import numpy as np
import pytest

import oracle as O
from rumb.instances import config_instance

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(ctx):
    n, m, a, p = config_instance("n10_all_k20")
    beta = O.beta_default(p.size)
    prob = ctx.bm_problem(n, m, a, p)
    r0, fit, kept = ctx.bm_solve(prob, ctx.bm_params(beta, abs_tol=5e-4, rel_tol=None), keep=True)
    rng = np.random.default_rng(0)
    P = np.clip(p[None, :] + rng.normal(0, 0.02, (8, p.size)), 0.0, 1.0)
    return n, m, a, p, beta, prob, kept, P, r0


def test_batch_float64_equals_one_at_a_time(ctx, setup):
    n, m, a, p, beta, prob, kept, P, r0 = setup
    par = ctx.bm_params(beta, abs_tol=5e-4, rel_tol=None, dtype="float64")
    res, info = ctx.bm_solve_batch(prob, par, P, warm=kept, slots=3)
    assert info["slots"] == 3
    for b in range(P.shape[0]):
        one, _, _ = ctx.bm_solve(ctx.bm_problem(n, m, a, P[b]), par, warm=kept)
        assert res[b]["stop_reason"] == one["stop_reason"] == "gap_abs"
        assert res[b]["iters"] == one["iters"]
        assert abs(res[b]["ub"] - one["ub"]) <= 1e-12 and abs(res[b]["lb"] - one["lb"]) <= 1e-12


def test_batch_float32_brackets_hold(ctx, setup):
    n, m, a, p, beta, prob, kept, P, r0 = setup
    par64 = ctx.bm_params(beta, abs_tol=1e-7, rel_tol=None, dtype="float64")
    ref, _ = ctx.bm_solve_batch(prob, par64, P, warm=kept)
    par = ctx.bm_params(beta, abs_tol=5e-4, rel_tol=None, dtype="float32")
    res, info = ctx.bm_solve_batch(prob, par, P, warm=kept)
    for b in range(P.shape[0]):
        assert res[b]["stop_reason"] in ("gap_abs", "stall")
        assert res[b]["lb"] <= ref[b]["ub"] + 1e-9 and ref[b]["lb"] <= res[b]["ub"] + 1e-9
        if res[b]["stop_reason"] == "gap_abs":
            assert res[b]["ub"] - res[b]["lb"] <= 5e-4


def test_batch_thresholds_and_cold_start(ctx, setup):
    n, m, a, p, beta, prob, kept, P, r0 = setup
    par = ctx.bm_params(beta, abs_tol=1e-9, rel_tol=None, dtype="float64", max_iter=20000)
    d = r0["ub"]
    below = np.full(P.shape[0], np.nan)
    above = np.full(P.shape[0], np.nan)
    below[:4] = d + 2.0          # far above every draw's distance: decided below at the first check
    above[4:] = 1e-3             # far below: decided above once the lower bound passes it
    res, info = ctx.bm_solve_batch(prob, par, P, below=below, above=above)   # cold start
    for b in range(4):
        assert res[b]["stop_reason"] == "ub_target" and res[b]["ub"] <= d + 2.0
    for b in range(4, P.shape[0]):
        assert res[b]["stop_reason"] == "lb_target" and res[b]["lb"] >= 1e-3
