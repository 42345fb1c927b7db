"""BM-ADMM on the GPU, through the C ABI, against the oracle (tolerances written per test).

float64 paths are compared at 1e-12 relative per transform and 1e-9 absolute after many
iterations (the GPU fuses multiply-adds, the oracle rounds twice); float32 paths at the float32
rounding floor. Certified brackets must agree with the oracle's within 1e-6 and overlap the
reference's own certified brackets on its paper instances (tests/golden/refs.json)."""
import json
import math
import os

import numpy as np
import pytest

import oracle as O
import paper_instances as PI
from rumb import _lib
from rumb.instances import mixture_instance, config_instance

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
P = math.sqrt(2.0)


def _coef_sets():
    Qt, Q, _ = O.eigen_data(4, P, 1.0)
    return [(1.0, 0.0, -1.0, P), (1.0, -1.0, 0.0, P), tuple(Qt.reshape(-1)), tuple(Q.reshape(-1)),
            (1.0, -1.0, 0.0, 1.0), (1.0, 1.0, 0.0, 1.0), (1.0, 0.0, 1.0, 1.0), (0.5, 0.8660254, -0.8660254, 0.5)]


@pytest.mark.parametrize("n", [2, 3, 5, 6, 7, 10, 14, 15, 18, 20])
def test_butterfly_matches_oracle(ctx, n):
    rng = np.random.default_rng(n)
    v = rng.standard_normal(n << (n - 1))
    for co in _coef_sets():
        ref = O.butterfly(n, v, *co)
        got = ctx.butterfly(n, v, *co)
        scale = max(1.0, float(np.max(np.abs(ref))))
        assert np.max(np.abs(got - ref)) <= 1e-12 * scale * n, co
        v32 = v.astype(np.float32)
        ref32 = O.butterfly(n, v32, *co).astype(np.float64)
        got32 = ctx.butterfly(n, v32, *co).astype(np.float64)
        assert np.max(np.abs(got32 - ref32)) <= 2e-6 * scale * n, co


def _prox_case(n, rng, kind):
    m2 = n << (n - 1)
    v = rng.standard_normal(m2) * 0.5 + 0.2
    xhat = np.zeros(m2)
    w = np.zeros(m2)
    if kind != "none":
        menus = np.arange(1, 1 << n)
        for S in menus:
            if bin(int(S)).count("1") < 2 or rng.random() > 0.4:
                continue
            members = [i for i in range(n) if (S >> i) & 1]
            obs = members if kind == "full" else [i for i in members if rng.random() < 0.5]
            for i in obs:
                pos = O.slab_index(n, np.array([S]), np.array([i]))[0]
                w[pos] = 1.0
                xhat[pos] = rng.random()
    return v, xhat, w


@pytest.mark.parametrize("n", [2, 3, 5, 8, 12, 13])
@pytest.mark.parametrize("kind", ["none", "full", "mixed"])
def test_prox_matches_oracle(ctx, n, kind):
    rng = np.random.default_rng(100 * n + len(kind))
    v, xhat, w = _prox_case(n, rng, kind)
    beta2 = 2.7
    ref = O.prox(n, v, xhat, w, beta2)
    got = ctx.prox(n, v, xhat, w, beta2)
    assert np.max(np.abs(got - ref)) <= 1e-12
    ref32 = O.prox(n, v.astype(np.float32), xhat.astype(np.float32), w.astype(np.float32), np.float32(beta2))
    got32 = ctx.prox(n, v.astype(np.float32), xhat.astype(np.float32), w.astype(np.float32), beta2)
    assert np.max(np.abs(got32.astype(np.float64) - ref32)) <= 1e-5


@pytest.mark.parametrize("n", [4, 6, 10, 14])
def test_push_and_lower_bound_match_oracle(ctx, n):
    menu, alt, p = mixture_instance(n, 0.5 if n > 6 else 1.0, K=5, N=100, seed=n)
    obs = O.slab_index(n, menu, alt)
    rng = np.random.default_rng(n)
    x = rng.random(n << (n - 1)) * 0.3
    ub_ref, xub = O.push_ub64(n, x, obs, p)
    ub, fit = ctx.push_ub64(n, x, menu, alt, p)
    assert abs(ub - ub_ref) <= 1e-11 * max(1.0, ub_ref)
    np.testing.assert_allclose(fit, xub[obs], rtol=0, atol=1e-12)
    y = x[obs]
    lb_ref = O.fw_lb64(n, obs, y, p)
    lb = ctx.fw_lb64(n, menu, alt, y, p)
    assert abs(lb - lb_ref) <= 1e-10 * max(1.0, lb_ref)
    # from a float32 iterate: the push reads float32 and computes in float64
    ub32, _ = ctx.push_ub64(n, x.astype(np.float32), menu, alt, p)
    ub32_ref, _ = O.push_ub64(n, x.astype(np.float32).astype(np.float64), obs, p)
    assert abs(ub32 - ub32_ref) <= 1e-11 * max(1.0, ub32_ref)


def _instance(case):
    if case == "n10_all_k20":
        return config_instance(case)
    n = int(case[1:3])                        # "n14_mix", "n16_mix": split passes P1..P4 (n >= 14)
    from rumb.instances import mixture_instance
    m, a, p = mixture_instance(n, 0.05 if n <= 14 else 0.02, K=20, N=300, seed=n)
    return n, m, a, p


@pytest.mark.parametrize("case", ["n10_all_k20", "n14_mix", "n16_mix"])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_iterates_track_oracle(ctx, case, dtype):
    n, menu, alt, p = _instance(case)
    beta = O.beta_default(p.size)
    dt = np.float64 if dtype == "float64" else np.float32
    bm = O.BMOracle(n, menu, alt, p, dtype=dt)
    prob = ctx.bm_problem(n, menu, alt, p)
    par = ctx.bm_params(beta, dtype=dtype)
    st = ctx.bm_iterate(prob, par, None, 0, cold_start=True)
    np.testing.assert_allclose(st["x2"], bm.x2, atol=1e-12 if dt == np.float64 else 1e-6)
    total = 0
    # float32: the GPU contracts and orders the 4 (n - 1) butterfly stages of an iteration
    # differently from the oracle; at n >= 14 (the split passes) their rounding reaches ~5e-5 of the
    # largest value after one iteration. float64 pins the arithmetic itself (1e-11 .. 1e-9).
    if dt == np.float64:
        tol = {1: 1e-11, 10: 1e-10, 100: 1e-9}
    elif n < 14:
        tol = {1: 1e-5, 10: 1e-4, 100: 5e-4}
    else:
        tol = {1: 2e-4, 10: 1e-3, 100: 4e-3}
    for k in (1, 9, 90):
        st = ctx.bm_iterate(prob, par, st, k)
        bm.iterate(k)
        total += k
        for name in ("x2", "s", "y", "z"):
            d = np.max(np.abs(st[name].astype(np.float64) - getattr(bm, name).astype(np.float64)))
            assert d <= tol[total] * max(1.0, float(np.max(np.abs(getattr(bm, name))))), (name, total, d)


@pytest.mark.parametrize("form", [0, 1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("case", ["n10_all_k20", "n16_mix"])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_prox_forms_track_oracle(ctx, monkeypatch, case, form, dtype):
    """Every form of the iteration's prox kernel (RUMB_PROX_FORM: 0 the shared-memory tile, 1..3
    two, four or eight lanes per menu reading the slab into registers, 4 the tile with one member walk
    and the projection element by element, 5 the same with two staged arrays, 6 that with two threads per menu) keeps the iterates on
    the oracle's: float64 to 1e-10 after 10 iterations, float32 at its rounding floor."""
    monkeypatch.setenv("RUMB_PROX_FORM", str(form))
    n, menu, alt, p = _instance(case)
    beta = O.beta_default(p.size)
    dt = np.float64 if dtype == "float64" else np.float32
    bm = O.BMOracle(n, menu, alt, p, dtype=dt)
    prob = ctx.bm_problem(n, menu, alt, p)
    par = ctx.bm_params(beta, dtype=dtype)
    st = ctx.bm_iterate(prob, par, None, 10, cold_start=True)
    bm.iterate(10)
    tol = 1e-10 if dt == np.float64 else (1e-4 if n < 14 else 1e-3)
    for name in ("x2", "s", "y", "z"):
        ref = getattr(bm, name).astype(np.float64)
        d = np.max(np.abs(st[name].astype(np.float64) - ref))
        assert d <= tol * max(1.0, float(np.max(np.abs(ref)))), (name, d)


@pytest.mark.parametrize("fuse", [0, 1])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_fused_and_unfused_sequences_track_oracle(ctx, monkeypatch, fuse, dtype):
    """With two transform windows (n = 16) an iteration sequence runs three passes per iteration
    (RUMB_FUSE=1: P4 carries the next iteration's A', windows alternating) or four (RUMB_FUSE=0);
    both keep the iterates on the oracle's over sequences of odd and even length."""
    monkeypatch.setenv("RUMB_FUSE", str(fuse))
    n, menu, alt, p = _instance("n16_mix")
    beta = O.beta_default(p.size)
    dt = np.float64 if dtype == "float64" else np.float32
    bm = O.BMOracle(n, menu, alt, p, dtype=dt)
    prob = ctx.bm_problem(n, menu, alt, p)
    par = ctx.bm_params(beta, dtype=dtype)
    st = ctx.bm_iterate(prob, par, None, 7, cold_start=True)
    st = ctx.bm_iterate(prob, par, st, 4)
    bm.iterate(11)
    tol = 1e-10 if dt == np.float64 else 1e-3
    for name in ("x2", "s", "y", "z"):
        ref = getattr(bm, name).astype(np.float64)
        d = np.max(np.abs(st[name].astype(np.float64) - ref))
        assert d <= tol * max(1.0, float(np.max(np.abs(ref)))), (name, d)


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_three_window_iteration_tracks_oracle(ctx, dtype):
    """n = 21 splits the rest bits into three windows (the middle ones run as plain and dual
    passes, the eigenvectors in unit form there too): 3 iterations against the oracle."""
    from rumb.instances import mixture_instance
    n = 21
    menu, alt, p = mixture_instance(n, 0.0005, K=10, N=200, seed=21)
    beta = O.beta_default(p.size)
    dt = np.float64 if dtype == "float64" else np.float32
    O.set_threads(0)
    bm = O.BMOracle(n, menu, alt, p, dtype=dt)
    prob = ctx.bm_problem(n, menu, alt, p)
    par = ctx.bm_params(beta, dtype=dtype)
    st = ctx.bm_iterate(prob, par, None, 3, cold_start=True)
    bm.iterate(3)
    # float32: the rounding of 4 (n - 1) butterfly stages per iteration in another order, as in
    # test_iterates_track_oracle at n >= 14
    tol = 1e-11 if dt == np.float64 else 1e-3
    for name in ("x2", "s", "y", "z"):
        ref = getattr(bm, name).astype(np.float64)
        d = np.max(np.abs(st[name].astype(np.float64) - ref))
        assert d <= tol * max(1.0, float(np.max(np.abs(ref)))), (name, d)


def test_certified_solve_matches_oracle(ctx):
    n, menu, alt, p = config_instance("n10_all_k20")
    beta = O.beta_default(p.size)
    bm = O.BMOracle(n, menu, alt, p)
    ref = bm.solve(check=50, abs_tol=1e-5, rel_tol=1e-4)
    for graph in (True, False):
        res, fit, _ = ctx.bm_solve(ctx.bm_problem(n, menu, alt, p),
                                   ctx.bm_params(beta, check=50, abs_tol=1e-5, rel_tol=1e-4, use_graph=graph))
        assert res["stop_reason"] == ref["stop"]
        assert res["iters"] == ref["iters"]
        assert abs(res["ub"] - ref["ub"]) <= 1e-6 and abs(res["lb"] - ref["lb"]) <= 1e-6
        np.testing.assert_allclose(fit, ref["p_fit"], atol=1e-6)
        assert res["lb"] <= res["ub"]


@pytest.mark.parametrize("key", ["n18_sparse", "n18_m4"])
def test_brackets_overlap_reference_certificates(ctx, key):
    refs = json.load(open(os.path.join(GOLD, "refs.json")))["refs"]
    n = int(key.split("_")[0][1:])
    cd, mp = PI.get_instance(n, key.split("_", 1)[1])
    assert PI.fingerprint(cd) == refs[key]["cd_hash"]
    beta = O.beta_default(mp)
    res, _, _ = ctx.bm_solve(ctx.bm_problem(n, cd[:, 0], cd[:, 1], cd[:, 2]),
                             ctx.bm_params(beta, abs_tol=1e-5, rel_tol=None, time_limit=600))
    assert res["stop_reason"] == "gap_abs"
    assert res["lb"] <= refs[key]["opt"] + 1e-9 and res["ub"] >= refs[key]["lb"] - 1e-9
    assert res["ub"] - res["lb"] <= 1e-5


def test_float32_and_mixed_states_certify(ctx):
    n, menu, alt, p = config_instance("n10_all_k20")
    beta = O.beta_default(p.size)
    r64, _, _ = ctx.bm_solve(ctx.bm_problem(n, menu, alt, p), ctx.bm_params(beta, abs_tol=1e-5, rel_tol=None))
    for dt in ("float32", "mixed"):
        r, _, _ = ctx.bm_solve(ctx.bm_problem(n, menu, alt, p),
                               ctx.bm_params(beta, abs_tol=1e-5, rel_tol=None, dtype=dt, max_iter=200000))
        assert r["lb"] <= r["ub"]
        # both brackets hold the same distance
        assert r["lb"] <= r64["ub"] + 1e-9 and r64["lb"] <= r["ub"] + 1e-9
        if dt == "mixed":
            assert r["stop_reason"] == "gap_abs"


def test_warm_start_and_thresholds(ctx):
    n, menu, alt, p = config_instance("n10_all_k20")
    beta = O.beta_default(p.size)
    prob = ctx.bm_problem(n, menu, alt, p)
    r0, _, kept = ctx.bm_solve(prob, ctx.bm_params(beta, abs_tol=1e-5, rel_tol=None), keep=True)
    # warm restart from the kept state closes at once
    r1, _, _ = ctx.bm_solve(prob, ctx.bm_params(beta, abs_tol=1e-5, rel_tol=None), warm=kept)
    assert r1["iters"] <= 50 and r1["stop_reason"] == "gap_abs"
    # threshold stops
    r2, _, _ = ctx.bm_solve(prob, ctx.bm_params(beta, abs_tol=1e-9, rel_tol=None, ub_target=r0["ub"] + 0.5))
    assert r2["stop_reason"] == "ub_target"
    r3, _, _ = ctx.bm_solve(prob, ctx.bm_params(beta, abs_tol=1e-9, rel_tol=None, lb_target=r0["lb"] - 0.5))
    assert r3["stop_reason"] == "lb_target"
    r4, _, _ = ctx.bm_solve(prob, ctx.bm_params(beta, abs_tol=1e-12, rel_tol=None, max_iter=100))
    assert r4["stop_reason"] == "max_iter" and r4["iters"] == 100
    kept.close()


def test_invalid_input_is_an_error_not_a_fault(ctx):
    with pytest.raises(_lib.RumbError) as e:
        ctx.bm_solve(ctx.bm_problem(4, [3, 5], [2, 0], [0.5, 0.5]), ctx.bm_params(1.0))
    assert e.value.code == _lib.E_INVAL
    with pytest.raises(_lib.RumbError):
        ctx.bm_solve(ctx.bm_problem(31, [3], [0], [1.0]), ctx.bm_params(1.0))
    # the context still works afterwards
    n, menu, alt, p = config_instance("n10_all_k20")
    r, _, _ = ctx.bm_solve(ctx.bm_problem(n, menu, alt, p), ctx.bm_params(2.5, max_iter=50))
    assert r["iters"] == 50


@pytest.mark.parametrize("dtype", ["float64", "mixed"])
def test_overlapped_checks_certify_the_same_bracket(ctx, dtype):
    """Checks on a second stream beside the next interval: the same checks of the same states, so
    the same bracket, found one interval later (the stop takes effect after the running interval)."""
    n, menu, alt, p = _instance("n14_mix")
    beta = O.beta_default(p.size)
    prob = ctx.bm_problem(n, menu, alt, p)
    base, fit0, _ = ctx.bm_solve(prob, ctx.bm_params(beta, abs_tol=1e-6, rel_tol=None, dtype=dtype))
    ov, fit1, _ = ctx.bm_solve(prob, ctx.bm_params(beta, abs_tol=1e-6, rel_tol=None, dtype=dtype,
                                                   overlap_check=True))
    assert ov["stop_reason"] == base["stop_reason"] == "gap_abs"
    assert ov["ub"] - ov["lb"] <= 1e-6
    assert ov["lb"] <= base["ub"] + 1e-12 and base["lb"] <= ov["ub"] + 1e-12
    if dtype == "float64":
        # mixed hands over to float64 one interval later, so only float64 repeats the trajectory
        assert ov["n_push"] == base["n_push"]
        assert ov["iters"] == base["iters"] + 50
        assert ov["ub"] == base["ub"] and ov["lb"] == base["lb"]
        np.testing.assert_array_equal(fit1, fit0)
