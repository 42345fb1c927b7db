"""The reference's public interface on the GPU: RUM.calculate_distance and Session.solve for
method="bm_admm" and "flow_cg" (tests/test_cpu.py of the reference: brackets, singleton
constants, exit flags, errors)."""
import math

import numpy as np
import pytest

import oracle as O
from rumb import RUM
from rumb.instances import config_instance, mixture_instance

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def n10():
    n, m, a, p = config_instance("n10_all_k20")
    return n, m, a, p


def test_bm_admm_and_flow_cg_brackets_agree(n10):
    n, m, a, p = n10
    rum = RUM(m, a, p)
    r1 = rum.calculate_distance(method="bm_admm", abs_tol=1e-5, rel_tol=0)
    r2 = rum.calculate_distance(method="flow_cg", method_args={"dtype": "uint24", "pricing": "stream"},
                                abs_tol=1e-5, rel_tol=0)
    r3 = rum.calculate_distance(method="flow_cg", method_args={"dtype": "float32", "pricing": "mask"},
                                abs_tol=1e-5, rel_tol=0)
    for r in (r1, r2, r3):
        assert r.exit_flag in (1, 3), r
        assert r.lb <= r.ub and r.ub - r.lb <= 1e-5
        assert r.p_fit is not None and r.p_fit.shape == p.shape
        assert abs(np.linalg.norm(r.p_fit - p) - r.ub) < 1e-9
    # all three brackets contain the same distance
    lo = max(r.lb for r in (r1, r2, r3))
    hi = min(r.ub for r in (r1, r2, r3))
    assert lo <= hi + 1e-12
    # and match the oracle's float64 BM-ADMM bracket within 1e-6
    bm = O.BMOracle(n, m, a, p)
    ref = bm.solve(check=50, abs_tol=1e-5, rel_tol=None)
    assert abs(r1.ub - ref["ub"]) <= 1e-6 and abs(r1.lb - ref["lb"]) <= 1e-6
    assert r1.iterations == ref["iters"]


def test_auto_method_and_result_record(n10):
    n, m, a, p = n10
    r = RUM(m, a, p).calculate_distance()
    assert r.method == "flow_cg" and "n <= 10" in r.auto_reason
    d = r.to_dict()
    assert d["method"] == "flow_cg" and "p_fit" not in d and isinstance(d["trace"], list)
    assert "exit_flag" in repr(r)


def test_singleton_rows_are_a_constant():
    n = 6
    m, a, p = mixture_instance(n, 1.0, K=4, N=50, seed=2)
    m2 = np.concatenate([m, [1, 4]])
    a2 = np.concatenate([a, [0, 2]])
    p2 = np.concatenate([p, [0.7, 1.0]])
    base = RUM(m, a, p).calculate_distance(method="bm_admm", abs_tol=1e-7, rel_tol=0)
    withs = RUM(m2, a2, p2).calculate_distance(method="bm_admm", abs_tol=1e-7, rel_tol=0)
    assert abs(withs.ub ** 2 - (base.ub ** 2 + 0.09)) < 1e-6
    assert withs.p_fit[-2] == 1.0 and withs.p_fit[-1] == 1.0


def test_exit_flags(n10):
    n, m, a, p = n10
    rum = RUM(m, a, p)
    r = rum.calculate_distance(method="bm_admm", method_args={"max_iter": 100}, abs_tol=1e-9, rel_tol=0)
    assert r.exit_flag == -1 and r.iterations == 100
    r = rum.calculate_distance(method="bm_admm", abs_tol=1e-12, rel_tol=0, max_time=0.05)
    assert r.exit_flag == 0
    r = rum.calculate_distance(method="flow_cg", method_args={"max_iters": 3}, abs_tol=1e-9, rel_tol=0)
    assert r.exit_flag == -1


def test_session_thresholds_and_warm_start(n10):
    n, m, a, p = n10
    rum = RUM(m, a, p)
    for method in ("bm_admm", "flow_cg"):
        with rum.session(method=method) as s:
            r0 = s.solve(p, abs_tol=5e-4, rel_tol=0, keep=True)
            assert r0.exit_flag in (1, 3)
            d = r0.ub
            rng = np.random.default_rng(0)
            pb = np.clip(p + rng.normal(0, 0.01, p.size), 0, 1)
            below = s.solve(pb, abs_tol=5e-4, rel_tol=0, below=d + 1.0, warm=True)
            assert below.exit_flag == 5 and below.ub < d + 1.0
            above = s.solve(pb, abs_tol=5e-4, rel_tol=0, above=max(d - 1.0, 1e-3), warm=True)
            assert above.exit_flag == 5 and above.lb >= max(d - 1.0, 1e-3)


def test_float32_and_mixed_dtypes(n10):
    n, m, a, p = n10
    rum = RUM(m, a, p)
    r64 = rum.calculate_distance(method="bm_admm", abs_tol=1e-5, rel_tol=0)
    rmx = rum.calculate_distance(method="bm_admm", method_args={"dtype": "mixed"}, abs_tol=1e-5, rel_tol=0)
    assert rmx.exit_flag in (1, 3)
    assert rmx.lb <= r64.ub + 1e-12 and r64.lb <= rmx.ub + 1e-12
    assert rmx.method_args["dtype"] == "mixed"
