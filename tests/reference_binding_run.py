"""Runs the reference's own RUM class with rumb's binding installed, and rumb's RUM, on one
instance; prints both Result records as JSON (the body of tests/test_reference_binding.py, run in
a process of its own because the reference needs a stand-in module for CuPy).

    python tests/reference_binding_run.py <reference root>

The GPU engine under rumb's runner is replaced by a host stand-in built on the oracle's certified
solve (the same loop: push every check, lower bound every lb_every checks, stop on the gap), so
the run needs no GPU; what it checks is the binding: the reference's planner and runner tables
reach rumb's planner and runner with the reference's task, and the reference builds its Result
from what rumb's runner left in the task's state.
"""
import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (os.path.join(ROOT, "rum-testing-gpu_b200"), os.path.join(ROOT, "oracle"), HERE):
    sys.path.insert(0, p)


class HostEngine:
    """Stands in for rumb's library context: bm_solve runs the oracle's certified solve."""

    def mem_info(self):
        return 64 << 30, 80 << 30

    @staticmethod
    def bm_params(beta, **kw):
        return types.SimpleNamespace(beta=beta, **kw)

    @staticmethod
    def bm_problem(n, menu, alt, p):
        return (n, np.asarray(menu), np.asarray(alt), np.asarray(p, dtype=np.float64))

    def bm_solve(self, prob, par, warm=None, keep=False, trace=None):
        import oracle as O
        n, menu, alt, p = prob
        bm = O.BMOracle(n, menu, alt, p, beta=par.beta, alpha=par.alpha, precond_p=par.precond_p)
        r = bm.solve(check=par.check, lb_every=par.lb_every, max_iter=par.max_iter, abs_tol=par.abs_tol,
                     rel_tol=par.rel_tol)
        if trace is not None:
            trace.extend((it, w, float("nan"), ub, lb) for it, w, ub, lb in r["trace"])
        res = dict(iters=r["iters"], setup_s=0.0, ub=r["ub"], lb=r["lb"], per_iter_ms=0.0, push_s=0.0,
                   iters_f32=0, device_ms=0.0, stop_reason=r["stop"])
        return res, r["p_fit"], None


def record(res):
    return dict(distance=res.distance, lb=res.lb, ub=res.ub, exit_flag=res.exit_flag, iterations=res.iterations,
                p_fit=np.asarray(res.p_fit).tolist(), method=res.method)


def main(ref_root):
    from unittest import mock
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/numba_cache_binding")
    sys.modules.setdefault("cupy", mock.MagicMock(name="cupy"))
    sys.path.insert(0, ref_root)
    from solver import rum_solver as ref
    from rumb import rum_solver as mine
    from rumb import RUM
    from rumb.instances import mixture_instance
    import rumb_backend_stub
    mine._CTX[0] = HostEngine()
    rumb_backend_stub.install(ref, mine)
    m, a, p = mixture_instance(6, 1.0, K=5, N=100, seed=3)
    kw = dict(method="bm_admm", method_args={"dtype": "float64"}, abs_tol=1e-6, rel_tol=0.0)
    out = {"reference": record(ref.RUM(m, a, p).calculate_distance(**kw)),
           "rumb": record(RUM(m, a, p).calculate_distance(**kw))}
    print(json.dumps(out))


if __name__ == "__main__":
    main(sys.argv[1])
