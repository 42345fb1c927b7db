"""rumb: certified random-utility (RUM) distances on B200 GPUs.

The hot paths (BM-ADMM's iteration and float64 certificate, Flow-CG's Bellman-Ford pricing) run
in librumb.so, hand-written CUDA for sm_100a behind a C ABI (include/rumb.h); this package is the
host side, with the reference's interface:

    from rumb import RUM
    res = RUM(menu, alternative, p_hat).calculate_distance(method="bm_admm")
"""
from .rum_solver import RUM, Result, Session  # noqa: F401
