"""rumb: certified random-utility (RUM) distances on B200 GPUs.

The hot paths (BM-ADMM's iteration and float64 certificate, Flow-CG's Bellman-Ford pricing) run
in librumb.so, hand-written CUDA for sm_100a behind a C ABI (include/rumb.h); this package is the
host side, with the reference's interface:

    from rumb import RUM
    res = RUM(menu, alternative, p_hat).calculate_distance(method="bm_admm")

    from rumb import cells_from_panel              # rum's rows from a panel / replies table
    rum = RUM(*cells_from_panel(panel, 25), num_alternatives=25)
    pv = rum.bootstrap(panel=panel).p_value()
"""
from .rum_solver import RUM, Result, Session  # noqa: F401
from .draws import cells_from_panel  # noqa: F401
