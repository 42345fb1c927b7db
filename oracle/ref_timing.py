"""Times the reference's own float64 BM-ADMM kernels on this GPU -- TEST INFRASTRUCTURE ONLY.

    python oracle/ref_timing.py [workload]

Replays solve_kadmm_v2's iteration with the reference's kernels (oracle/ref_replay.py: NVRTC-built
from the reference's source strings, Bfly2's calibrated stage plan, one_iter captured as a CUDA
graph as the reference's use_graph path does) and its float64 check (push_to_ub64 +
fw_lb_rows_gpu), and prints per-iteration and per-check milliseconds as JSON. The launches are
issued from Python like the reference's, without CuPy's own per-call overhead.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "rum-testing-gpu_b200"))

import ref_replay  # noqa: E402
from rumb.instances import config_instance  # noqa: E402
from rumb.params import bm_beta_default  # noqa: E402


def main(workload="n18_d1pct_k50"):
    n, m, a, p = config_instance(workload)[:4]
    r = ref_replay.BMReplay(n, m, a, p, bm_beta_default(p.size))
    out = dict(workload=workload, plan=r.plan, t_iter_graph_ms=r.time_iterations(50, graph=True),
               t_iter_eager_ms=r.time_iterations(20, graph=False), t_check_ms=r.time_check(5))
    print(json.dumps(out))


if __name__ == "__main__":
    main(*sys.argv[1:])
