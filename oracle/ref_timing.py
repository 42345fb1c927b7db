"""Times the reference's own float64 BM-ADMM kernels on this GPU -- TEST INFRASTRUCTURE ONLY.

    python oracle/ref_timing.py [workload]
    python oracle/ref_timing.py pricing [workload]     # the reference's pricing kernels per sweep

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


def pricing(workload="n18_d05pct_k50", reps=10):
    """The reference's pricing kernels on one sweep's layers, timed with CUDA events around the
    layer launches only (no host reads between layers, no backtrace): a lower bound of its sweep.
    Stream storage: bf_stream_u24 / bf_stream_u16 (one 256-thread CTA per 1024 ranks, x-major rows
    scanned per rank); mask storage: bf_update (a thread per subset)."""
    import math
    import numpy as np
    import torch
    from rumb import flow_cg
    n, m, a, p = config_instance(workload)[:4]
    menus, alts, p32, offsets, _ = flow_cg.prepare_choice_data(m, a, p, n)
    scores = np.random.default_rng(0).standard_normal(menus.size).astype(np.float32)
    L = ref_replay._Launcher(ref_replay._mods()["pricing"])
    counts = [math.comb(n, k) for k in range(n + 1)]
    cap, k_pred = max(counts), n - 10
    nblk = (cap + 1023) // 1024
    binom = torch.from_numpy(ref_replay._binom(n).view(np.int64)).cuda()
    gm = torch.from_numpy(np.ascontiguousarray(menus).view(np.int64)).cuda()
    gs = torch.from_numpy(scores).cuda()
    go = torch.from_numpy(np.asarray(offsets, dtype=np.uint64).view(np.int64)).cuda()
    out = dict(workload=workload, rows=int(menus.size))
    I, ULL = ref_replay._I, ref_replay._ULL

    def timed(sweep):
        for _ in range(2):
            sweep()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            sweep()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    for mode in ("u24", "u16"):
        vbuf = [torch.zeros(cap, dtype=torch.int16, device="cuda") for _ in range(2)]
        lbuf = [torch.zeros(cap, dtype=torch.uint8, device="cuda") for _ in range(2)]
        mbuf = [torch.zeros(nblk, dtype=torch.float32, device="cuda") for _ in range(2)]
        ebuf = [torch.zeros(nblk, dtype=torch.float32, device="cuda") for _ in range(2)]
        pred = {k: torch.zeros(counts[k], dtype=torch.uint8, device="cuda") for k in range(k_pred, n + 1)}
        dummy = torch.zeros(1, dtype=torch.uint8, device="cuda")

        def sweep(mode=mode, vbuf=vbuf, lbuf=lbuf, mbuf=mbuf, ebuf=ebuf, pred=pred, dummy=dummy):
            cur, prev = 0, 1
            for k in range(1, n + 1):
                store = 1 if k >= k_pred else 0
                pk = pred[k] if store else dummy
                if mode == "u24":
                    args = [binom, (I, n), (I, k), (ULL, counts[k]), vbuf[prev], lbuf[prev], mbuf[prev], ebuf[prev],
                            vbuf[cur], lbuf[cur], mbuf[cur], ebuf[cur], pk, (I, store), gm, gs, go]
                else:
                    args = [binom, (I, n), (I, k), (ULL, counts[k]), vbuf[prev], mbuf[prev], ebuf[prev],
                            vbuf[cur], mbuf[cur], ebuf[cur], pk, (I, store), gm, gs, go]
                L.launch("bf_stream_" + mode, (counts[k] + 1023) // 1024, 256, args)
                cur, prev = prev, cur

        out[mode + "_layers_ms"] = timed(sweep)
    V = torch.zeros(1 << n, dtype=torch.float32, device="cuda")
    P = torch.zeros(1 << n, dtype=torch.uint8, device="cuda")
    gm32 = torch.from_numpy(np.asarray(menus, dtype=np.uint64).astype(np.uint32).view(np.int32)).cuda()
    states = [torch.from_numpy(ref_replay._gosper(n, c)).cuda() for c in range(n + 1)]

    def mask_sweep():
        for c in range(1, n + 1):
            ns = states[c].numel()
            L.launch("bf_update", (ns + 255) // 256, 256, [V, P, gm32, gs, go, states[c], (I, ns)])

    out["mask_layers_ms"] = timed(mask_sweep)
    print(json.dumps(out))


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "pricing":
        pricing(*sys.argv[2:])
    else:
        main(*sys.argv[1:])
