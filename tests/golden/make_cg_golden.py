"""Records the Flow-CG column sequence of the n18_d05pct_k50 workload (n = 18, 0.5 % menus) as a golden vector.

    python tests/golden/make_cg_golden.py          # on a GPU host, after build()

The library's CG loop runs n18_d05pct_k50 (n = 18, 0.5 % menus, K = 50, N = 500) to abs 1e-5 in
uint24 storage and for 1,000 columns in uint16 storage (whose quantization margin keeps its bound
above abs 1e-5 at this density); at every iteration the residual it priced is priced again by the
reference's own stream kernels (baseline/ref_replay.py, NVRTC-compiled from the reference's
source) and the run is kept only if every ranking is the reference kernels' ranking. The file
holds the rankings (rank positions, one row per CG iteration) and the final bracket per storage;
tests/test_gpu_cg.py checks the library against it on GPUs where the reference kernels are not
built.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(ROOT, "rum-testing-gpu_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "baseline"),
          os.path.dirname(HERE)):
    if p not in sys.path:
        sys.path.insert(0, p)


def main():
    import ref_replay
    import test_gpu_ref_replay as T
    from rumb import _lib
    if not ref_replay.available():
        raise SystemExit("baseline/_ref is not built: run build() where the reference tree is present")
    ctx = _lib.Context(0)
    out = {}
    for mode in ("u24", "u16"):
        res, bad = T._config3_run(ctx, mode, check_reference=True)
        if bad or res["stop_reason"] != ("gap_abs" if mode == "u24" else "max_iters"):
            raise SystemExit("%s: not recorded (%s, %d mismatches: %s)" % (mode, res["stop_reason"], len(bad), bad[:3]))
        out["picked_" + mode] = np.array(res["picked"], dtype=np.int32)
        out["bracket_" + mode] = np.array([res["lb"], res["distance"]])
        print(mode, len(res["picked"]), "columns", res["lb"], res["distance"])
    np.savez_compressed(os.path.join(HERE, "cg_config3.npz"), **out)


if __name__ == "__main__":
    main()
