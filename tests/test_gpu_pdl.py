"""Programmatic dependent launch changes when the iteration's kernels and the pricing sweeps' layer
kernels are scheduled, never what they compute: a child process with RUMB_PDL=0 (plain stream
order; the switch is read once per process) gives the same iterates and the same priced column,
bit for bit, as this process with it on."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

_WORK = r'''
import sys
import numpy as np
sys.path[:0] = [%(pkg)r, %(tests)r, %(oracle)r]
from rumb import _lib
from rumb.instances import mixture_instance
import oracle as O
import paper_instances as PI
ctx = _lib.Context(0)
n, m, a, p = 12, *mixture_instance(12, 0.1, K=8, N=200, seed=5)
beta = O.beta_default(p.size)
out = {}
for dt in ("float64", "float32"):
    st = ctx.bm_iterate(ctx.bm_problem(n, m, a, p), ctx.bm_params(beta, dtype=dt), None, 60, cold_start=True)
    for k in ("x2", "s", "y", "z"):
        out[dt + "_" + k] = st[k]
cd, _ = PI.gen_pairwise(20)
menus, alts, p32, offsets, _ = O.cg_layout(20, cd[:, 0], cd[:, 1], cd[:, 2])
scores = np.random.RandomState(3).randn(menus.size).astype(np.float32)
for mode in ("mask", "u16"):
    pr = _lib.Pricer(ctx, 20, menus, offsets, mode=mode)
    v, r, mg = pr.price(scores)
    out[mode + "_v"], out[mode + "_r"], out[mode + "_m"] = np.float64(v), r, np.float64(mg)
    pr.close()
np.savez(sys.argv[1], **out)
'''


def _run(path, pdl):
    code = _WORK % dict(pkg=os.path.join(ROOT, "rum-testing-gpu_b200"), tests=HERE, oracle=os.path.join(ROOT, "oracle"))
    env = dict(os.environ, RUMB_PDL=pdl)
    r = subprocess.run([sys.executable, "-c", code, path], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return np.load(path)


def test_pdl_off_gives_the_same_bits(tmp_path):
    on = _run(str(tmp_path / "on.npz"), "1")
    off = _run(str(tmp_path / "off.npz"), "0")
    assert set(on.files) == set(off.files)
    for k in on.files:
        np.testing.assert_array_equal(on[k], off[k], err_msg=k)
