"""The library against the reference's own kernels, JIT-compiled by NVRTC from the reference's
source strings and replayed (oracle/build_ref.py, oracle/ref_replay.py): Flow-CG pricing must
agree bit for bit (values, rankings, per-layer steps). Skipped where oracle/_ref was not built
(it needs the reference's source tree at build time)."""
import numpy as np
import pytest

import oracle as O
import paper_instances as PI
import ref_replay
from rumb import _lib
from rumb.instances import config_instance

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_replay.available(), reason="oracle/_ref not built")]


def _cases():
    yield "pair8", PI.gen_pairwise(8)[0], 8
    yield "med12", PI.gen_medium(12, mult=3)[0], 12
    yield "pair16", PI.gen_pairwise(16)[0], 16
    n, m, a, p = config_instance("n18_d05pct_k50")
    yield "n18_d05pct", np.column_stack([m, a, p]).astype(np.float64), n


CASES = list(_cases())


@pytest.mark.parametrize("name,cd,n", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("mode", ["f32", "u16", "u24"])
def test_stream_pricer_matches_reference_kernels(ctx, name, cd, n, mode):
    menus, alts, p32, offsets, _ = O.cg_layout(n, cd[:, 0], cd[:, 1], cd[:, 2])
    pr = _lib.Pricer(ctx, n, menus, offsets, mode=mode)
    rng = np.random.RandomState(11)
    for trial in range(2):
        scores = (rng.randn(menus.size) * (1.0 if trial == 0 else 0.02)).astype(np.float32)
        v_ref, r_ref, m_ref, steps_ref = ref_replay.price_stream(menus, alts, scores, offsets, n, mode=mode)
        v, r, m, steps = pr.price(scores, want_steps=True)
        assert v == v_ref, (v, v_ref)
        np.testing.assert_array_equal(r, r_ref)
        np.testing.assert_array_equal(steps, steps_ref)
        assert abs(m - m_ref) <= 1e-6 * max(1.0, m_ref)      # the reference sums the steps in float32
    pr.close()


@pytest.mark.parametrize("name,cd,n", CASES[:3], ids=[c[0] for c in CASES[:3]])
def test_mask_pricer_matches_reference_kernel(ctx, name, cd, n):
    menus, alts, p32, offsets, _ = O.cg_layout(n, cd[:, 0], cd[:, 1], cd[:, 2])
    pr = _lib.Pricer(ctx, n, menus, offsets, mode="mask")
    scores = np.random.RandomState(5).randn(menus.size).astype(np.float32)
    v_ref, r_ref = ref_replay.price_mask(menus, scores, offsets, n)
    v, r, _ = pr.price(scores)
    assert v == v_ref and np.array_equal(r, r_ref)
