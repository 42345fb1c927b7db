"""Records the reference's own Flow-CG pricing kernels' outputs as golden vectors.

    python tests/golden/make_replay_golden.py <out.npz>        # on a GPU host, after build()

The reference's kernel source strings are extracted into baseline/_ref by baseline/build_ref.py (at
build time, where the reference tree is present), compiled here by NVRTC with the reference's
options and launched through baseline/ref_replay.py. For seeded instances and seeded float32
scores, the file keeps the scores and the reference kernels' outputs: Vmax (float32), rank_pos,
margin and per-layer steps for the f32, u16 and u24 stream pricers, and Vmax / rank_pos for the
mask sweep. The instances themselves are regenerated from their seeds by the tests. These are the
pins of the u16/u24 columns that no test of the reference holds; the oracle is checked against them
on the CPU (tests/test_oracle_golden.py) and the library on the GPU (tests/test_gpu_cg.py).
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


def cases():
    """(name, n, menu, alt, p) of the recorded instances (seeded; the tests rebuild them)."""
    import paper_instances as PI
    from rumb.instances import config_instance
    out = []
    for name, cd, n in (("pair8", PI.gen_pairwise(8)[0], 8), ("med12", PI.gen_medium(12, mult=3)[0], 12),
                        ("pair16", PI.gen_pairwise(16)[0], 16)):
        out.append((name, n, cd[:, 0], cd[:, 1], cd[:, 2]))
    n, m, a, p = config_instance("n18_d05pct_k50")
    out.append(("n18_d05pct", n, m, a, p))
    return out


def scores_for(name, size, trial):
    rng = np.random.RandomState(1000 + 17 * trial + sum(map(ord, name)))
    return (rng.randn(size) * (1.0 if trial == 0 else 0.02)).astype(np.float32)


def main(out):
    import oracle as O
    import ref_replay
    if not ref_replay.available():
        raise SystemExit("baseline/_ref is not built: run build() where the reference tree is present")
    rec = {}
    for name, n, m, a, p in cases():
        menus, alts, p32, offsets, _ = O.cg_layout(n, m, a, p)
        for trial in range(2):
            s = scores_for(name, menus.size, trial)
            key = "%s_t%d" % (name, trial)
            rec[key + "_scores"] = s
            for mode in ("f32", "u16", "u24"):
                v, r, mg, steps = ref_replay.price_stream(menus, alts, s, offsets, n, mode=mode)
                rec["%s_%s_vmax" % (key, mode)] = np.float32(v)
                rec["%s_%s_rank" % (key, mode)] = np.asarray(r, dtype=np.int32)
                rec["%s_%s_margin" % (key, mode)] = np.float64(mg)
                rec["%s_%s_steps" % (key, mode)] = np.asarray(steps, dtype=np.float32)
            if n <= 16:
                v, r = ref_replay.price_mask(menus, s, offsets, n)
                rec[key + "_mask_vmax"] = np.float32(v)
                rec[key + "_mask_rank"] = np.asarray(r, dtype=np.int32)
    np.savez_compressed(out, **rec)
    print("wrote %s (%d arrays)" % (out, len(rec)))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "pricer_replay.npz"))
