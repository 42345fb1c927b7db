"""Generates tests/golden/draws.npz by running the reference's own bootstrap draws (CPU code).

    python tests/golden/make_draws_golden.py <reference root>

It imports solver/inference/draws.py from the path given (read-only, never copied): for a seeded
respondent panel (rumb.instances.panel_instance, n = 8) it records the reference's weight rows and
every draw's rows (Draws.rows, solver/inference/draws.py:151-159,247-285) for every weight scheme,
a replies table's draws (MenuDraws) and cells (cells_from_panel), three refusal messages,
and the interval formulas (solver/inference/hong_li.py:81-107) on seeded brackets.
The tests compare the library's draws (host builder and GPU kernel) against this file; nothing at
test time reads the reference itself.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "rum-testing-gpu_b200"))


def main(ref_root):
    sys.path.insert(0, ref_root)
    from solver.inference import draws as RD
    from rumb.instances import panel_instance
    panel, (m, a, p) = panel_instance(8, 0.4, 40, 6, 4, seed=21)
    out = dict(panel_respondent=np.asarray(panel["respondent"], dtype=np.int64),
               panel_menu=np.asarray(panel["menu"], dtype=np.int64),
               panel_chosen=np.asarray(panel["chosen"], dtype=np.int64),
               menu=np.asarray(m, dtype=np.int64), alternative=np.asarray(a, dtype=np.int64),
               p_hat=np.asarray(p, dtype=np.float64))
    for weights in RD.WEIGHTS:
        d = RD.Draws(panel, m, a, p, B=12, weights=weights, seed=5)
        out["W_" + weights] = np.asarray(d.W, dtype=np.float64)
        out["rows_" + weights] = np.asarray(d.rows(np.arange(12)), dtype=np.float64)
    # a replies table (the panel without respondents) and its own rows
    replies = dict(menu=out["panel_menu"], chosen=out["panel_chosen"])
    rm, ra, rp = RD.cells_from_panel(replies, 8)
    out["rep_menu"], out["rep_alt"], out["rep_p"] = rm, ra, rp
    md = RD.MenuDraws(replies, rm, ra, rp, B=12, seed=5)
    out["rows_replies"] = np.asarray(md.rows(np.arange(12)), dtype=np.float64)
    am, aa, ap = RD.cells_from_panel(panel, 8, alternatives=[0])
    out["alt0_menu"], out["alt0_alt"], out["alt0_p"] = am, aa, ap
    # the messages of three refusals
    msgs = []
    for bad in (lambda: RD.Draws(panel, m, a, p + 0.01, B=2),
                lambda: RD.Draws(dict(respondent=out["panel_respondent"], menu=out["panel_menu"]), m, a, p, B=2),
                lambda: RD.Draws(panel, np.r_[m, 255], np.r_[a, 0], np.r_[p, 0.5], B=2)):
        try:
            bad()
            msgs.append("")
        except ValueError as e:
            msgs.append(str(e))
    out["errors"] = np.array(msgs)
    # the interval formulas (solver/inference/hong_li.py:81-107) on seeded brackets
    from solver.inference import hong_li as HL
    rng = np.random.default_rng(9)
    L = rng.random(200) * 3.0
    U = L + rng.random(200) * 0.5
    dev = rng.random(200)
    out["hl_L"], out["hl_U"], out["hl_dev"] = L, U, dev
    for j, alpha in enumerate((0.05, 0.1, 0.5)):
        low, high, q = HL.ci_lower(1.2, 1.3, L, U, alpha, 22.8, 0.124)
        out["hl_ci_%d" % j] = np.array([low, high, q[0], q[1]])
        out["hl_di_%d" % j] = np.array(HL.distance_interval(1.2, 1.3, dev, alpha))
        out["hl_band_%d" % j] = np.array(HL.quantile_band(L, U, alpha))
    grid = [(a_, o_, 100, al) for a_ in (0, 3, 5, 9) for o_ in (0, 2, 6) for al in (0.05, 0.1)]
    out["hl_locked_in"] = np.array(grid, dtype=np.float64)
    out["hl_locked"] = np.array([HL.locked(int(a_), int(o_), int(b_), al) for a_, o_, b_, al in grid])
    np.savez_compressed(os.path.join(HERE, "draws.npz"), **out)
    print("wrote", os.path.join(HERE, "draws.npz"))


if __name__ == "__main__":
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "baseline"))
    import build_ref
    root = sys.argv[1] if len(sys.argv) > 1 else build_ref.reference_root()
    if root is None:
        raise SystemExit("the reference's source tree was not found (give it as the argument, or RUM_REFERENCE_ROOT)")
    main(root)
