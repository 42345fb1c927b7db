"""Generates tests/golden/records.json from the reference's own record writers (CPU code).

    python tests/golden/make_record_golden.py [<reference root>]

It imports solver/rum_solver.py and solver/inference/bootstrap.py from the path given (read-only,
never copied) and records, as JSON text:
  * Result.to_dict() (solver/rum_solver.py:143-149) of a Result built from fixed field values
    (a certified bracket with a trace, method arguments and an info dict);
  * Bootstrap.record() (solver/inference/bootstrap.py:356-370), "when" left out, of a freshly
    built bootstrap of a seeded respondent panel (rumb.instances.panel_instance, n = 8) and of its
    replies table (before any solve: the record's layout, settings, fingerprints, scaling and
    draw summary).
tests/test_host.py builds the same objects with the library and compares the JSON text byte for
byte; nothing at test time reads the reference itself.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "rum-testing-gpu_b200"))
sys.path.insert(0, os.path.join(ROOT, "baseline"))

# the Result the tests build on both sides (field values only; the class comes from each side)
RESULT_FIELDS = dict(exit_flag=3, status="abs_tol and rel_tol met", message="", distance=2.0206668658931326,
                     lb=2.0206569574048343, ub=2.0206668658931326, abs_gap=9.908488298302e-06,
                     rel_gap=4.903568e-06, abs_tol=1e-05, rel_tol=0.0001, met_abs=True, met_rel=True,
                     method="bm_admm", auto_reason="", method_args={"dtype": "float64", "check": 50},
                     iterations=43850, iteration_unit="ADMM iterations", time=4.1, time_setup=0.2,
                     time_solve=3.9, seed=0, trace=[(50, 0.01, 2.5, 0.0), (100, 0.02, 2.1, 1.9)],
                     machine="1x B200", info={"gpu_bytes_planned": 123456, "lb_dtype": "float64"})


def panel_case():
    from rumb.instances import panel_instance
    panel, (m, a, p) = panel_instance(8, 0.4, 40, 6, 4, seed=21)
    return panel, m, a, p


def main(ref_root):
    sys.path.insert(0, ref_root)
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/numba_cache")
    from solver.rum_solver import RUM as RRUM, Result as RResult
    from solver.inference.bootstrap import Bootstrap as RBoot
    from solver.inference.draws import cells_from_panel
    out = {"result_to_dict": json.dumps(RResult(**RESULT_FIELDS).to_dict())}
    panel, m, a, p = panel_case()
    rec = RBoot(RRUM(m, a, p), panel=panel, B=12, weights="multinomial", seed=5).record()
    rec.pop("when")
    out["bootstrap_panel_record"] = json.dumps(rec, indent=1)
    replies = dict(menu=panel["menu"], chosen=panel["chosen"])
    rm, ra, rp = cells_from_panel(replies, 8)
    rec = RBoot(RRUM(rm, ra, rp), replies=replies, B=6, seed=3).record()
    rec.pop("when")
    out["bootstrap_replies_record"] = json.dumps(rec, indent=1)
    path = os.path.join(HERE, "records.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    import build_ref
    root = sys.argv[1] if len(sys.argv) > 1 else build_ref.reference_root()
    if root is None:
        raise SystemExit("the reference's source tree is needed (argument or RUM_REFERENCE_ROOT)")
    main(root)
