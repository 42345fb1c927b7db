"""The reference-side binding (tests/rumb_backend_stub.py) installed in
the reference's own RUM class: calculate_distance(method="bm_admm") through the reference's
planner and runner tables reaches rumb's planner and runner, and returns the Result rumb's own RUM
returns (distance, bracket, exit flag, iterations, p_fit). Runs where the reference's source tree
is present (it is never copied here, and the GPU box does not have it); the GPU engine is the host
stand-in of tests/reference_binding_run.py."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "baseline"))
import build_ref  # noqa: E402

ROOT_REF = build_ref.reference_root()


@pytest.mark.skipif(ROOT_REF is None, reason="the reference's source tree is not on this machine")
def test_reference_rum_with_the_binding_returns_rumbs_result():
    r = subprocess.run([sys.executable, os.path.join(HERE, "reference_binding_run.py"), ROOT_REF],
                       capture_output=True, text=True, timeout=600, cwd="/tmp")
    assert r.returncode == 0, r.stderr[-3000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    ref, mine = out["reference"], out["rumb"]
    assert ref["method"] == mine["method"] == "bm_admm"
    assert ref["exit_flag"] == mine["exit_flag"] == 1
    assert ref["iterations"] == mine["iterations"]
    assert ref["distance"] == mine["distance"] and ref["lb"] == mine["lb"] and ref["ub"] == mine["ub"]
    np.testing.assert_array_equal(ref["p_fit"], mine["p_fit"])
    assert mine["ub"] - mine["lb"] <= 1e-6
