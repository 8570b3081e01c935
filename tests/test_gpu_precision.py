"""The precision study (tests/precision_study.py) at a small size: every dot
precision reaches the stop tolerance in the FP64-recomputed residual, and
its solution agrees with the FP64 CPU solve of the same system."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def test_precision_study_small(tmp_path):
    out = tmp_path / "p.json"
    subprocess.run([sys.executable, os.path.join(HERE, "precision_study.py"), "--side", "96", "--steps", "4",
                    "--check", "2,4", "--workers", "2", "--json", str(out)], check=True, timeout=600)
    r = json.loads(out.read_text())
    assert r["vertices"] == 96 * 96
    for name, s in r["summary"].items():
        assert s["steps_at_cap"] == 0, name
        assert s["cg_residual_max"] <= 1e-4, name
    for c in r["trajectory_checks"] + r["same_system"]:
        # the CG recurrence and the recomputed residual agree to within a few times the tolerance
        assert c["true_residual"] <= 5e-4, c
        assert c["dv_rel_err"] <= 1e-2, c
