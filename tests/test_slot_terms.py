"""The slot-major assembly's per-block term lists, built on the host
(bounce_b200/csrc/topology.cpp), checked on the CPU: each term couples its
block's row and column, a block's terms follow the row's force-list order,
every element sits in (vertices)^2 blocks, and the codes lie where the
kernel reads them.  The check is a small C++ program (slot_terms_check.cpp)
compiled with g++ against the library's topology source."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


@pytest.mark.skipif(shutil.which("g++") is None, reason="no g++")
def test_slot_term_lists(tmp_path):
    exe = tmp_path / "slot_terms_check"
    subprocess.run(["g++", "-O1", "-std=c++17", "-o", str(exe), os.path.join(HERE, "slot_terms_check.cpp"),
                    os.path.join(ROOT, "bounce_b200", "csrc", "topology.cpp")], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip().endswith("ok")
