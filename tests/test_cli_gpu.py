"""The drop-in command line driver produces the reference's output file."""
import os
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu
G = os.path.join(ROOT, "tests", "golden")


def test_gpsm_run_output_is_byte_identical_to_the_reference(gpu, tmp_path):
    out = tmp_path / "ans.txt"
    exe = os.path.join(ROOT, "gpsm_b200", "gpsm_run")
    r = subprocess.run([exe, os.path.join(G, "small_er_data.g"), os.path.join(G, "small_er_query.g"), str(out), "0"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "match used:" in r.stderr
    ref = open(os.path.join(G, "small_er_ans.txt"), "rb").read()
    assert open(out, "rb").read() == ref
