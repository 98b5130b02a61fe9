"""The reference install and its plain-path runner (baseline/), on the CPU.

bench.py times the reference's own torch path beside the fused kernel; these
tests check that the install is the reference's code, unmodified, and that the
runner produces the fields the bench line reads.
"""

import json
import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(REPO, "baseline", "_ref", "torch_sim")
SRC = "/root/reference/torch_sim"

needs_install = pytest.mark.skipif(not os.path.isdir(REF),
                                   reason="reference not installed in baseline/_ref")


@needs_install
@pytest.mark.skipif(not os.path.isdir(SRC), reason="reference source tree absent")
def test_installed_reference_is_the_source_tree():
    sys.path.insert(0, os.path.join(REPO, "baseline"))
    try:
        import install_ref
    finally:
        sys.path.pop(0)
    assert install_ref._same_tree(SRC, REF)
    # and the other way round: nothing added beyond byte-compiled caches
    assert install_ref._same_tree(REF, SRC)


@needs_install
def test_reference_runner_reports_rate_and_force_error():
    cmd = [sys.executable, os.path.join(REPO, "baseline", "ref_plain_gpu.py"), "--device", "cpu",
           "--n-systems", "16", "--systems", "2", "--steps", "1", "--warmup", "1",
           "--dtype", "float64"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads([x for x in r.stdout.splitlines() if x.startswith("{")][-1])
    assert out["systems"] == 2 and out["atoms"] > 0 and out["value"] > 0
    assert out["threads"] >= 1
    # float64 against float64 by the same model: the same forces
    assert out["force_err_vs_fp64"] == 0.0
