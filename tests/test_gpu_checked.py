"""Bounds-checked build: the parity cases rerun on libdream_das_checked.so,
whose gathers test every A-scan index against the extent of Y (the
memory-checker run for the CUDA kernels). Images must match and no index may
fall outside Y.
"""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_checked_build_no_violations():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = os.path.join(ROOT, "dream_b200", "libdream_das_checked.so")
    assert os.path.exists(lib), "build it with `python -m dream_b200.build --checked`"
    env = dict(os.environ, DREAM_DAS_CHECKED="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "checked_run.py")], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["runs"] > 100 and out["plans"] > 10
    assert out["mismatches"] == []
    assert out["violations"] == 0
