"""Host check of the hand-written adjoint (vector-Jacobian products of u2v, MUSCL-minmod,
HLLC, HLLD in all eight fan regions, the explicit collision source and the CFL
candidates) against central finite differences of the forward device functions, compiled
for the host with g++.  No GPU needed."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(ROOT, "pip_b200", "csrc")


def _cuda_include():
    for c in (os.environ.get("CUDA_HOME", ""), "/usr/local/cuda"):
        if c and os.path.isfile(os.path.join(c, "include", "cuda_runtime.h")):
            return os.path.join(c, "include")
    return None


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_adjoint_vjps_match_finite_differences(tmp_path):
    inc = _cuda_include()
    if inc is None:
        pytest.skip("cuda_runtime.h not found")
    exe = tmp_path / "adjoint_fd_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-Wno-unknown-pragmas", "-I", CSRC, "-I", inc,
                    os.path.join(HERE, "adjoint_fd_check.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL OK" in r.stdout
    # every HLLD region was exercised
    line = [l for l in r.stdout.splitlines() if "hlld regions checked" in l][0]
    counts = [int(t.split(":")[1]) for t in line.split()[3:]]
    assert len(counts) == 8 and min(counts) > 0
