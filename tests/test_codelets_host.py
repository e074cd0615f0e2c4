"""CPU: every register codelet (radix 2..64, including the composite ones) is
compiled for the host with nvcc and checked against a direct DFT in double."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("nvcc") is None and not os.path.exists("/usr/local/cuda/bin/nvcc"),
                    reason="nvcc not available")
def test_codelets_against_direct_dft(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = tmp_path / "codelet_check"
    src = os.path.join(ROOT, "tests", "host", "codelet_check.cu")
    subprocess.check_call([nvcc, "-std=c++17", "--expt-relaxed-constexpr", "-Wno-deprecated-gpu-targets",
                           "-I", os.path.join(ROOT, "sip_b200", "csrc"), "-o", str(exe), src])
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL OK" in r.stdout
