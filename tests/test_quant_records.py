"""The quantised four-wide records' quantiser on the CPU: every decoded child
box contains its exact box (the walk over them can then never prune what the
exact boxes keep) and stays within two steps of it. Compiles
tests/quant_check.cu (host code only) with nvcc and runs it."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


@pytest.mark.skipif(not os.path.exists(NVCC) and shutil.which("nvcc") is None, reason="needs nvcc")
def test_quantised_boxes_contain_exact_boxes(tmp_path):
    exe = str(tmp_path / "quant_check")
    subprocess.run([NVCC if os.path.exists(NVCC) else "nvcc", "-O2", "-std=c++17", "-Xcompiler", "-ffp-contract=off",
                    os.path.join(HERE, "quant_check.cu"), "-o", exe], check=True, capture_output=True, timeout=300)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("ok ")
