"""The stencil kernels replace IEEE FP32 division by the update divisor with
a multiply-based correctly rounded division (Markstein's correction in FP64,
rounded once to FP32). This test compiles a small CUDA program
around the library's device function and checks it against IEEE division on
the GPU for all 2^32 numerators with the pressure divisor 6 and, for
diffusion divisors, for a sample of numerators plus every tiny one
(0 < |n| < 2^-99); bit equality is required."""

import pathlib
import shutil
import subprocess

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


@pytest.mark.gpu
def test_update_division_is_ieee(tmp_path, cuda):
    exe = tmp_path / "division_check"
    subprocess.run([NVCC, "-std=c++20", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", f"-I{ROOT / 'include'}", f"-I{ROOT / 'stable-fluids_b200' / 'csrc'}",
                    str(ROOT / "tests" / "kernels" / "division_check.cu"), "-o", str(exe), "-lcuda"], check=True, capture_output=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    lines = [l.split() for l in r.stdout.splitlines() if l.strip()]
    assert len(lines) == 5, r.stdout + r.stderr
    assert int(lines[0][1]) == 2 ** 32 - 2 ** 24  # every finite FP32 value for divisor 6
    for d, checked, bad in lines:
        assert int(bad) == 0, (d, checked, bad)
    assert r.returncode == 0
