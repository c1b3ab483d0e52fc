"""The denoising service's batching rule on the CPU (tests/service_take_driver.cpp):
requests of the oldest request's length class are taken in arrival order while
the estimated device-memory footprint fits the budget; the oldest request is
always taken when nothing is in flight; other classes keep their order; a held
service takes nothing. Host only: no GPU."""
import os
import shutil
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_service_batching_rule(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    cuda = os.path.dirname(os.path.dirname(os.path.realpath(nvcc)))
    lib = os.path.join(cuda, "lib64")
    exe = str(tmp_path / "take")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "dada2-rs_b200", "csrc"), "-I",
                    os.path.join(ROOT, "include"), "-I", os.path.join(cuda, "include"),
                    os.path.join(ROOT, "tests", "service_take_driver.cpp"), "-o", exe, "-L", lib,
                    f"-Wl,-rpath,{lib}", "-lcudart", "-lpthread"], check=True, capture_output=True)
    res = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert res.returncode == 0, res.stdout
