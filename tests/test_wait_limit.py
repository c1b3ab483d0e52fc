"""The host wait of a compare launch is bounded (CPU only, no device).

A compare call waits for its launch by polling the stream. If the device
stopped making progress that wait must end with an error, not block the
caller for good. tests/wait_limit_driver.cpp drives the product's wait
(poll_with_limit in dgpu_common.h) with fake stream queries, one of which
stalls forever, injected on the host."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_compare_wait_ends_with_a_timeout_on_a_stalled_stream(tmp_path):
    import shutil

    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    cuda_inc = os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(nvcc))), "include")
    exe = str(tmp_path / "wait_limit_driver")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "dada2-rs_b200", "csrc"), "-I", cuda_inc,
                    os.path.join(ROOT, "tests", "wait_limit_driver.cpp"), "-o", exe, "-pthread"], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60,
                       env={**os.environ, "DGPU_WAIT_LIMIT_S": "7"})
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip() == "ok"
