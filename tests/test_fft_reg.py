"""The register line FFT used by the FFT passes for P = 64 and 128 agrees
with a direct DFT (host build of the same device code, the 8 threads of a
line run phase by phase): relative error < 1e-14 (FP64), < 1e-6 (FP32)."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "scadyn_b200", "csrc")


def test_register_fft_matches_direct_dft(tmp_path):
    exe = tmp_path / "fft_reg_check"
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    subprocess.check_call([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2", "-I", CSRC, os.path.join(HERE, "fft_reg_check.cu"), "-o", str(exe)])
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
