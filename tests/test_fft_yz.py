"""The fused y-z FFT pass (scadyn_b200/csrc/fft_yz.cuh) run on the host
thread by thread, in the kernel's phase order, agrees with a direct separable
DFT convolution (FP64 < 1e-13, FP32 < 2e-6) for C2's lengths, powers of two
and 5-smooth lengths, with padding rows and partial z chunks; no write
leaves the plane or the shared-memory image."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "scadyn_b200", "csrc")


def test_fused_yz_pass_matches_direct_convolution(tmp_path):
    exe = tmp_path / "fft_yz_check"
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    subprocess.check_call([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2", "-I", CSRC,
                           os.path.join(HERE, "fft_yz_check.cu"), "-o", str(exe)])
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
