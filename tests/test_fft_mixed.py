"""The mixed-radix register line FFT for 5-smooth padded lengths
(scadyn_b200/csrc/fft_mixed.cuh) agrees with a direct DFT (host build of the
same device code, the T threads of a line run phase by phase): relative error
< 1e-14 (FP64), < 1e-6 (FP32) for P = 80 ... 320, T = 4 and 8."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "scadyn_b200", "csrc")


def test_mixed_radix_fft_matches_direct_dft(tmp_path):
    exe = tmp_path / "fft_mixed_check"
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    subprocess.check_call([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2", "-I", CSRC,
                           os.path.join(HERE, "fft_mixed_check.cu"), "-o", str(exe)])
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
