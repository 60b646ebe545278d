"""The tensor-core near-zone schedules (scadyn_b200/csrc/near_mma.cuh; split,
merged and wide -- the merged schedule over 32 right-hand sides -- the last
two also checked for their constant descriptor steps), run on
the host through an interpreter of the tcgen05 operand descriptors: the f16
hi/lo planes and x blocks built by the kernels' own element functions give
the complex products A x and A^T x of a tile to FP32 accuracy (relative error
< 2e-6) for every group-size regime (M = 64 and 128, partial K steps), with
absent and skipped right-hand sides, and no instruction reads past the tile,
its x block and the ring slack the kernel reserves."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "scadyn_b200", "csrc")


def test_near_mma_schedule_reproduces_tile_products(tmp_path):
    exe = tmp_path / "near_mma_check"
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    subprocess.check_call([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2",
                           "--expt-relaxed-constexpr", "-I", CSRC, os.path.join(HERE, "near_mma_check.cu"),
                           "-o", str(exe)])
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "60 of 60 tiles ok" in r.stdout
