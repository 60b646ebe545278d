"""The linear basis as pseudo-tets (scadyn_b200/csrc/linear_basis.h), host
build of the library's own functions: the expanded 3x3 blocks, mirrored only
between different tets, rebuild matmul_Acorr's near-zone matrix in the
unknown order basis_unknown gives, and that order is a bijection; the box
split keeps a tet's basis functions in one group (constant basis: unchanged)."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "scadyn_b200", "csrc")


def test_linear_blocks_expand_to_matmul_Acorr(tmp_path):
    exe = tmp_path / "linear_basis_check"
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    subprocess.check_call([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2",
                           "-I", CSRC, os.path.join(HERE, "linear_basis_check.cu"), "-o", str(exe)])
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 mismatches" in r.stdout


def test_box_split_keeps_whole_tets(tmp_path):
    exe = tmp_path / "linear_basis_split_check"
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    subprocess.check_call([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2",
                           "-I", CSRC, os.path.join(HERE, "linear_basis_split_check.cu"), "-o", str(exe)])
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 failures" in r.stdout
