"""The host check of the slot and tile tables (scadyn_b200/csrc/layout_check.h),
which upload_layout runs before every near-zone layout reaches the device: it
accepts the layouts the library builds (set_order and build_tile_layout run on
the host from the library's objects, for the constant and the linear basis, on
a sphere's binning) and rejects each planted inconsistency of a hand-built
layout."""
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(ROOT, "scadyn_b200", "csrc")


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    from scadyn_b200 import build
    build.build()
    objs = [os.path.join(ROOT, "scadyn_b200", "_build", s.replace(".cu", ".o")) for s in build.SOURCES]
    out = tmp_path_factory.mktemp("layout") / "layout_check"
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    subprocess.check_call([nvcc, *build.ARCH, "-std=c++17", "-O1", "--expt-relaxed-constexpr", "-I", CSRC,
                           "-I", os.path.join(ROOT, "include"), os.path.join(HERE, "layout_check_main.cu"),
                           *objs, "-o", str(out)])
    return str(out)


@pytest.mark.parametrize("nb", [1, 4])
def test_layout_check(exe, small_sphere, nb):
    from oracle import oracle as O
    g = O.Geometry(small_sphere.coord, small_sphere.etopol, small_sphere.param, k=1.0 / small_sphere.a, grid_size=1.8)
    cx, cy, cz = g.cube_dims
    cent = small_sphere.coord[small_sphere.etopol - 1].mean(axis=1)
    M = np.floor((cent - g.min_coord) / g.box_delta).astype(np.int64)
    cube = (M[:, 0] + cx * (M[:, 1] + cy * M[:, 2])).astype(np.int32)
    cube = np.repeat(cube, nb)
    req = np.array([cx, cy, cz, nb, cube.size], np.int32).tobytes() + cube.tobytes()
    r = subprocess.run([exe], input=req, capture_output=True)
    out = r.stdout.decode()
    assert r.returncode == 0, out + r.stderr.decode()
    assert "production layout: ok" in out
    assert "planted:" in out
