"""The C-ABI library builds for sm_100a, loads without a GPU and exports every
entry point the headers under include/ declare.  No device calls."""
import ctypes
import os
import re

import pytest

from scadyn_b200 import api, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(scd_[A-Za-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_library_builds_and_loads():
    path = build.build()
    assert os.path.exists(path)
    lib = ctypes.CDLL(path)
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_binding_covers_header():
    from scadyn_b200 import server
    assert sorted(api.EXPORTS + server.EXPORTS) == declared_symbols()


def test_api_binds_all_signatures():
    from scadyn_b200 import server
    lib = server._lib()
    for name in api.EXPORTS + server.EXPORTS:
        assert getattr(lib, name).restype is not None


def test_no_device_is_reported_not_crashed():
    """Without a GPU scd_create returns SCD_NO_DEVICE instead of failing."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(api.ScadynError) as e:
        api.Solver(8, 8, 8, 1.0, (0, 0, 0), 10)
    assert e.value.code == api.SCD_NO_DEVICE


def test_c_consumer_compiles_links_and_runs(tmp_path):
    """The headers are plain C: a C program includes both, links the library
    and calls through it (without a GPU, scd_create reports SCD_NO_DEVICE)."""
    import subprocess
    import torch
    src = tmp_path / "consumer.c"
    src.write_text(r'''
#include <stdio.h>
#include "scadyn_gpu.h"
#include "scadyn_server.h"
int main(void) {
    scd_grid_desc d = {8, 8, 8, 1.0, {0, 0, 0}, 10, 0, 2, 1, 0};
    scd_ctx *c = 0;
    int rc = scd_create(&c, &d);
    printf("%d\n", rc);
    if (c) scd_destroy(c);
    return 0;
}
''')
    lib = build.build()
    exe = tmp_path / "consumer"
    subprocess.check_call(["gcc", "-std=c99", "-Wall", "-Werror", str(src), "-I", os.path.join(ROOT, "include"),
                           lib, "-Wl,-rpath," + os.path.dirname(lib), "-o", str(exe)])
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.strip()
    if not torch.cuda.is_available():
        assert int(out) == api.SCD_NO_DEVICE
    else:
        assert int(out) == api.SCD_OK


def test_server_estimate_is_host_side_and_monotone():
    """scd_server_estimate (the admission figure) needs no device: it grows
    with the mesh, the VSWF order and FP64 storage of the near zone, and
    counts both precision forms' buffers."""
    from scadyn_b200 import meshgen
    from scadyn_b200 import server as srv
    lib = srv._lib()
    import ctypes as C

    def est(mesh, Nmax, storage=api.STORE_C64, precision=api.PREC_MIXED):
        r, keep = srv.Server._request(None, mesh, 1.0 / mesh.a, 1.8, Nmax, storage=storage, precision=precision)
        b = C.c_int64()
        assert lib.scd_server_estimate(C.byref(r), C.byref(b)) == api.SCD_OK
        return b.value

    small, big = meshgen.sphere(4, seed=1), meshgen.sphere(7, seed=1)
    assert est(big, 4) > est(small, 4) > 0
    assert est(small, 8) > est(small, 4)
    fp64 = api.PREC_FP64
    assert est(small, 4, storage=api.STORE_C128, precision=fp64) > est(small, 4, precision=fp64) > 0
    # the mixed form with complex64 storage adds the tensor-core tile planes
    assert est(small, 4) > est(small, 4, precision=fp64)
