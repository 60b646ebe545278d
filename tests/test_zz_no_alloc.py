"""scd_T_assemble_noalloc: T = mat^H X on caller-owned device buffers with no
allocation inside the library.

It serves hosts that cannot let a library call cudaMalloc, such as a Fortran
host whose device memory all comes from its own allocator (CUDA Fortran
device arrays, OpenACC data regions).  Its output must match the T columns
that scd_solve_columns assembles for the same solutions, on two calls in a
row.  This file is named to be collected last."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from scadyn_b200 import api
from tests.gpu_helpers import solver_from_oracle

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_noalloc_T_matches_solve_columns(small_op, small_sphere):
    import torch
    s = solver_from_oracle(small_op)
    try:
        mat = O.vswf2constant(small_sphere.coord, small_sphere.etopol, small_op.geom.k, 2)   # (ncol, n)
        ncol, n = mat.shape
        Tc, iters, X, rc = s.solve_columns(mat, tol=1e-8, want_x=True)   # Tc[c, r] = T(r, c)
        dev = torch.device("cuda:0")
        mat_d = torch.from_numpy(np.ascontiguousarray(mat)).to(dev)      # memory of Fortran mat(n, ncol)
        X_d = torch.from_numpy(np.ascontiguousarray(X)).to(dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        # call 1: all columns
        T1 = torch.zeros((ncol, ncol), dtype=torch.complex128, device=dev)  # memory of T(ncol, ncol)
        api.T_assemble_noalloc(mat_d.data_ptr(), n, ncol, X_d.data_ptr(), ncol, T1.data_ptr(), stream)
        torch.cuda.synchronize(dev)
        assert rel(T1.cpu().numpy(), Tc) < RTOL
        # call 2, right after: a column subset (the scratch keeps call 1's data)
        ncb = 5
        T2 = torch.full((ncb, ncol), complex(np.nan, np.nan), dtype=torch.complex128, device=dev)
        api.T_assemble_noalloc(mat_d.data_ptr(), n, ncol, X_d[:ncb].data_ptr(), ncb, T2.data_ptr(), stream)
        torch.cuda.synchronize(dev)
        assert rel(T2.cpu().numpy(), Tc[:ncb]) < RTOL
    finally:
        s.close()


def test_noalloc_rejects_oversize():
    import torch
    dev = torch.device("cuda:0")
    buf = torch.zeros(16, dtype=torch.complex128, device=dev)
    with pytest.raises(api.ScadynError) as e:
        # 1024 x 1024 outputs exceed the fixed scratch
        api.T_assemble_noalloc(buf.data_ptr(), 1, 1024, buf.data_ptr(), 1024, buf.data_ptr(), 0)
    assert e.value.code == api.SCD_BAD_ARG
