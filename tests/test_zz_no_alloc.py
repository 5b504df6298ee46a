"""The allocation-free PCG entry point, mlp_pcg_device_noalloc.

It exists for host applications that cannot let the library call cudaMalloc
while they solve, because their device memory is owned by their own allocator
or held to a fixed budget; its vectors live in a static device array of the
library instead. It must return what mlp_pcg_device returns, call after call
(the shared array keeps the previous call's contents), allocate no device
memory while it runs, and refuse systems larger than the array. This file is
collected last so that a run stopping at the first failure has already run
every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_N = 131072
TOL = 1e-10  # relative, as in the PCG parity tests


def _solve(M, entry, A, P, b_dev, x_dev, fp32):
    from ml_prec_b200._capi import Stats, check, lib
    st = Stats()
    fn = getattr(lib(), entry)
    check(fn(A.h, C.c_void_p(b_dev.data_ptr()), P.h, C.c_void_p(x_dev.data_ptr()), 1e-8, 0, int(fp32),
             C.byref(st), None))
    return x_dev.cpu().numpy().copy(), st.niter


@pytest.mark.parametrize("fp32", [False, True])
def test_noalloc_matches_allocating_pcg_twice(fp32):
    import torch
    import ml_prec_b200 as M
    from ml_prec_b200 import fields
    kx, ky, kz = fields.field("layered", 2)
    A, b = M.CSRMatrix.spe(60, 220, 8, kx, ky, kz, c=1.0)  # 105,600 unknowns
    assert A.n <= MAX_N
    P = M.MultiSplitPrec(A, fp32=fp32, q=(0.8,), niter=(5,), max_levels=15, degree_max=2)
    dev = torch.device("cuda", 0)
    b_dev = torch.from_numpy(b).to(dev)
    x_ref, it_ref = _solve(M, "mlp_pcg_device", A, P, b_dev, torch.empty_like(b_dev), fp32)
    outs = [torch.empty_like(b_dev) for _ in range(2)]
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info(0)[0]
    for out in outs:  # two calls in a row share the static scratch
        x, it = _solve(M, "mlp_pcg_device_noalloc", A, P, b_dev, out, fp32)
        assert it == it_ref
        assert np.linalg.norm(x - x_ref) <= TOL * np.linalg.norm(x_ref)
    torch.cuda.synchronize()
    # the device's free memory is unchanged: nothing was allocated on it
    assert torch.cuda.mem_get_info(0)[0] == free_before


def test_noalloc_rejects_systems_beyond_its_array():
    import torch
    import ml_prec_b200 as M
    from ml_prec_b200 import fields
    from ml_prec_b200._capi import Stats, lib
    kx, ky, kz = fields.field("iid", 1)
    A, b = M.CSRMatrix.spe(60, 220, 10, kx, ky, kz, c=1.0)  # 132,000 unknowns
    assert A.n > MAX_N
    P = M.MultiSplitPrec(A, q=(0.8,), niter=(5,), max_levels=15, degree_max=2)
    dev = torch.device("cuda", 0)
    b_dev = torch.from_numpy(b).to(dev)
    x_dev = torch.empty_like(b_dev)
    st = Stats()
    rc = lib().mlp_pcg_device_noalloc(A.h, C.c_void_p(b_dev.data_ptr()), P.h, C.c_void_p(x_dev.data_ptr()),
                                      1e-8, 0, 0, C.byref(st), None)
    assert rc == 9  # MLP_ERR_LIMIT
    assert b"131072" in lib().mlp_last_error()
