"""The learned curvature's tensor-core path (needs a B200).

The MLP's products run on tcgen05 tiles: BF16 operands in shared memory,
FP32 accumulation in tensor memory.  A single 128 x n tile is checked here
against the FP32 product of the same BF16 values (tolerance 1e-5 relative to
the largest |entry|: only the summation order differs)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from icls_gpu.binding import gpu_backend


@pytest.mark.parametrize("n,k", [(16, 16), (128, 32), (64, 128), (128, 128)])
def test_tc_tile_matches_fp32_product(gpu_available, n, k):
    import torch
    g = torch.Generator().manual_seed(n * 1000 + k)
    a = torch.randn(128, k, generator=g).to(torch.bfloat16)
    b = torch.randn(n, k, generator=g).to(torch.bfloat16)
    ref = a.float() @ b.float().T
    da, db = a.cuda(), b.cuda()
    dd = torch.zeros(128, n, dtype=torch.float32, device="cuda")
    fn = gpu_backend().lib.icls_tc_gemm_bf16
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]
    fn.restype = C.c_int
    rc = fn(da.data_ptr(), db.data_ptr(), dd.data_ptr(), n, k, torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    out = dd.cpu()
    err = float((out - ref).abs().max()) / float(ref.abs().max())
    assert err <= 1e-5, err
