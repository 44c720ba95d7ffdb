"""The divergence check that allocates no device memory (needs a B200).

icls_chkdiv_noalloc serves callers that cannot let the library allocate
device memory: their device memory is claimed by their own pool, or an
allocation failure inside a diagnostic check is not acceptable.  The caller
owns u, v, w and the result buffer; the per-block partial sums live in a
fixed file-scope device array shared by all calls.  This test compares it,
on two calls in a row, with icls_chkdiv of a context holding the same field.
The file sorts last so a stop-at-first-failure run has already run the rest.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from icls_gpu import Solver, field_shape, make_config
from icls_gpu.binding import chkdiv_noalloc


def test_chkdiv_noalloc_matches_context_chkdiv(gpu_available):
    import torch

    cfg = make_config(itot=64, jtot=32, ktot=48, lmax=1)
    shp = field_shape(cfg, "u")
    rng = np.random.default_rng(42)
    fields = [np.asfortranarray(rng.standard_normal(shp)) for _ in range(3)]

    s = Solver(cfg)
    for name, a in zip(("u", "v", "w"), fields):
        s.upload(name, a)
    tot, mx, ijk, rc = s.chkdiv(0, raise_on_error=False)
    assert rc == 0 and mx > 0.0

    dev = [torch.from_numpy(a.ravel(order="F").copy()).to("cuda") for a in fields]
    out = torch.full((5,), -1.0, dtype=torch.float64, device="cuda")
    dxi, dyi, dzi = cfg.itot / cfg.lx, cfg.jtot / cfg.ly, cfg.ktot / cfg.lz
    stream = torch.cuda.current_stream().cuda_stream
    for _call in range(2):
        out.fill_(-1.0)
        rc = chkdiv_noalloc(dev[0].data_ptr(), dev[1].data_ptr(), dev[2].data_ptr(),
                            cfg.itot, cfg.jtot, cfg.ktot, dxi, dyi, dzi, out.data_ptr(), stream)
        assert rc == 0
        torch.cuda.synchronize()
        r = out.cpu().numpy()
        # same partition and combination order as the context path
        assert abs(r[0] - tot) <= 1e-12 * max(1.0, abs(tot), mx)
        assert r[1] == mx
        assert (int(r[2]), int(r[3]), int(r[4])) == tuple(ijk)

    # a grid beyond the stated limit is refused before any launch
    rc = chkdiv_noalloc(dev[0].data_ptr(), dev[1].data_ptr(), dev[2].data_ptr(),
                        2048, 2048, 2048, dxi, dyi, dzi, out.data_ptr(), stream)
    assert rc == 9  # ICLS_E_SIZE
