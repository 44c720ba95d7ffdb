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


def _expected(u, v, w, dxi, dyi, dzi):
    """Sum, max|div| and the first column-major location, on the host."""
    div = ((w[1:-1, 1:-1, 1:-1] - w[1:-1, 1:-1, :-2]) * dzi + (v[1:-1, 1:-1, 1:-1] - v[1:-1, :-2, 1:-1]) * dyi
           + (u[1:-1, 1:-1, 1:-1] - u[:-2, 1:-1, 1:-1]) * dxi)
    a = np.abs(div).ravel(order="F")
    q = int(np.argmax(a))  # numpy returns the first maximum
    imax, jmax, _ = div.shape
    return div.sum(), a[q], (q % imax + 1, (q // imax) % jmax + 1, q // (imax * jmax) + 1)


def test_chkdiv_noalloc_tie_across_blocks_takes_the_first_cell(gpu_available):
    """Two equal maxima handled by different blocks: the reported location is
    the earlier column-major cell even though a later block holds it.  The
    grid's cell count (310,545) is not a multiple of the grid stride."""
    import torch

    imax, jmax, kmax = 67, 45, 103
    stride = 1184 * 256
    shp = (imax + 2, jmax + 2, kmax + 2)
    u = np.zeros(shp, order="F")
    v = np.zeros(shp, order="F")
    w = np.zeros(shp, order="F")
    qa = 1000 * 256 + 5          # block 1000, first pass
    qb = stride + 3 * 256 + 7    # block 3, second pass; qa < qb
    for q in (qa, qb):
        i, j, k = q % imax + 1, (q // imax) % jmax + 1, q // (imax * jmax) + 1
        assert i < imax
        u[i, j, k] = 0.75
    dxi = dyi = dzi = 64.0
    tot, mx, ijk = _expected(u, v, w, dxi, dyi, dzi)
    dev = [torch.from_numpy(a.ravel(order="F").copy()).to("cuda") for a in (u, v, w)]
    out = torch.full((5,), -1.0, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for _call in range(2):
        out.fill_(-1.0)
        assert chkdiv_noalloc(dev[0].data_ptr(), dev[1].data_ptr(), dev[2].data_ptr(),
                              imax, jmax, kmax, dxi, dyi, dzi, out.data_ptr(), stream) == 0
        torch.cuda.synchronize()
        r = out.cpu().numpy()
        assert r[0] == tot == 0.0
        assert r[1] == mx
        assert (int(r[2]), int(r[3]), int(r[4])) == ijk
        q = (ijk[0] - 1) + imax * ((ijk[1] - 1) + jmax * (ijk[2] - 1))
        assert q == qa


def test_chkdiv_noalloc_near_the_cell_limit(gpu_available):
    """A grid within one grid stride of ICLS_NOALLOC_MAX_CELLS (2^31-1): the
    last pass of the grid-stride loop steps past INT_MAX, which a 32-bit
    index would wrap.  Zero fields with one planted column near the last
    cell; needs about 52 GB of device memory and is skipped without it."""
    import torch

    imax, jmax, kmax = 1023, 1023, 2052
    n = imax * jmax * kmax
    assert 2**31 - 1 - 1184 * 256 < n <= 2**31 - 1
    shp = (imax + 2, jmax + 2, kmax + 2)
    nbytes = 3 * shp[0] * shp[1] * shp[2] * 8
    free, _total = torch.cuda.mem_get_info()
    if free < nbytes + (8 << 30):
        pytest.skip("needs %.1f GB free on the device" % (nbytes / 1e9))
    dev = [torch.zeros(shp[0] * shp[1] * shp[2], dtype=torch.float64, device="cuda") for _ in range(3)]
    try:
        # w(i,j,kmax) = s: div at (i,j,kmax) is s*dzi, the last interior row
        i, j, k = imax - 3, jmax - 1, kmax
        c = i + shp[0] * (j + shp[1] * k)
        dev[2][c] = 0.5
        out = torch.full((5,), -1.0, dtype=torch.float64, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        for _call in range(2):
            out.fill_(-1.0)
            assert chkdiv_noalloc(dev[0].data_ptr(), dev[1].data_ptr(), dev[2].data_ptr(),
                                  imax, jmax, kmax, 8.0, 8.0, 8.0, out.data_ptr(), stream) == 0
            torch.cuda.synchronize()
            r = out.cpu().numpy()
            assert r[0] == 4.0 and r[1] == 4.0
            assert (int(r[2]), int(r[3]), int(r[4])) == (i, j, k)
    finally:
        del dev
        torch.cuda.empty_cache()
