"""Checkpoint and restart: loadflds (loadd.f90:28-103) plus the history file
that makes a restart continue the uninterrupted run exactly.

CPU tests drive the oracle's restatement of the same file layout; the GPU
tests drive the CUDA library and cross-read its files with the oracle."""
import os

import numpy as np
import pytest

from oracle.oracle import Oracle
from icls_gpu import IclsError, init_drops, initial_velocity, static_drop

FIELDS = ("u", "v", "w", "pnew", "lvset", "jiemian")


def _workload(n=16):
    wl = static_drop(n, steps=6)
    wl.cfg.inflate_step = 2   # mass corrections fall after the restart point
    return wl


def _start(make, wl):
    s = make(wl.cfg)
    s.setup(init_drops(wl.cfg, wl.centres, wl.radii), *initial_velocity(wl.cfg, 0.0))
    return s


def _run(s, first, last):
    for i in range(first, last + 1):
        s.step(i, 0)


def _state(s):
    out = {k: s.download(k) for k in FIELDS}
    out["duold"] = s.download("duold")
    out["volume"] = s.volumes()[0]
    return out


def _file_layout(path, cfg, nr, time, dt):
    n = cfg.itot * cfg.jtot * cfg.ktot
    raw = np.fromfile(path, dtype="<f8")
    assert raw.size == n * (5 + cfg.lmax) + 3
    assert raw[-3] == time and raw[-2] == nr and raw[-1] == dt
    return raw


def _check_restart(make, tmp_path, wl, exact=True):
    ref = _start(make, wl)
    _run(ref, 1, 6)
    want = _state(ref)

    a = _start(make, wl)
    _run(a, 1, 3)
    path = str(tmp_path / "fld0000003")
    a.write_checkpoint(path, 3)
    sc = a.scalars()
    raw = _file_layout(path, wl.cfg, 3, sc["time"], sc["dt"])
    n = wl.cfg.itot * wl.cfg.jtot * wl.cfg.ktot
    # u(1:imax,1:jmax,1:kmax), i fastest, first in the file; lvset(1) fifth
    assert np.array_equal(raw[:n], a.interior("u").ravel(order="F"))
    assert np.array_equal(raw[4 * n:5 * n], a.interior("lvset").ravel(order="F"))
    assert os.path.exists(path + ".hist")

    b = make(wl.cfg)
    assert b.read_checkpoint(path) == 3
    assert b.scalars()["time"] == sc["time"]
    _run(b, 4, 6)
    got = _state(b)
    for k, v in want.items():
        if exact:
            assert np.array_equal(got[k], v), k
        else:
            assert np.max(np.abs(got[k] - v)) <= 1e-13 * max(1.0, np.max(np.abs(v))), k
    return path


def test_oracle_restart_continues_exactly(tmp_path):
    _check_restart(Oracle, tmp_path, _workload())


def test_oracle_restart_without_history_differs(tmp_path):
    """Without the history file the restart is loadflds + init_program as in
    the reference (init.f90:22-117): the AB2 history restarts from the
    current state, so the continuation departs from the uninterrupted run."""
    wl = _workload()
    ref = _start(Oracle, wl)
    _run(ref, 1, 6)
    a = _start(Oracle, wl)
    _run(a, 1, 3)
    path = str(tmp_path / "fld0000003")
    a.write_checkpoint(path, 3, history=False)
    assert not os.path.exists(path + ".hist")
    b = Oracle(wl.cfg)
    assert b.read_checkpoint(path) == 3
    _run(b, 4, 6)
    assert not np.array_equal(b.download("u"), ref.download("u"))


def test_oracle_checkpoint_errors(tmp_path):
    wl = _workload()
    o = Oracle(wl.cfg)
    with pytest.raises(IclsError) as e:
        o.read_checkpoint(str(tmp_path / "missing"))
    assert e.value.code == 10
    a = _start(Oracle, wl)
    path = str(tmp_path / "fld0000000")
    a.write_checkpoint(path, 0)
    with open(path, "r+b") as f:           # truncate the field file
        f.truncate(1000)
    with pytest.raises(IclsError) as e:
        Oracle(wl.cfg).read_checkpoint(path)
    assert e.value.code == 10
    a.write_checkpoint(path, 0)
    other = static_drop(24, steps=1)       # history of another grid
    with pytest.raises(IclsError):
        Oracle(other.cfg).read_checkpoint(path)


@pytest.mark.gpu
def test_gpu_restart_continues_exactly(tmp_path):
    from icls_gpu import Solver
    _check_restart(Solver, tmp_path, _workload(32))


@pytest.mark.gpu
def test_gpu_checkpoint_reads_in_oracle(tmp_path):
    """Files written by the CUDA library load into the oracle unchanged, and
    both continue to the same state within the FP64 parity bound."""
    from icls_gpu import Solver
    wl = _workload(32)
    g = _start(Solver, wl)
    _run(g, 1, 3)
    path = str(tmp_path / "fld0000003")
    g.write_checkpoint(path, 3)
    o = Oracle(wl.cfg)
    assert o.read_checkpoint(path) == 3
    for k in ("u", "v", "w", "pnew"):
        assert np.array_equal(o.interior(k), g.interior(k)), k
    for k in ("lvset", "duold", "pold", "p_x"):      # whole arrays from path.hist
        assert np.array_equal(o.download(k), g.download(k)), k
    # jiemian is recomputed from the level set by init_program on both sides
    assert np.max(np.abs(o.interior("jiemian") - g.interior("jiemian"))) <= 1e-15
    _run(g, 4, 5)
    _run(o, 4, 5)
    for k in ("u", "v", "w", "lvset"):
        a, b = g.download(k), o.download(k)
        assert np.max(np.abs(a - b)) <= 1e-12 * max(1.0, np.max(np.abs(b))), k


@pytest.mark.gpu
def test_gpu_restart_fp32_form_continues_exactly(tmp_path):
    """The FP32 form stores its fields as floats; the checkpoint holds them as
    doubles (exact both ways), so its restart is exact too."""
    from icls_gpu import FP32, Solver
    from icls_gpu.config import IclsConfig
    wl = _workload(32)
    cf = IclsConfig.from_buffer_copy(wl.cfg)
    cf.precision = FP32
    wl.cfg = cf
    _check_restart(Solver, tmp_path, wl)
