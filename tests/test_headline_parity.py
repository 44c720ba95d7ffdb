"""Plain FP64 CUDA path vs the CPU oracle at the measured sizes (needs a B200).

The throughput workload itself, 256^3 with 48 seeded drops, and the rising
bubble at its stated 128 x 128 x 256 grid, each run side by side with the
oracle from the same seeded state.  At 256^3 the oracle takes tens of
seconds per step on the host cores, so the run is 4 steps long; the
cadences are shortened so that every branch of ls_main runs with all 48
drops batched in the same launches:

* reinit_step = 2: the WENO5 reinitialisation (levelset.f90:592-882) runs at
  steps 2 and 4;
* inflate_step = 2 with a trigger of 1e-12 (icls_config.mass_threshold, in
  place of the reference's fixed 1e-5, which 4 steps of drift do not reach):
  the mass correction (levelset.f90:377-582) inflates every drop at steps 2
  and 4, and the test checks that each drop's drift passes the trigger.

The parity bar is relative L2 <= 1e-10 on every drop's phi, u, v, w and p.
"""
import os

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

from icls_gpu import Solver
from icls_gpu.config import init_drops, init_drops_boxed, multi_drop, rising_bubble, workload_velocity
from oracle.oracle import Oracle, set_threads

set_threads(max(1, os.cpu_count() or 1))

TOL = 1e-10


def _pair(wl, ls):
    u, v, w = workload_velocity(wl)
    g, o = Solver(wl.cfg), Oracle(wl.cfg)
    for s in (g, o):
        s.setup(ls, u, v, w)
    return g, o


def _assert_fields(g, o, lmax):
    errs = {}
    for l in range(1, lmax + 1):
        errs["lvset%d" % l] = rel_l2(g.download("lvset", l), o.download("lvset", l))
    for name in ("u", "v", "w", "pnew"):
        errs[name] = rel_l2(g.download(name), o.download(name))
    bad = {k: e for k, e in errs.items() if not e <= TOL}
    assert not bad, bad
    return errs


def test_multi_drop_256_48_parity():
    wl = multi_drop(256, 48, seed=2024, steps=4)
    cfg = wl.cfg
    cfg.reinit_step = 2
    cfg.inflate_step = 2
    cfg.mass_threshold = 1e-12
    # the signed distance is capped at 12 cells; the first tube_construction
    # clips at 6 (levelset.f90:107-119), so this equals the full-grid input
    ls = init_drops_boxed(cfg, wl.centres, wl.radii)
    g, o = _pair(wl, ls)
    del ls
    try:
        for istep in range(1, 5):
            if istep % cfg.inflate_step == 0:
                # the trigger of ls_mass_correction, on the volumes the
                # previous step's update_materials left (levelset.f90:382-390)
                v, v0 = o.volumes()
                drift = np.abs(v - v0) / v0
                assert np.all(drift > cfg.mass_threshold), drift.min()
            g.step(istep, 0)
            o.step(istep, 0)
        errs = _assert_fields(g, o, cfg.lmax)
        (vg, v0g), (vo, v0o) = g.volumes(), o.volumes()
        assert np.array_equal(v0g, v0o) or np.max(np.abs(v0g - v0o) / v0o) <= 1e-12
        assert np.max(np.abs(vg - vo) / vo) <= 1e-11
        print("256^3 x 48, 4 steps: worst phi %.2e, u %.2e, v %.2e, w %.2e, p %.2e" % (
            max(e for k, e in errs.items() if k.startswith("lvset")), errs["u"], errs["v"], errs["w"],
            errs["pnew"]))
    finally:
        g.close()
        o.close()


def test_rising_bubble_128x256_parity():
    """The rising bubble at its stated grid (128 x 128 x 256, reinitialisation
    and mass-correction check every step, buoyancy along -z) for 14 steps,
    then its reported diagnostics: centroid and rise velocity (disp_cg,
    disp_speed, write_vtk.f90:438-566)."""
    wl = rising_bubble(128, steps=14)
    ls = init_drops(wl.cfg, wl.centres, wl.radii, wl.all_images)
    g, o = _pair(wl, ls)
    try:
        for istep in range(1, 15):
            g.step(istep, 0)
            o.step(istep, 0)
        _assert_fields(g, o, 1)
        assert abs(g.volumes()[0][0] - o.volumes()[0][0]) <= 1e-12
        (cg, vel), (cgo, velo) = g.disp(1), o.disp(1)
        assert np.max(np.abs(cg - cgo)) <= 1e-12
        assert np.max(np.abs(vel - velo)) <= 1e-10 * np.max(np.abs(velo))
        assert vel[2] > 0.0
    finally:
        g.close()
        o.close()
