"""The precision form (ICLS_FP32) against the plain FP64 path (needs a B200).

The form stores and computes advection, reinitialisation, momentum,
correction and curvature in FP32, stores the pressures and face jumps that
those stencils read in FP32, and keeps FP64 for the Poisson solve (its
right-hand side and work array), the volume integral and the GFM jump
assembly.  Its errors against the FP64 run
of the same input are reported (printed, run with -s) and bounded here:

  phi      relative L2 <= 1e-5 on the band |phi| <= 4dz around the
           interface; over the whole array <= 2e-2 (reported apart: cells on
           the reinitialisation threshold |phi| = NB + dz, 7dz from the
           interface, switch their right-hand side on or off depending on
           the last bit, which moves them by up to dtau/2 in either form)
  u, v, w  relative L2 <= 1e-3 (the static drop's velocity is the spurious
           current, O(1e-4), so its relative error is the loosest)
  volume   per-drop relative difference <= 1e-6
  curv     relative L2 on the |phi| <= 2dz shell <= 1e-3
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

from icls_gpu import FP32, FP64, Solver, init_drops, initial_velocity, multi_drop, static_drop
from icls_gpu.config import IclsConfig


def with_precision(cfg, prec):
    c = IclsConfig.from_buffer_copy(cfg)
    c.precision = prec
    return c


def run(wl, prec, steps):
    cfg = with_precision(wl.cfg, prec)
    ls = init_drops(cfg, wl.centres, wl.radii, wl.all_images)
    u, v, w = initial_velocity(cfg, wl.shear_v)
    s = Solver(cfg)
    s.setup(ls, u, v, w)
    for istep in range(1, steps + 1):
        s.step(istep, 0)
    return s


def shell_error(a, b, cfg):
    """relative L2 of curv on the |phi| <= 2dz shell of drop 1"""
    phi = b.download("lvset", 1)[2:-2, 2:-2, 2:-2]  # shape C part of shape L
    mask = np.abs(phi) <= 2.0 * cfg.lz / cfg.ktot
    ca, cb = a.download("curv"), b.download("curv")
    return rel_l2(ca[mask], cb[mask])


def phi_errors(a, b, L, cfg):
    """relative L2 on the |phi| <= 4dz band and over the whole array"""
    band, whole = 0.0, 0.0
    dz = cfg.lz / cfg.ktot
    for l in range(1, L + 1):
        pa, pb = a.download("lvset", l), b.download("lvset", l)
        m = np.abs(pb) <= 4.0 * dz
        band = max(band, rel_l2(pa[m], pb[m]))
        whole = max(whole, rel_l2(pa, pb))
    return band, whole


def report(name, errs):
    print("\n%s: " % name + ", ".join("%s %.3e" % kv for kv in errs.items()))


def test_field_round_trip_fp32():
    wl = static_drop(32, steps=1)
    cfg = with_precision(wl.cfg, FP32)
    s = Solver(cfg)
    u, _, _ = initial_velocity(cfg, 0.0)
    rng = np.random.default_rng(3)
    a = np.asfortranarray(rng.standard_normal(u.shape))
    s.upload("u", a)
    b = s.download("u")
    assert np.array_equal(b, a.astype(np.float32).astype(np.float64))
    s.upload("pnew", a)  # the pressures are stored in the field type too
    assert np.array_equal(s.download("pnew"), a.astype(np.float32).astype(np.float64))
    s.upload("p", a)  # the Poisson work array stays FP64 in both forms
    assert np.array_equal(s.download("p"), a)


def test_static_drop_fp32_vs_fp64():
    wl = static_drop(32, steps=20)
    a = run(wl, FP32, 20)
    b = run(wl, FP64, 20)
    errs = {n: rel_l2(a.download(n), b.download(n)) for n in ("u", "v", "w", "pnew")}
    errs["phi_band"], errs["phi_all"] = phi_errors(a, b, 1, wl.cfg)
    va, vb = a.volumes()[0], b.volumes()[0]
    errs["volume"] = float(np.max(np.abs(va - vb) / vb))
    errs["curv"] = shell_error(a, b, wl.cfg)
    report("static drop 32^3, 20 steps, FP32 form vs FP64", errs)
    assert errs["phi_band"] <= 1e-5
    assert errs["phi_all"] <= 2e-2
    for n in ("u", "v", "w"):
        assert errs[n] <= 1e-3, n
    assert errs["volume"] <= 1e-6
    assert errs["curv"] <= 1e-3


def test_multidrop_fp32_vs_fp64():
    wl = multi_drop(n=128, ndrop=4, seed=5, steps=10, rmin=0.06, rmax=0.08, dt=2e-5)
    wl.cfg.reinit_step = 3
    wl.cfg.inflate_step = 4
    a = run(wl, FP32, 10)
    b = run(wl, FP64, 10)
    errs = {n: rel_l2(a.download(n), b.download(n)) for n in ("u", "v", "w", "pnew")}
    errs["phi_band"], errs["phi_all"] = phi_errors(a, b, 4, wl.cfg)
    va, vb = a.volumes()[0], b.volumes()[0]
    errs["volume"] = float(np.max(np.abs(va - vb) / vb))
    report("4 drops 128^3, 10 steps, FP32 form vs FP64", errs)
    assert errs["phi_band"] <= 1e-5
    assert errs["phi_all"] <= 2e-2
    for n in ("u", "v", "w"):
        assert errs[n] <= 1e-3, n
    assert errs["volume"] <= 1e-6
