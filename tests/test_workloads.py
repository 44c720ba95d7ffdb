"""Synthetic inputs of the configurations (CPU only).

The combined configuration's initial velocity is a seeded random field that
must be divergence-free on the staggered grid (to roundoff), vanish across
the z walls and have the requested rms; its drops keep the seeded gap."""
import math

import numpy as np

from icls_gpu import combined, solenoidal_velocity, workload_velocity


def _divergence(cfg, u, v, w):
    dx, dy, dz = cfg.lx / cfg.itot, cfg.ly / cfg.jtot, cfg.lz / cfg.ktot
    s = np.s_[1:-1, 1:-1, 1:-1]
    return ((u[s] - u[:-2, 1:-1, 1:-1]) / dx + (v[s] - v[1:-1, :-2, 1:-1]) / dy +
            (w[s] - w[1:-1, 1:-1, :-2]) / dz)


def test_solenoidal_velocity_is_discretely_divergence_free():
    wl = combined(n=48, ndrop=4, seed=3, rmin=0.06, rmax=0.1)
    u, v, w = solenoidal_velocity(wl.cfg, 11, rms=0.2, kmax=8)
    n = wl.cfg.itot
    scale = 0.2 * n  # velocity / dx
    assert np.max(np.abs(_divergence(wl.cfg, u, v, w))) <= 1e-12 * scale
    s = np.s_[1:-1, 1:-1, 1:-1]
    rms = math.sqrt((np.mean(u[s] ** 2) + np.mean(v[s] ** 2) + np.mean(w[s] ** 2)) / 3.0)
    assert abs(rms - 0.2) <= 1e-12
    assert np.max(np.abs(w[1:-1, 1:-1, n])) <= 1e-14  # top wall face
    assert np.max(np.abs(w[1:-1, 1:-1, 0])) == 0.0     # bottom wall face


def test_solenoidal_velocity_is_seeded():
    wl = combined(n=32, ndrop=2, seed=5, rmin=0.08, rmax=0.1)
    a = solenoidal_velocity(wl.cfg, 7)
    b = solenoidal_velocity(wl.cfg, 7)
    c = solenoidal_velocity(wl.cfg, 8)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    assert not np.array_equal(a[0], c[0])


def test_combined_configuration():
    wl = combined(n=96, ndrop=12, seed=2024, rmin=0.07, rmax=0.1)
    cfg = wl.cfg
    assert (cfg.itot, cfg.jtot, cfg.ktot, cfg.lmax) == (96, 96, 96, 12)
    assert cfg.We == 5.0 and cfg.rho2 / cfg.rho1 == 10.0 and cfg.miu2 / cfg.miu1 == 10.0
    gap = 4.0 / 96
    for a in range(12):
        for b in range(a + 1, 12):
            d = np.array(wl.centres[a]) - np.array(wl.centres[b])
            d[:2] -= np.round(d[:2])
            assert np.linalg.norm(d) >= wl.radii[a] + wl.radii[b] + gap - 1e-12
    u, v, w = workload_velocity(wl)
    assert np.max(np.abs(_divergence(cfg, u, v, w))) <= 1e-12 * 0.2 * 96


def test_seeded_layouts_are_fixed():
    """The benchmark's drop layout is a function of its seed alone: the first
    and last drops of multi_drop(256, 48) as seeded (draws x, y, z per drop)."""
    from icls_gpu import multi_drop
    w = multi_drop(256, 48)
    assert np.allclose(w.centres[0], (0.21432320123825765, 0.3094520308816917, 0.7599965010723276), rtol=0, atol=1e-15)
    assert w.radii[0] == 0.05027494013943845
    assert np.allclose(w.centres[-1], (0.033898820090026094, 0.5818307796575592, 0.630942175696876), rtol=0, atol=1e-15)
    assert w.radii[-1] == 0.041416709589228044


def test_y_walls_seeding_keeps_clear():
    """With walls in y, every drop keeps one radius plus the 4-cell gap from
    y = 0 and y = ly, as from the z walls."""
    from icls_gpu import BCY_WALLS, multi_drop
    w = multi_drop(128, 12, rmin=0.06, rmax=0.12, y_walls=True)
    assert w.cfg.bc_y == BCY_WALLS and w.cfg.constPoi == 0
    gap = 4.0 / 128
    for c, r in zip(w.centres, w.radii):
        assert c[1] - r >= gap - 1e-15 and 1.0 - c[1] - r >= gap - 1e-15
