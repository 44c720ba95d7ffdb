"""Output stage: post2d's mid-yz plane file (output.f90:179-432), the
timestep.txt record (main.f90:243-256) and the neighbour-restricted ipot
(interface.f90:225-277)."""
import os

import numpy as np
import pytest

from oracle.oracle import Oracle
from icls_gpu import init_drops, initial_velocity, make_config, static_drop
from icls_gpu.output import append_timestep, fortran_e, fortran_es, post2d


def test_fortran_edit_descriptors():
    assert fortran_e(0.0) == "  0.0000000E+00"
    assert fortran_e(1.0) == "  0.1000000E+01"
    assert fortran_e(-0.015625) == " -0.1562500E-01"
    assert fortran_e(123456.75) == "  0.1234568E+06"
    assert fortran_e(9.99999999) == "  0.1000000E+02"
    assert fortran_es(1.0) == "  1.00000000E+00"
    assert fortran_es(-2.5e-7) == " -2.50000000E-07"


def _oracle_after(steps=2, n=16):
    wl = static_drop(n, steps=steps)
    o = Oracle(wl.cfg)
    o.setup(init_drops(wl.cfg, wl.centres, wl.radii), *initial_velocity(wl.cfg, 0.0))
    for s in range(1, steps + 1):
        o.step(s, 0)
    return wl.cfg, o


def test_plane_matches_field():
    cfg, o = _oracle_after()
    for name, l in (("u", 1), ("pnew", 1), ("lvset", 1), ("rho_u", 1)):
        a = o.download(name, l)
        lo, _ = o.bounds(name)
        for i in (lo[0], cfg.itot // 2, lo[0] + a.shape[0] - 1):
            assert np.array_equal(o.download_plane_x(name, i, l), a[i - lo[0]]), (name, i)


def test_post2d_file(tmp_path):
    cfg, o = _oracle_after()
    path = post2d(o, 2, str(tmp_path))
    assert os.path.basename(path) == "yz_mid0000002.dat"
    lines = open(path).read().splitlines()
    assert lines[0].startswith(' VARIABLES = "y","z","u","v","w","p","s","indie","fixhv"')
    assert len(lines) == 2 + cfg.jtot * cfg.ktot
    rows = np.array([[float(line[15 * c:15 * (c + 1)]) for c in range(9)] for line in lines[2:]])
    u, v, w, p = (o.download(k) for k in ("u", "v", "w", "pnew"))
    ls = o.download("lvset")
    i = cfg.itot // 2
    k, j = 3, 5                                   # row (k-1)*jtot + (j-1)
    r = rows[(k - 1) * cfg.jtot + (j - 1)]
    want = [(j - 0.5) / cfg.jtot, (k - 0.5) / cfg.ktot, 0.5 * (u[i, j, k] + u[i - 1, j, k]),
            0.5 * (v[i, j, k] + v[i, j - 1, k]), 0.5 * (w[i, j, k] + w[i, j, k - 1]), p[i, j, k],
            ls[i + 2, j + 2, k + 2], o.download("jiemian")[i, j, k], 0.0]
    assert np.allclose(r, want, rtol=1e-6, atol=1e-12)


def test_timestep_record(tmp_path):
    cfg = make_config(itot=32, jtot=32, ktot=32, lmax=2, inflate_step=2)
    o = Oracle(cfg)
    o.setup(init_drops(cfg, [(0.3, 0.5, 0.5), (0.7, 0.5, 0.5)], [0.15, 0.15]), *initial_velocity(cfg, 0.0))
    for s in (1, 2):
        o.step(s, 0)
    rec = o.timestep_record(2)
    v, v0 = o.volumes()
    sc = o.scalars()
    assert rec[0] == 2 and rec[1] == sc["time"] and rec[2] == sc["dt"]
    assert rec[3] == sum(1.0 - v / v0)
    # two spheres of radius 0.15 centred 0.4 apart: interfaces 0.1 apart
    assert abs(rec[4] * (1 / 32) - 0.1) < 2.5 / 32
    assert rec[4] == o.ipot()[0, 1] * 32
    assert rec[5] == sc["maxchk_glb"]
    f = tmp_path / "timestep.txt"
    append_timestep(str(f), rec)
    append_timestep(str(f), rec)
    lines = f.read_text().splitlines()
    assert len(lines) == 2 and len(lines[0]) == 96
    assert np.allclose([float(lines[0][16 * c:16 * (c + 1)]) for c in range(6)], rec, rtol=1e-8)


@pytest.mark.gpu
def test_gpu_plane_and_record_parity():
    from icls_gpu import Solver
    cfg = make_config(itot=48, jtot=48, ktot=48, lmax=3, inflate_step=2)
    ls = init_drops(cfg, [(0.25, 0.5, 0.5), (0.6, 0.5, 0.5), (0.5, 0.2, 0.8)], [0.12, 0.12, 0.1])
    sims = []
    for s in (Oracle(cfg), Solver(cfg)):
        s.setup(ls, *initial_velocity(cfg, 0.0))
        for i in (1, 2):
            s.step(i, 0)
        sims.append(s)
    o, g = sims
    for name in ("u", "pnew", "lvset", "jiemian"):
        a = g.download(name)
        lo, _ = g.bounds(name)
        assert np.array_equal(g.download_plane_x(name, 24), a[24 - lo[0]]), name
    ro, rg = o.timestep_record(2), g.timestep_record(2)
    assert np.array_equal(ro[:3], rg[:3])
    assert abs(ro[3] - rg[3]) <= 1e-12 and abs(ro[4] - rg[4]) <= 1e-12 and abs(ro[5] - rg[5]) <= 1e-12


@pytest.mark.gpu
def test_gpu_ipot_many_drops_matches_oracle():
    """With 12 drops most pairs are far apart: the GPU sweeps only pairs
    whose written regions meet, the others keep the reference's 1e3."""
    from icls_gpu import Solver, seeded_drops
    cfg = make_config(itot=64, jtot=64, ktot=64, lmax=12)
    centres, radii = seeded_drops(cfg, 12, seed=5, rmin=0.06, rmax=0.09)
    ls = init_drops(cfg, centres, radii)
    o, g = Oracle(cfg), Solver(cfg)
    uvw = initial_velocity(cfg, 0.0)
    for s in (o, g):
        s.setup(ls, *uvw)
        s.step(1, 0)      # tube construction narrows each drop's region
    do, dg = o.ipot(), g.ipot()
    assert np.array_equal(do, dg)
    assert np.any(do == 1e3) and np.any((do > 0) & (do < 1e3))
