"""CPU oracle pinned to known answers (no GPU needed).

The reference ships no tests or fixtures and cannot be built here (no
Fortran compiler, MPI or LAPACK), so the oracle is checked against answers
that follow from the reference's own definitions:
  * VFFTPACK's documented transform (fft.f:1123-1142, 403-452);
  * the least-squares pseudo-inverse of init_matrix (init.f90:1587-1723);
  * sphere curvature -2/R of get_curvature (interface.f90:20-119);
  * the Poisson eigen-solve of solver2d (solver.f90:68-196, initsolver.f90);
  * exactness of HOUC5/WENO5 on linear data (hyperPDE.f90:397-800);
  * divergence below the chkdiv limit after correc (chkdiv.f90:60);
  * a frozen regression record of a 16^3 static drop.
"""
import json
import os

import numpy as np
import pytest

from conftest import rel_l2

from oracle.oracle import Oracle, set_threads, vrfftb, vrfftf
from icls_gpu import (HOUC5, WENO5, field_shape, init_drops, initial_velocity, make_config,
                      rising_bubble, static_drop)

HERE = os.path.dirname(os.path.abspath(__file__))
set_threads(min(8, os.cpu_count() or 1))


def test_fft_matches_vfftpack_definition():
    g = np.load(os.path.join(HERE, "golden", "fft_vfftpack.npz"))
    for n in (8, 16, 64, 256):
        x, f = g["x%d" % n], g["f%d" % n]
        out = vrfftf(x)
        assert np.max(np.abs(out - f)) < 1e-12 * max(1.0, np.max(np.abs(f)))
        back = vrfftb(out)
        assert np.max(np.abs(back - x)) < 1e-13


def test_fft_matches_numpy_rfft_mapping():
    rng = np.random.default_rng(7)
    for n in (4, 32, 128):
        x = rng.standard_normal((5, n))
        F = np.fft.rfft(x, axis=1) / np.sqrt(n)
        ref = np.zeros_like(x)
        ref[:, 0] = F[:, 0].real
        for k in range(1, n // 2):
            ref[:, 2 * k - 1] = F[:, k].real
            ref[:, 2 * k] = F[:, k].imag
        ref[:, n - 1] = F[:, n // 2].real
        assert np.allclose(vrfftf(x), ref, atol=1e-13, rtol=0)


def test_pseudo_inverse_is_left_inverse():
    cfg = make_config(itot=16, jtot=16, ktot=16)
    o = Oracle(cfg)
    P = o.pseudo_inv()
    h = 1.0 / 16
    rows = []
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                a2, a3, a4 = h * dx, h * dy, h * dz
                rows.append([1, a2, a3, a4, .5 * a2 * a2, .5 * a3 * a3, .5 * a4 * a4, a2 * a3, a2 * a4, a3 * a4])
    A = np.array(rows)
    assert np.allclose(P @ A, np.eye(10), atol=1e-9)
    # gradient row is the central difference weight dist/(18 h)
    assert np.allclose(P[1], A[:, 1] / (18 * h * h), rtol=1e-12, atol=1e-9)


@pytest.mark.parametrize("R_cells", [8.0, 14.0])
def test_sphere_curvature_known_answer(R_cells):
    n = 48
    cfg = make_config(itot=n, jtot=n, ktot=n, lmax=1)
    o = Oracle(cfg)
    R = R_cells / n
    ls = init_drops(cfg, [(0.5, 0.5, 0.5)], [R])
    o.setup(ls)
    o.get_curvature(1)
    kappa = o.interior("curv")
    phi = o.interior("lvset")
    shell = np.abs(phi) < 0.5 / n
    k = kappa[shell]
    assert k.size > 100
    err = np.abs(np.median(k) - (-2.0 / R)) / (2.0 / R)
    assert err < 0.03


def test_poisson_manufactured_solution():
    n, nz = 16, 12
    cfg = make_config(itot=n, jtot=n, ktot=nz, lmax=1)
    o = Oracle(cfg)
    o.setup(init_drops(cfg, [(0.5, 0.5, 0.5)], [0.2]))
    rng = np.random.default_rng(3)
    pe = rng.standard_normal((n, n, nz))
    dxi, dzi = n / cfg.lx, nz / cfg.lz
    # 7-point Laplacian, periodic x,y, Neumann z (initsolver.f90:36-49)
    pz = np.concatenate([pe[:, :, :1], pe, pe[:, :, -1:]], axis=2)
    lap = (np.roll(pe, 1, 0) - 2 * pe + np.roll(pe, -1, 0)) * dxi ** 2 + \
          (np.roll(pe, 1, 1) - 2 * pe + np.roll(pe, -1, 1)) * dxi ** 2 + \
          (pz[:, :, 2:] - 2 * pe + pz[:, :, :-2]) * dzi ** 2
    full = np.zeros(field_shape(cfg, "p"), order="F")
    full[1:-1, 1:-1, 1:-1] = lap
    o.upload("p", full)
    o.solver2d()
    sol = o.interior("p")
    d = (sol - sol.mean()) - (pe - pe.mean())
    assert np.max(np.abs(d)) < 1e-10 * np.max(np.abs(pe))


@pytest.mark.parametrize("scheme", [HOUC5, WENO5])
def test_advection_exact_on_linear_field(scheme):
    n = 32
    cfg = make_config(itot=8, jtot=8, ktot=n, lmax=1, ls_adv_space=scheme, timestep=1e-3)
    o = Oracle(cfg)
    dz = 1.0 / n
    k = np.arange(-2, n + 4)
    zc = (k - 0.5) * dz
    a = 0.01
    ls = np.broadcast_to((a * (zc - 0.5))[None, None, :], field_shape(cfg, "lvset")).copy(order="F")
    w0 = 0.3
    w = np.full(field_shape(cfg, "w"), w0, order="F")
    z = np.zeros(field_shape(cfg, "u"), order="F")
    o.setup(ls[..., None], z, z, w)
    o.tube_construction(1)
    o.ls_advection(1)
    phi = o.download("lvset")
    exp = ls - cfg.timestep * w0 * a
    inner = slice(2 + 12, 2 + n - 11)
    assert np.max(np.abs(phi[2:10, 2:10, inner] - exp[2:10, 2:10, inner])) < 1e-15


def test_static_drop_divergence_free_and_conserving():
    wl = static_drop(32, steps=5)
    o = Oracle(wl.cfg)
    o.setup(init_drops(wl.cfg, wl.centres, wl.radii), *initial_velocity(wl.cfg, 0.0))
    v0 = o.volumes()[1][0]
    for s in range(1, 6):
        o.step(s, 0)
    tot, mx, ijk, rc = o.chkdiv(5, raise_on_error=False)
    assert rc == 0 and mx < 1e-12
    assert abs(o.volumes()[0][0] - v0) / v0 < 1e-4


def test_disp_diagnostics_known_answers():
    """disp_cg / disp_speed (write_vtk.f90:438-566): a drop centred in the box
    has its centroid at the centre and no velocity at rest; a rising bubble
    (gravity along -z, lighter than its surroundings) moves up."""
    wl = static_drop(32, steps=1)
    ls = init_drops(wl.cfg, wl.centres, wl.radii, wl.all_images)
    o = Oracle(wl.cfg)
    o.setup(ls, *initial_velocity(wl.cfg, 0.0))
    cg, vel = o.disp(1)
    assert np.max(np.abs(cg - 0.5)) <= 1e-12
    assert np.max(np.abs(vel)) == 0.0
    wb = rising_bubble(32, steps=3)
    lb = init_drops(wb.cfg, wb.centres, wb.radii, wb.all_images)
    b = Oracle(wb.cfg)
    b.setup(lb, *initial_velocity(wb.cfg, 0.0))
    for s in range(1, 4):
        b.step(s, 0)
    cg, vel = b.disp(1)
    assert abs(cg[2] - 0.5) <= 1e-3 and vel[2] > 0.0 and abs(vel[0]) < 1e-3 * vel[2]


def test_oracle_regression_record():
    with open(os.path.join(HERE, "golden", "oracle_static16.json")) as f:
        rec = json.load(f)
    set_threads(1)
    try:
        wl = static_drop(16, steps=3)
        o = Oracle(wl.cfg)
        o.setup(init_drops(wl.cfg, wl.centres, wl.radii), *initial_velocity(wl.cfg, 0.0))
        for s in range(1, 4):
            o.step(s, 0)
        for name in ("lvset", "u", "v", "w", "pnew"):
            a = o.download(name)
            assert abs(np.linalg.norm(a.ravel()) - rec[name + "_l2"]) <= 1e-12 * max(1.0, rec[name + "_l2"])
            assert abs(a[8, 8, 8] - rec[name + "_probe"]) <= 1e-12 * max(1e-12, abs(rec[name + "_probe"])) + 1e-20
        assert abs(o.volumes()[0][0] - rec["volume"]) < 1e-14
    finally:
        set_threads(min(8, os.cpu_count() or 1))


def test_error_paths():
    from icls_gpu import IclsError
    with pytest.raises(IclsError):
        Oracle(make_config(itot=2, jtot=16, ktot=16))
    o = Oracle(make_config(itot=16, jtot=16, ktot=16))
    with pytest.raises(IclsError):
        o.ls_main(1)  # before init_program -> E_STATE
    # a non-solenoidal field trips chkdiv's abort (chkdiv.f90:60-87)
    o.setup(init_drops(o.cfg, [(0.5, 0.5, 0.5)], [0.25]))
    u = np.random.default_rng(0).standard_normal(field_shape(o.cfg, "u"))
    o.upload("u", np.asfortranarray(u))
    with pytest.raises(IclsError) as e:
        o.chkdiv(5)
    assert e.value.code == 4
    # step 0 only reports (chkdiv.f90:63)
    assert o.chkdiv(0)[3] == 0


def _exact_sum(x):
    import ctypes as C
    from oracle.oracle import backend
    lib = backend().lib
    lib.ora_exact_sum.argtypes = [C.POINTER(C.c_double), C.c_longlong]
    lib.ora_exact_sum.restype = C.c_double
    a = np.ascontiguousarray(x, dtype=np.float64)
    return lib.ora_exact_sum(a.ctypes.data_as(C.POINTER(C.c_double)), len(a))


def test_exact_sum_is_correctly_rounded_and_order_free():
    """The volume integral's sum of H: exact, rounded once (ties to even).
    For elements of magnitude above 2^-92 (none is truncated) it equals
    math.fsum, the correctly rounded sum, in every order."""
    import math
    rng = np.random.default_rng(3)
    # a drop's Heaviside field: far field exactly 1, a shell of fractions
    h = np.ones(200_000)
    shell = rng.integers(0, h.size, 4_000)
    h[shell] = rng.uniform(0.0, 1.0, shell.size)
    h[rng.integers(0, h.size, 50)] = -rng.uniform(0, 1e-17, 50)  # H < 0 by rounding
    for x in (h, rng.standard_normal(10_000) * 10.0 ** rng.integers(-20, 1, 10_000)):
        ref = math.fsum(x)
        assert _exact_sum(x) == ref
        assert _exact_sum(x[::-1]) == ref
        assert _exact_sum(rng.permutation(x)) == ref
    # ties to even and the sticky bit
    assert _exact_sum([1.0, 2.0 ** -53]) == 1.0
    assert _exact_sum([1.0 + 2.0 ** -52, 2.0 ** -53]) == 1.0 + 2.0 ** -51
    assert _exact_sum([1.0, 2.0 ** -53, 2.0 ** -100]) == 1.0 + 2.0 ** -52
    assert _exact_sum([1e-300, -1e-300, 0.0]) == 0.0
    assert _exact_sum([-0.75, 0.25]) == -0.5
    # a running double sum of the same shell depends on the order; this does not
    run = [0.0, 0.0]
    for t, x in enumerate((h, h[::-1])):
        s = 0.0
        for v in x:
            s += v
        run[t] = s
    assert _exact_sum(h) == _exact_sum(h[::-1])
    assert run[0] != run[1] or run[0] == math.fsum(h)
