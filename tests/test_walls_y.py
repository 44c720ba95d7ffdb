"""BC_in_y = 'Walls', 'InOut', 'OutOut': the y boundaries of bounduvw and
boundp (bound.f90:81-282), initsolver's tridiagonal-in-y branch
(initsolver.f90:85-156) and solver2d_cos (solver.f90:202-317).

CPU tests pin the oracle: the quarter-wave cosine transforms against their
documented definitions (fft.f:120-124, 270-274) and each other, and the
pressure solve against a manufactured solution of the discrete Poisson
problem with the reference's ghost-cell conditions.  GPU tests compare the
CUDA library with the oracle."""
import numpy as np
import pytest
import scipy.fft

from oracle.oracle import Oracle, vcosqb, vcosqf
from icls_gpu import (BCY_INOUT, BCY_OUTOUT, BCY_PERIODIC, BCY_WALLS, IclsError, NS_WENO5,
                      field_shape, inflow_profile, init_drops, initial_velocity, make_config, static_drop)

BCS = (BCY_WALLS, BCY_INOUT, BCY_OUTOUT)


@pytest.mark.parametrize("n", [6, 16, 48, 64])
def test_cosq_definitions_and_round_trip(n):
    x = np.random.default_rng(n).standard_normal((3, n))
    # VCOSQB: sum_k 4 x(k) cos((2k-1)(i-1) pi/2n)/sqrt(4n) = DCT-II/sqrt(n)
    assert np.allclose(vcosqb(x), scipy.fft.dct(x, type=2, axis=1) / np.sqrt(n), rtol=0, atol=1e-13)
    # VCOSQF: (x(1) + sum_{k>=2} 2 x(k) cos((2i-1)(k-1) pi/2n))/sqrt(4n) = DCT-III/(2 sqrt(n))
    assert np.allclose(vcosqf(x), scipy.fft.dct(x, type=3, axis=1) / (2 * np.sqrt(n)), rtol=0, atol=1e-13)
    # fft.f:129-131: VCOSQB is the normalised inverse of VCOSQF
    assert np.max(np.abs(vcosqf(vcosqb(x)) - x)) < 1e-13
    assert np.max(np.abs(vcosqb(vcosqf(x)) - x)) < 1e-13


def _laplacian(cfg, bc, q):
    """The 7-point Laplacian of q(1:imax,1:jmax,1:kmax) with the ghost cells
    solver2d_cos inverts: periodic x, zero Neumann z (the cosine modes), and
    in y the end conditions of initsolver.f90:104-124 (Neumann p0=p1,
    Dirichlet p0=-p1)."""
    dxi, dyi, dzi = cfg.itot / cfg.lx, cfg.jtot / cfg.ly, cfg.ktot / cfg.lz
    g = np.pad(q, 1)
    g[0, 1:-1, 1:-1], g[-1, 1:-1, 1:-1] = q[-1], q[0]
    g[:, :, 0], g[:, :, -1] = g[:, :, 1], g[:, :, -2]
    front = -1.0 if bc == BCY_OUTOUT else 1.0
    back = 1.0 if bc == BCY_WALLS else -1.0
    g[:, 0, :] = front * g[:, 1, :]
    g[:, -1, :] = back * g[:, -2, :]
    c = g[1:-1, 1:-1, 1:-1]
    return (dxi * dxi * (g[2:, 1:-1, 1:-1] - 2 * c + g[:-2, 1:-1, 1:-1])
            + dyi * dyi * (g[1:-1, 2:, 1:-1] - 2 * c + g[1:-1, :-2, 1:-1])
            + dzi * dzi * (g[1:-1, 1:-1, 2:] - 2 * c + g[1:-1, 1:-1, :-2]))


def _walls_config(n=16, bc=BCY_WALLS, **kw):
    return make_config(itot=n, jtot=n + 4, ktot=n, ly=(n + 4) / n, bc_y=bc, **kw)


def _solve(solver, cfg, f):
    shp = field_shape(cfg, "p")
    a = np.zeros(shp, order="F")
    a[1:-1, 1:-1, 1:-1] = f
    solver.upload("p", a)
    solver.solver2d()
    return solver.download("p")[1:-1, 1:-1, 1:-1]


@pytest.mark.parametrize("bc", BCS)
def test_oracle_solver2d_cos_manufactured(bc):
    cfg = _walls_config(bc=bc)
    o = Oracle(cfg)
    o.setup(init_drops(cfg, [(0.5, 0.5, 0.5)], [0.25]))
    q = np.random.default_rng(bc).standard_normal((cfg.itot, cfg.jtot, cfg.ktot))
    if bc == BCY_WALLS:
        q -= q.mean()          # the Neumann problem fixes p up to a constant
    p = _solve(o, cfg, _laplacian(cfg, bc, q))
    if bc == BCY_WALLS:
        p = p - p.mean()
    assert np.max(np.abs(p - q)) < 1e-10 * np.max(np.abs(q))


def test_inflow_profile_mean():
    """inflow_profile (init.f90:418-455): the parabola's mean over the inlet
    plane is v_bulk_desired (with the reference's discrete rounding)."""
    cfg = make_config(itot=48, jtot=16, ktot=48)
    v = inflow_profile(cfg, 1.0)
    assert v.shape == (50, 50)
    assert v[1:17, :].max() == 0 and v[33:, :].max() == 0 and v[:, 10:].max() == 0
    assert abs(v.sum() / (48 * 48) - 1.0) < 0.05


@pytest.mark.parametrize("bc", BCS)
def test_oracle_walls_run(bc):
    """A drop between y walls: divergence-free and finite over 5 steps, the
    wall rows as bound.f90 sets them."""
    cfg = _walls_config(bc=bc, inflate_step=20, reinit_step=1, reinit_iter_max=2)
    cfg.timestep = 1e-4
    o = Oracle(cfg)
    if bc == BCY_INOUT:
        o.set_inflow(inflow_profile(cfg, 0.1))
    ls = init_drops(cfg, [(0.5, 0.5 * cfg.ly, 0.5)], [0.2])
    o.setup(ls, *initial_velocity(cfg, 0.0))
    for s in range(1, 6):
        o.step(s, 0)
    tot, mx, ijk, rc = o.chkdiv(5, raise_on_error=False)
    u, v, w, pn = (o.download(k) for k in ("u", "v", "w", "pnew"))
    for a in (u, v, w, pn):
        assert np.all(np.isfinite(a))
    if bc != BCY_OUTOUT:
        assert rc == 0 and mx < 1e-12
    else:
        # OutOut's front ghost v(i,0,k) = v(i,1,k) + dy/dz (w(i,1,k) - w(i,1,k-1))
        # (bound.f90:152) cancels only the z part of the divergence: cells
        # j = 1 keep du/dx, so the reference's own chkdiv stops such a run
        # (chkdiv.f90:60-87); the cells j >= 2 are divergence-free
        assert rc == 4 and ijk[1] == 1
        dxi, dyi, dzi = cfg.itot / cfg.lx, cfg.jtot / cfg.ly, cfg.ktot / cfg.lz
        div = ((u[1:-1, 1:-1, 1:-1] - u[:-2, 1:-1, 1:-1]) * dxi + (v[1:-1, 1:-1, 1:-1] - v[1:-1, :-2, 1:-1]) * dyi
               + (w[1:-1, 1:-1, 1:-1] - w[1:-1, 1:-1, :-2]) * dzi)
        assert np.max(np.abs(div[:, 1:, :])) < 1e-12
        dudx = (u[1:-1, 1, 1:-1] - u[:-2, 1, 1:-1]) * dxi
        assert np.max(np.abs(div[:, 0, :] - dudx)) < 1e-9 and abs(mx - np.max(np.abs(dudx))) < 1e-9
    if bc == BCY_WALLS:
        assert np.all(v[1:-1, 0, 1:-1] == 0) and np.all(v[1:-1, -2, 1:-1] == 0)
        assert np.array_equal(u[1:-1, 0, 1:-1], -u[1:-1, 1, 1:-1])
        assert np.array_equal(pn[1:-1, 0, 1:-1], pn[1:-1, 1, 1:-1])
    elif bc == BCY_INOUT:
        vin = inflow_profile(cfg, 0.1)
        assert np.array_equal(v[1:-1, 0, 1:-1], vin[1:-1, 1:-1])
        assert np.array_equal(pn[1:-1, -1, 1:-1], -pn[1:-1, -2, 1:-1])
    else:
        assert np.array_equal(pn[1:-1, 0, 1:-1], -pn[1:-1, 1, 1:-1])


def test_ns_conv_weno5_rejected():
    """The reference stops in boundfu when NS_conv='WENO5' (bound.f90:310-322)."""
    with pytest.raises(IclsError) as e:
        Oracle(make_config(itot=16, jtot=16, ktot=16, ns_conv=NS_WENO5))
    assert e.value.code == 8


# ----------------------------------------------------------------- GPU
def _gpu_solver(cfg):
    from icls_gpu import Solver
    return Solver(cfg)


@pytest.mark.gpu
def test_gpu_ns_conv_weno5_rejected():
    with pytest.raises(IclsError) as e:
        _gpu_solver(make_config(itot=16, jtot=16, ktot=16, ns_conv=NS_WENO5))
    assert e.value.code == 8


@pytest.mark.gpu
@pytest.mark.parametrize("bc", BCS)
@pytest.mark.parametrize("n", [16, 48, 64])
def test_gpu_solver2d_cos_parity(bc, n):
    cfg = _walls_config(n=n, bc=bc)
    o, g = Oracle(cfg), _gpu_solver(cfg)
    ls = init_drops(cfg, [(0.5, 0.5 * cfg.ly, 0.5)], [0.25])
    o.setup(ls)
    g.setup(ls)
    f = np.random.default_rng(n + bc).standard_normal((cfg.itot, cfg.jtot, cfg.ktot))
    if bc == BCY_WALLS:
        f -= f.mean()
    a, b = _solve(g, cfg, f), _solve(o, cfg, f)
    if bc == BCY_WALLS:
        a, b = a - a.mean(), b - b.mean()
    assert np.max(np.abs(a - b)) <= 1e-11 * np.max(np.abs(b))
    # the y-wall halos of boundp (bound.f90:207-282) on the GPU's p
    g.boundp("p")
    pg = g.download("p")
    front = -1.0 if bc == BCY_OUTOUT else 1.0
    back = 1.0 if bc == BCY_WALLS else -1.0
    assert np.array_equal(pg[1:-1, 0, 1:-1], front * pg[1:-1, 1, 1:-1])
    assert np.array_equal(pg[1:-1, -1, 1:-1], back * pg[1:-1, -2, 1:-1])


@pytest.mark.gpu
@pytest.mark.parametrize("bc", BCS)
@pytest.mark.parametrize("yc", [0.5, 0.18])
def test_gpu_walls_multistep_parity(bc, yc):
    """8 steps with mass corrections every 4; at yc = 0.18 the drop's band
    reaches the y = 0 boundary, so the inflation velocities take the wall
    rows of boundp(dheav) and bounduvw(u_l,v_l,w_l) (levelset.f90:466-478)."""
    cfg = _walls_config(n=32, bc=bc, inflate_step=4, reinit_step=1, reinit_iter_max=2)
    cfg.timestep = 1e-4
    ls = init_drops(cfg, [(0.5, yc * cfg.ly, 0.5)], [0.2])
    uvw = initial_velocity(cfg, 0.0)
    sims = []
    for s in (Oracle(cfg), _gpu_solver(cfg)):
        if bc == BCY_INOUT:
            s.set_inflow(inflow_profile(cfg, 0.1))
        s.setup(ls, *uvw)
        for i in range(1, 9):
            s.step(i, 0)
        sims.append(s)
    o, g = sims
    for k in ("u", "v", "w", "pnew", "lvset", "dudt", "dvdt", "dwdt", "vcc"):
        a, b = g.download(k), o.download(k)
        assert np.max(np.abs(a - b)) <= 1e-10 * max(1.0, np.max(np.abs(b))), k
    # wall rows are set exactly as bound.f90 sets them
    v = g.download("v")
    if bc == BCY_WALLS:
        assert np.all(v[1:-1, 0, 1:-1] == 0) and np.all(v[1:-1, -2, 1:-1] == 0)


@pytest.mark.gpu
def test_gpu_walls_fp32_form_tracks_fp64():
    """The FP32 form between y walls: 8 steps stay within the form's
    tolerances of the FP64 path (volume to 1e-6, velocities to 1e-4 of their
    scale) with the wall rows exact."""
    from icls_gpu import FP32
    from icls_gpu.config import IclsConfig
    cfg = _walls_config(n=32, bc=BCY_WALLS, inflate_step=4, reinit_step=1, reinit_iter_max=2)
    cfg.timestep = 1e-4
    cf = IclsConfig.from_buffer_copy(cfg)
    cf.precision = FP32
    ls = init_drops(cfg, [(0.5, 0.5 * cfg.ly, 0.5)], [0.2])
    uvw = initial_velocity(cfg, 0.0)
    sims = []
    for c in (cfg, cf):
        s = _gpu_solver(c)
        s.setup(ls, *uvw)
        for i in range(1, 9):
            s.step(i, 0)
        sims.append(s)
    p64, p32 = sims
    v0, v1 = p64.volumes()[0][0], p32.volumes()[0][0]
    assert abs(v1 - v0) / v0 <= 1e-6
    for k in ("u", "v", "w"):
        a, b = p32.download(k), p64.download(k)
        assert np.max(np.abs(a - b)) <= 1e-4 * max(1e-3, np.max(np.abs(b))), k
    v = p32.download("v")
    assert np.all(v[1:-1, 0, 1:-1] == 0) and np.all(v[1:-1, -2, 1:-1] == 0)
