"""Runtime configuration, field table and initial conditions.

``IclsConfig`` mirrors ``icls_config`` in include/icls_gpu.h, which restates
the compile-time parameters of the reference's src/param.f90 (grid 27-38,
dt 47, materials 58-63, Re/We/iFr 69-77, flags 93-172, level-set settings
199-275) as a runtime struct.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

# scheme selectors (enum values of include/icls_gpu.h)
HOUC5, WENO5 = 0, 1
SPEED_UNFM, SPEED_CURV = 0, 1
FP64, FP32 = 0, 1
CURV_STENCIL, CURV_MLP = 0, 1
BCY_PERIODIC, BCY_WALLS, BCY_INOUT, BCY_OUTOUT = 0, 1, 2, 3
NS_CNTR2, NS_WENO5 = 0, 1

# status codes
OK, E_CONFIG, E_CUDA, E_NAN, E_DIVERGENCE, E_ARG, E_NOMEM, E_STATE, E_UNSUPPORTED, E_SIZE, E_IO, E_TIMEOUT = range(12)
STATUS_NAMES = {
    0: "OK", 1: "E_CONFIG", 2: "E_CUDA", 3: "E_NAN", 4: "E_DIVERGENCE",
    5: "E_ARG", 6: "E_NOMEM", 7: "E_STATE", 8: "E_UNSUPPORTED", 9: "E_SIZE",
    10: "E_IO", 11: "E_TIMEOUT",
}


class IclsConfig(C.Structure):
    _fields_ = [
        ("itot", C.c_int), ("jtot", C.c_int), ("ktot", C.c_int), ("lmax", C.c_int),
        ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double),
        ("timestep", C.c_double),
        ("rho1", C.c_double), ("rho2", C.c_double), ("miu1", C.c_double), ("miu2", C.c_double),
        ("Re", C.c_double), ("We", C.c_double), ("iFr", C.c_double),
        ("g_unit", C.c_double * 3),
        ("v_wall_lower", C.c_double), ("v_wall_upper", C.c_double),
        ("TwoD", C.c_int), ("constPoi", C.c_int), ("solveLS", C.c_int),
        ("ls_adv_space", C.c_int), ("re_initialization", C.c_int),
        ("reinit_step", C.c_int), ("reinit_iter_max", C.c_int),
        ("mass_correction", C.c_int), ("inflate_step", C.c_int),
        ("ispeed_dependence", C.c_int), ("i_space", C.c_int),
        ("ioutchk", C.c_int), ("precision", C.c_int), ("curvature_model", C.c_int),
        ("mlp_fallback_tol", C.c_double),
        ("bc_y", C.c_int), ("ns_conv", C.c_int),
        ("mass_threshold", C.c_double),
        ("mass_gain_one", C.c_int),
    ]

    def as_dict(self):
        d = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            d[name] = list(v) if name == "g_unit" else v
        return d


class IclsScalars(C.Structure):
    _fields_ = [
        ("time", C.c_double), ("dt", C.c_double), ("rho_avr", C.c_double),
        ("v_bulk", C.c_double), ("norm_old", C.c_double), ("maxchk_glb", C.c_double),
        ("reinit_residual", C.c_double), ("reinit_iters", C.c_int), ("last_inflated", C.c_int),
    ]


def inflow_profile(cfg: IclsConfig, v_bulk_desired: float = 1.0) -> np.ndarray:
    """v_inflow(0:i1,0:k1) of inflow_profile (init.f90:418-455), one process:
    a parabola over k = 1..9 and itot/3 < i <= 2 itot/3 whose mean over the
    inlet plane is v_bulk_desired (param.f90:49)."""
    itot, ktot = cfg.itot, cfg.ktot
    dz = cfg.lz / ktot
    v = np.zeros((itot + 2, ktot + 2), order="F")
    i_start, i_end = itot // 3, itot // 3 * 2
    k_start, k_end = 0, 9
    ratio_i = 1.0 * (i_end - i_start) / itot
    ratio_k = 1.0 * (k_end - k_start) / ktot
    v_mean = v_bulk_desired / (ratio_i * ratio_k)
    for k in range(1, ktot + 1):
        if k_start < k <= k_end:
            coorz = (k - 0.5) * dz / (cfg.lz * ratio_k)
            for i in range(1, itot + 1):
                if i_start < i <= i_end:
                    v[i, k] = 6. * v_mean * coorz * (1. - coorz)
    return v


def make_config(**kw) -> IclsConfig:
    """Reference defaults (src/param.f90) with a 3-D grid, overridden by ``kw``."""
    c = IclsConfig()
    c.itot = c.jtot = c.ktot = 32
    c.lmax = 1
    c.lx = c.ly = c.lz = 1.0
    c.timestep = 5e-4                      # param.f90:47
    c.rho1, c.rho2 = 1.0, 10.0             # param.f90:58-60
    c.miu1, c.miu2 = 1.0, 0.1
    c.Re, c.We, c.iFr = 10.0, 1.0, 0.0     # param.f90:69-71
    c.g_unit[:] = [0.0, 0.0, 0.0]
    c.v_wall_lower = c.v_wall_upper = 0.0  # ns_np=.true. (param.f90:95)
    c.TwoD = 0
    c.constPoi = 0
    c.solveLS = 1
    c.ls_adv_space = HOUC5                 # param.f90:216
    c.re_initialization = 1
    c.reinit_step = 20                     # param.f90:230
    c.reinit_iter_max = 1                  # param.f90:233
    c.mass_correction = 1
    c.inflate_step = 20                    # param.f90:258
    c.ispeed_dependence = SPEED_CURV
    c.i_space = HOUC5
    c.ioutchk = 20                         # param.f90:85
    c.precision = FP64
    c.curvature_model = CURV_STENCIL
    c.mlp_fallback_tol = 0.02
    c.mass_threshold = 0.0                 # 0: the fixed 1e-5 of levelset.f90:382
    c.mass_gain_one = 0                    # 0: the reference's inflation gain
    for k, v in kw.items():
        if k == "g_unit":
            c.g_unit[:] = list(v)
        else:
            setattr(c, k, v)
    return c


# --------------------------------------------------------------------------
# field table: (name, shape kind); kinds C=(0:i1,..), I=(1:imax,..), L=(-2:i1+2,..)
FIELDS = [
    ("u", "C"), ("v", "C"), ("w", "C"),
    ("pnew", "C"), ("pold", "C"), ("p", "C"),
    ("dudt", "C"), ("dvdt", "C"), ("dwdt", "C"),
    ("duold", "I"), ("dvold", "I"), ("dwold", "I"),
    ("p_x", "C"), ("p_y", "C"), ("p_z", "C"),
    ("p_xold", "C"), ("p_yold", "C"), ("p_zold", "C"),
    ("p_jump", "C"),
    ("miu", "C"), ("rho", "C"), ("jiemian", "C"),
    ("rho_u", "I"), ("rho_v", "I"), ("rho_w", "I"),
    ("ucc", "I"), ("vcc", "I"), ("wcc", "I"),
    ("curv", "C"), ("normal_m", "I"), ("lvset", "L"),
]
FIELD_ID = {name: i for i, (name, _) in enumerate(FIELDS)}
FIELD_KIND = {name: kind for name, kind in FIELDS}


def field_shape(cfg: IclsConfig, name: str):
    """Fortran extents (n0, n1, n2) of a field (numpy arrays use order='F')."""
    kind = FIELD_KIND[name]
    pad = {"C": 2, "I": 0, "L": 6}[kind]
    return (cfg.itot + pad, cfg.jtot + pad, cfg.ktot + pad)


def field_lo(name: str):
    return {"C": 0, "I": 1, "L": -2}[FIELD_KIND[name]]


# --------------------------------------------------------------------------
# initial level sets
def init_drops(cfg: IclsConfig, centres, radii, all_images: bool = False) -> np.ndarray:
    """Signed-distance level sets, one per drop, shape L, order='F', stacked on
    a last axis.

    With ``all_images=False`` this is init.f90 'drp'/'mdp' (717-753, 901-984):
    distance to the sphere, then on the positive side the min with the +ly
    image and then the +lx image.  ``all_images=True`` takes the min over all
    nine periodic xy-images, which a seeded multi-drop box needs when drops
    sit near any side (the reference only tests +lx, +ly).
    """
    nx, ny, nz = field_shape(cfg, "lvset")
    dxi, dyi, dzi = cfg.itot / cfg.lx, cfg.jtot / cfg.ly, cfg.ktot / cfg.lz
    ii = (np.arange(-2, cfg.itot + 4) - 0.5) / dxi
    jj = (np.arange(-2, cfg.jtot + 4) - 0.5) / dyi
    kk = (np.arange(-2, cfg.ktot + 4) - 0.5) / dzi
    X, Y, Z = np.meshgrid(ii, jj, kk, indexing="ij")
    out = np.empty((nx, ny, nz, len(radii)), order="F")
    for l, ((xc, yc, zc), r) in enumerate(zip(centres, radii)):
        ph = np.sqrt(((X - xc) ** 2 + (Y - yc) ** 2) + (Z - zc) ** 2) - r
        if all_images:
            for sx in (-cfg.lx, 0.0, cfg.lx):
                for sy in (-cfg.ly, 0.0, cfg.ly):
                    if sx == 0.0 and sy == 0.0:
                        continue
                    p2 = np.sqrt(((X - xc - sx) ** 2 + (Y - yc - sy) ** 2) + (Z - zc) ** 2) - r
                    ph = np.minimum(ph, p2)
        else:
            p1 = np.sqrt(((X - xc) ** 2 + ((Y - yc) - cfg.ly) ** 2) + (Z - zc) ** 2) - r
            ph = np.where(ph > 0.0, np.minimum(ph, p1), ph)
            p2 = np.sqrt((((X - xc) - cfg.lx) ** 2 + (Y - yc) ** 2) + (Z - zc) ** 2) - r
            ph = np.where(ph > 0.0, np.minimum(ph, p2), ph)
        out[..., l] = ph
    return out


def init_drops_boxed(cfg: IclsConfig, centres, radii, cap_cells: float = 12.0) -> np.ndarray:
    """Like ``init_drops(all_images=True)`` but the signed distance is only
    evaluated in a box of half-width R + cap_cells around each drop (with the
    periodic xy-images); everywhere else it is capped at cap_cells*dx.  The
    first tube_construction clips every value beyond 6dz (levelset.f90:107-119)
    and the Heaviside saturates beyond 1.5dz (misc.f90:445-455), so any cap
    above 6 cells leaves the solution unchanged; it only bounds the set-up
    cost for many drops on a large grid."""
    nx, ny, nz = field_shape(cfg, "lvset")
    dx, dy, dz = cfg.lx / cfg.itot, cfg.ly / cfg.jtot, cfg.lz / cfg.ktot
    cap = cap_cells * dz
    out = np.full((nx, ny, nz, len(radii)), cap, order="F")
    for l, ((xc, yc, zc), r) in enumerate(zip(centres, radii)):
        h = r + cap
        klo = max(-2, int(np.floor((zc - h) / dz + 0.5)) - 1)
        khi = min(cfg.ktot + 3, int(np.ceil((zc + h) / dz + 0.5)) + 1)
        ks = np.arange(klo, khi + 1)
        kz = (ks - 0.5) * dz
        sub = out[:, :, :, l]
        for sx in (-1, 0, 1):
            ax = np.arange(-2, cfg.itot + 4)
            gx = (ax - 0.5) * dx + sx * cfg.lx
            mx = np.abs(gx - xc) <= h + dx
            if not mx.any():
                continue
            for sy in (-1, 0, 1):
                ay = np.arange(-2, cfg.jtot + 4)
                gy = (ay - 0.5) * dy + sy * cfg.ly
                my = np.abs(gy - yc) <= h + dy
                if not my.any():
                    continue
                X, Y, Z = np.meshgrid(gx[mx], gy[my], kz, indexing="ij")
                dist = np.sqrt(((X - xc) ** 2 + (Y - yc) ** 2) + (Z - zc) ** 2) - r
                I, J, K = np.meshgrid(ax[mx] + 2, ay[my] + 2, ks + 2, indexing="ij")
                sub[I, J, K] = np.minimum(sub[I, J, K], dist)
    return out


def seeded_drops(cfg: IclsConfig, ndrop: int, rmin: float, rmax: float, seed: int,
                 gap_cells: float = 4.0, max_tries: int = 200000, y_walls: bool = False):
    """Seeded drop radii/centres: radii uniform in [rmin,rmax], centres uniform
    in the box (kept one radius plus the gap away from the z walls, and from
    the y walls too with ``y_walls``), rejected until every pair keeps
    ``gap_cells`` cells between surfaces (periodic in x and y)."""
    rng = np.random.default_rng(seed)
    dx = cfg.lx / cfg.itot
    gap = gap_cells * dx
    centres, radii = [], []
    tries = 0
    while len(radii) < ndrop:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("could not place drops with the requested gap")
        r = rng.uniform(rmin, rmax)
        cx = rng.uniform(0, cfg.lx)  # draw order x, y, z: the seeded layouts stay fixed
        cy = rng.uniform(r + gap, cfg.ly - r - gap) if y_walls else rng.uniform(0, cfg.ly)
        c = np.array([cx, cy, rng.uniform(r + gap, cfg.lz - r - gap)])
        ok = True
        for c2, r2 in zip(centres, radii):
            d = c - c2
            d[0] -= cfg.lx * round(d[0] / cfg.lx)
            d[1] -= cfg.ly * round(d[1] / cfg.ly)
            if math.sqrt(float(d @ d)) < r + r2 + gap:
                ok = False
                break
        if ok:
            centres.append(c)
            radii.append(r)
    return [tuple(c) for c in centres], radii


# --------------------------------------------------------------------------
# the measured workloads: a static drop, the rising bubble, seeded multi-drop
# layouts and the combined turbulent case, each with its grid and step count
@dataclass
class Workload:
    name: str
    cfg: IclsConfig
    centres: list
    radii: list
    all_images: bool
    shear_v: float  # initial v = shear_v*(2z-1) (0 for rest)
    steps: int
    turbulence: tuple | None = None  # (seed, rms, kmax) of a solenoidal initial velocity


def static_drop(n: int = 64, steps: int = 200) -> Workload:
    """Static droplet: n^3 on [0,1]^3, R=0.25 at the centre, rho2/rho1=10,
    miu2/miu1=10, Re=100, We=0.1, WENO5, reinit every step with 2
    pseudo-steps, dt=1e-4, at rest."""
    cfg = make_config(itot=n, jtot=n, ktot=n, lmax=1, timestep=1e-4,
                      rho1=1.0, rho2=10.0, miu1=1.0, miu2=10.0, Re=100.0, We=0.1, iFr=0.0,
                      ls_adv_space=WENO5, reinit_step=1, reinit_iter_max=2, inflate_step=20)
    return Workload("static_drop_%d" % n, cfg, [(0.5, 0.5, 0.5)], [0.25], False, 0.0, steps)


def rising_bubble(nx: int = 128, steps: int = 2000, dt: float = 4e-5) -> Workload:
    """Rising bubble: nx x nx x 2nx on [0,1]x[0,1]x[0,2], R=0.125 at
    (0.5,0.5,0.5), rho2=0.1, miu2=0.1, Re=100, We=1000/24.5, iFr=0.98,
    g=-z, HOUC5, reinit every step."""
    cfg = make_config(itot=nx, jtot=nx, ktot=2 * nx, lmax=1, lx=1.0, ly=1.0, lz=2.0,
                      timestep=dt, rho1=1.0, rho2=0.1, miu1=1.0, miu2=0.1, Re=100.0,
                      We=1000.0 / 24.5, iFr=0.98, g_unit=(0.0, 0.0, -1.0),
                      ls_adv_space=HOUC5, reinit_step=1, reinit_iter_max=1, inflate_step=1)
    return Workload("rising_bubble_%dx%dx%d" % (nx, nx, 2 * nx), cfg, [(0.5, 0.5, 0.5)],
                    [0.125], False, 0.0, steps)


def multi_drop(n: int = 256, ndrop: int = 48, seed: int = 2024, steps: int = 1000,
               rmin: float = 0.03, rmax: float = 0.06, dt: float | None = None,
               y_walls: bool = False) -> Workload:
    """Seeded multi-drop shear box: n^3 on [0,1]^3, ndrop drops with radii
    uniform in [rmin,rmax] and a 4-cell surface gap, rho and miu ratio 10,
    We=2 (sigma=0.5), Re=10 (param.f90 default), shear v=0.5(2z-1) between
    walls moving at -+0.5 (the shear is put along y, the direction the
    reference's moving-wall boundary acts on; x and y are equivalent
    periodic directions), HOUC5, reference reinit/inflation cadence (20).
    That cadence is stable for the mass correction only below n ~= 90 on the
    unit box (each correction multiplies the volume error by 1 - K/20, K ~=
    0.44 n); at 256^3 the first correction, near step 280, starts a
    growing oscillation, and inflate_step ~= 112 corrects in one go."""
    cfg = make_config(itot=n, jtot=n, ktot=n, lmax=ndrop, timestep=1e-5,
                      rho1=1.0, rho2=10.0, miu1=1.0, miu2=10.0, Re=10.0, We=2.0,
                      v_wall_lower=-0.5, v_wall_upper=0.5, ls_adv_space=HOUC5,
                      reinit_step=20, reinit_iter_max=1, inflate_step=20)
    centres, radii = seeded_drops(cfg, ndrop, rmin, rmax, seed, y_walls=y_walls)
    if y_walls:  # BC_in_y = 'Walls': solver2d_cos, no driving gradient (ab2.f90:103-118)
        cfg.bc_y = BCY_WALLS
        cfg.constPoi = 0
    if dt is not None:
        cfg.timestep = dt
    return Workload("multi_drop_%d_%d" % (n, ndrop), cfg, centres, radii, True, 0.5, steps)


def combined(n: int = 384, ndrop: int = 200, seed: int = 2024, steps: int = 2000, rmin: float = 0.02,
             rmax: float = 0.04, rms: float = 0.2, kmax: int = 8, dt: float | None = None) -> Workload:
    """The combined-form configuration: n^3 on [0,1]^3, ndrop seeded drops
    with radii uniform in [rmin,rmax] and a 4-cell surface gap, a seeded
    random solenoidal velocity with a k^-5/3 spectrum over |k| = 1..kmax and
    the given rms (solenoidal_velocity), rho and miu ratio 10, sigma = 0.2
    (We = 5), Re = 10, walls at rest, HOUC5, reinitialisation and inflation
    every 20 steps.  The configuration is the plain method's; the FP32 form
    and the learned curvature are chosen by the caller (precision,
    curvature_model).

    dt defaults to 1e-5 up to 256^3 and shrinks with dx^2 beyond it (0.9 x
    1e-5 x (256/n)^2, 4e-6 at 384^3).  The explicit viscous term of the cells
    where the phases mix binds first; chkdt's estimate (chkdt.f90:62-104, the
    larger of the two pure phases' mu/rho) does not see it.  At 384^3 with
    dt = 1e-5 the velocity grows without bound from step 14 (max|u| 0.9 ->
    58 by step 23), while 4e-6 and 2e-6 stay steady over 60 steps.

    inflate_step stays at the reference's 20, which the timed steps never
    reach with a volume error above the 1e-5 trigger.  A long run at this
    size needs it near K ~= 0.44 n (about 170 at 384^3): at 20 each mass
    correction multiplies the volume error by 1 - K/20."""
    if dt is None:
        dt = 1e-5 if n <= 256 else float("%.2g" % (0.9e-5 * (256.0 / n) ** 2))
    cfg = make_config(itot=n, jtot=n, ktot=n, lmax=ndrop, timestep=dt,
                      rho1=1.0, rho2=10.0, miu1=1.0, miu2=10.0, Re=10.0, We=5.0,
                      ls_adv_space=HOUC5, reinit_step=20, reinit_iter_max=1, inflate_step=20)
    centres, radii = seeded_drops(cfg, ndrop, rmin, rmax, seed)
    return Workload("combined_%d_%d" % (n, ndrop), cfg, centres, radii, True, 0.0, steps,
                    (seed + 1, rms, kmax))


def solenoidal_velocity(cfg: IclsConfig, seed: int, rms: float = 0.2, kmax: int = 8, slope: float = -5.0 / 3.0):
    """u, v, w on shape C: a seeded random field that is divergence-free on
    the staggered grid to roundoff.  u = curl A with the vector potential on
    cell edges (A_x at ((i-1/2)dx, j dy, k dz), A_y at (i dx, (j-1/2)dy, k dz),
    A_z at (i dx, j dy, (k-1/2)dz)), so the discrete divergence of the face
    velocities is an exact telescoping sum.  A has Fourier modes in x and y
    (periodic) and half-wave sine modes sin(pi m z / lz) in z, so A_x and A_y
    vanish on the walls and w = 0 there; modes with 1 <= |k| <= kmax (k in
    cycles per length, m/2 along z) get random complex amplitudes scaled as
    |k|^((slope - 2)/2) / |k| (a shell energy spectrum ~ k^slope for the
    velocity).  The field is scaled to the given rms over the interior
    faces; halos are left to init_program's boundary pass."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = cfg.itot, cfg.jtot, cfg.ktot
    dx, dy, dz = cfg.lx / nx, cfg.ly / ny, cfg.lz / nz
    kx = np.fft.fftfreq(nx, d=1.0 / nx)[:, None] / cfg.lx
    ky = np.fft.fftfreq(ny, d=1.0 / ny)[None, :] / cfg.ly

    def component(sx, sy, zpos):
        """one potential component at x = (i0 + sx) dx, y = (j0 + sy) dy
        (i0, j0 = 0..n-1) and the given z positions"""
        out = np.zeros((nx, ny, zpos.size))
        for m in range(1, 2 * kmax + 1):
            kz = 0.5 * m / cfg.lz
            kk = np.sqrt(kx * kx + ky * ky + kz * kz)
            sel = (kk >= 1.0) & (kk <= kmax)
            if not sel.any():
                continue
            amp = np.where(sel, kk ** ((slope - 2.0) / 2.0) / np.maximum(kk, 1e-30), 0.0)
            coef = amp * (rng.standard_normal((nx, ny)) + 1j * rng.standard_normal((nx, ny)))
            # shift theorem: the plane sampled at the component's offsets
            coef = coef * np.exp(2j * np.pi * (np.fft.fftfreq(nx)[:, None] * sx + np.fft.fftfreq(ny)[None, :] * sy))
            plane = np.fft.ifft2(coef).real * (nx * ny)
            out += plane[:, :, None] * np.sin(np.pi * m * zpos / cfg.lz)[None, None, :]
        return out

    zk = np.arange(nz + 1) * dz            # k dz, k = 0..nz
    zc = (np.arange(nz) + 0.5) * dz        # (k - 1/2) dz, k = 1..nz
    Ax = component(0.5, 1.0, zk)
    Ay = component(1.0, 0.5, zk)
    Az = component(1.0, 1.0, zc)
    roll = np.roll
    u = (Az - roll(Az, 1, axis=1)) / dy - (Ay[:, :, 1:] - Ay[:, :, :-1]) / dz
    v = (Ax[:, :, 1:] - Ax[:, :, :-1]) / dz - (Az - roll(Az, 1, axis=0)) / dx
    w = (Ay[:, :, 1:] - roll(Ay, 1, axis=0)[:, :, 1:]) / dx - (Ax[:, :, 1:] - roll(Ax, 1, axis=1)[:, :, 1:]) / dy
    scale = rms / math.sqrt(float(np.mean(u * u) + np.mean(v * v) + np.mean(w * w)) / 3.0)
    out = []
    for f in (u, v, w):
        a = np.zeros(field_shape(cfg, "u"), order="F")
        a[1:nx + 1, 1:ny + 1, 1:nz + 1] = scale * f
        a[0] = a[nx]
        a[nx + 1] = a[1]
        a[:, 0] = a[:, ny]
        a[:, ny + 1] = a[:, 1]
        out.append(a)
    return tuple(out)


def workload_velocity(wl: Workload):
    """the initial u, v, w of a workload: the seeded solenoidal field, the
    shear, or rest"""
    if wl.turbulence is not None:
        seed, rms, kmax = wl.turbulence
        return solenoidal_velocity(wl.cfg, seed, rms, kmax)
    return initial_velocity(wl.cfg, wl.shear_v)


def initial_velocity(cfg: IclsConfig, shear_v: float):
    """u, v, w on shape C: rest, or v = shear_v*(2z-1) at cell-face heights."""
    shp = field_shape(cfg, "u")
    u = np.zeros(shp, order="F")
    v = np.zeros(shp, order="F")
    w = np.zeros(shp, order="F")
    if shear_v != 0.0:
        dz = cfg.lz / cfg.ktot
        z = (np.arange(0, cfg.ktot + 2) - 0.5) * dz / cfg.lz
        v[:, :, :] = (shear_v * (2.0 * z - 1.0))[None, None, :]
    return u, v, w
