"""The learned curvature's tensor-core path (needs a B200).

The MLP's products run on tcgen05 tiles: BF16 operands in shared memory,
FP32 accumulation in tensor memory.  A single 128 x n tile is checked here
against the FP32 product of the same BF16 values (tolerance 1e-5 relative to
the largest |entry|: only the summation order differs)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from icls_gpu.binding import gpu_backend


@pytest.mark.parametrize("n,k", [(16, 16), (128, 32), (64, 128), (128, 128)])
def test_tc_tile_matches_fp32_product(gpu_available, n, k):
    import torch
    g = torch.Generator().manual_seed(n * 1000 + k)
    a = torch.randn(128, k, generator=g).to(torch.bfloat16)
    b = torch.randn(n, k, generator=g).to(torch.bfloat16)
    ref = a.float() @ b.float().T
    da, db = a.cuda(), b.cuda()
    dd = torch.zeros(128, n, dtype=torch.float32, device="cuda")
    fn = gpu_backend().lib.icls_tc_gemm_bf16
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]
    fn.restype = C.c_int
    rc = fn(da.data_ptr(), db.data_ptr(), dd.data_ptr(), n, k, torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    out = dd.cpu()
    err = float((out - ref).abs().max()) / float(ref.abs().max())
    assert err <= 1e-5, err


# ---------------------------------------------------------------- network
def _lib():
    lib = gpu_backend().lib
    P = C.c_void_p
    sig = {
        "icls_mlp_create": [C.POINTER(P), C.c_ulonglong],
        "icls_mlp_destroy": [P],
        "icls_mlp_make_data": [P, C.c_ulonglong, C.c_longlong, C.c_longlong],
        "icls_mlp_train": [P, C.c_int, C.c_int, C.c_double, C.c_double, C.c_ulonglong, C.POINTER(C.c_double)],
        "icls_mlp_eval": [P, C.POINTER(C.c_double)],
        "icls_mlp_params": [P, C.POINTER(C.c_float), C.c_int],
        "icls_mlp_grad": [P, P, P, C.c_longlong, C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_double)],
    }
    for name, args in sig.items():
        getattr(lib, name).argtypes = args
        getattr(lib, name).restype = C.c_int
    return lib


def _sphere_stencils(n, seed):
    """27-value stencils of signed distances to seeded spheres, as the network
    takes them: (phi(x + o) - phi(x)), o in {-1,0,1}^3 (z outer), padded to 32"""
    rng = np.random.default_rng(seed)
    o = np.array([(i, j, k) for k in (-1, 0, 1) for j in (-1, 0, 1) for i in (-1, 0, 1)], dtype=float)
    X = np.zeros((n, 32))
    lab = np.zeros(n)
    for s in range(n):
        R = rng.uniform(3, 40)
        u = rng.normal(size=3)
        u /= np.linalg.norm(u)
        x = np.rint(rng.uniform(size=3) + (R + rng.uniform(-2, 2)) * u)
        c = rng.uniform(size=3)
        phi = np.linalg.norm(x + o - c, axis=1) - R
        X[s, :27] = phi - phi[13]
        lab[s] = -2.0 / np.linalg.norm(x - c)
    return X, lab


def test_mlp_gradient_matches_cpu_oracle(gpu_available):
    import torch
    from oracle.mlp_oracle import NPARAMS, OFF, gradient
    lib = _lib()
    m = C.c_void_p()
    assert lib.icls_mlp_create(C.byref(m), 7) == 0
    try:
        theta = np.zeros(NPARAMS, dtype=np.float32)
        assert lib.icls_mlp_params(m, theta.ctypes.data_as(C.POINTER(C.c_float)), 1) == 0
        n = 256
        X, lab = _sphere_stencils(n, 11)
        dX = torch.tensor(X, dtype=torch.float32).cuda()
        dl = torch.tensor(lab, dtype=torch.float32).cuda()
        g = np.zeros(NPARAMS, dtype=np.float32)
        loss = C.c_double()
        scale = 2.0 / n
        assert lib.icls_mlp_grad(m, dX.data_ptr(), dl.data_ptr(), n, scale, g.ctypes.data_as(C.POINTER(C.c_float)),
                                 C.byref(loss)) == 0
        ref, ref_loss = gradient(theta, dX.float().cpu().numpy(), dl.cpu().numpy(), scale)
        print("\nloss gpu %.6e oracle %.6e" % (loss.value, ref_loss))
        errs = {}
        for name, (a, b) in OFF.items():
            errs[name] = np.linalg.norm(g[a:b] - ref[a:b]) / max(np.linalg.norm(ref[a:b]), 1e-30)
        print("gradient relative L2 per block", {k: "%.2e" % v for k, v in errs.items()})
        assert abs(loss.value - ref_loss) <= 1e-4 * ref_loss
        for name, err in errs.items():
            assert err <= 2e-3, (name, err)
    finally:
        lib.icls_mlp_destroy(m)


def test_mlp_training_beats_plain_stencil(gpu_available):
    """4M seeded samples, 20 epochs of batch 8192 (the training configuration):
    the network's held-out curvature error against the analytic curvature is
    below the plain 10x27 stencil's."""
    lib = _lib()
    m = C.c_void_p()
    assert lib.icls_mlp_create(C.byref(m), 2024) == 0
    try:
        assert lib.icls_mlp_make_data(m, 99, 1 << 22, 1 << 16) == 0
        losses = (C.c_double * 20)()
        assert lib.icls_mlp_train(m, 20, 8192, 1e-3, 1e-5, 5, losses) == 0
        st = (C.c_double * 8)()
        assert lib.icls_mlp_eval(m, st) == 0
        print("\nloss per epoch", ["%.3e" % v for v in losses])
        print("held-out (kappa*dx): rms mlp-label %.3e, mlp-analytic %.3e, plain-analytic %.3e, "
              "label-analytic %.3e, max mlp-analytic %.3e, max plain-analytic %.3e, rms analytic %.3e, n %d"
              % (tuple(st[:7]) + (int(st[7]),)))
        assert losses[19] < losses[0]
        assert st[1] < st[2]
    finally:
        lib.icls_mlp_destroy(m)


def _shell_error(solver, h, radius_cells):
    """rms of (curv - analytic) * dx on the |phi| <= 1.5dx shell of the drop
    centred in the box"""
    n = solver.cfg.itot
    x = (np.arange(n + 2) - 0.5) * h
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    r = np.sqrt((X - 0.5) ** 2 + (Y - 0.5) ** 2 + (Z - 0.5) ** 2)
    phi = solver.download("lvset", 1)[2:-2, 2:-2, 2:-2]
    shell = np.abs(phi) <= 1.5 * h
    return float(np.sqrt(np.mean((solver.download("curv")[shell] + 2.0 / r[shell]) ** 2)) * h)


@pytest.fixture(scope="module")
def trained_net(gpu_available):
    """the network trained as in the training test, on 4M samples"""
    from icls_gpu.binding import Mlp
    net = Mlp(2024)
    net.make_data(99, 1 << 22, 1 << 14)
    net.train(epochs=20)
    yield net
    net.close()


def test_learned_curvature_in_the_loop(trained_net):
    """Static drops of radius 5 and 16 cells: the curvature gfm4p uses at the
    interface, from the network (with per-cell fallback) and from the plain
    stencil, against the analytic -2/r (after re_curvature's smoothing, which
    both share).  Measured: within 1% of kappa for the resolved drop (the
    stencil is better still there), and within 1.5x the stencil's error for
    the 5-cell drop, where the held-out gain of the training distribution
    (test above) does not carry over to a single sphere; then 20 steps run
    with the network in the loop."""
    from icls_gpu import CURV_MLP, Solver, init_drops, initial_velocity, static_drop
    from icls_gpu.binding import curvature_stats
    from icls_gpu.config import IclsConfig
    net = trained_net
    res = {}
    for rc in (5, 16):
        wl = static_drop(64, steps=20)
        wl.radii = [rc / 64.0]
        cfg_m = IclsConfig.from_buffer_copy(wl.cfg)
        cfg_m.curvature_model = CURV_MLP
        ls = init_drops(wl.cfg, wl.centres, wl.radii, wl.all_images)
        u, v, w = initial_velocity(wl.cfg, wl.shear_v)
        sp, sm = Solver(wl.cfg), Solver(cfg_m)
        net.attach(sm)
        for s in (sp, sm):
            s.setup(ls, u, v, w)
            s.gfm4p()
        h = 1.0 / 64
        res[rc] = (_shell_error(sp, h, rc), _shell_error(sm, h, rc), curvature_stats(sm, reset=True))
        print("\nR = %2d cells: re_curvature vs -2/r (kappa*dx rms) stencil %.3e, network %.3e; "
              "network evaluated %d cells, %d fell back" % (rc, res[rc][0], res[rc][1], res[rc][2][0], res[rc][2][1]))
        if rc == 16:
            for istep in range(1, 21):
                sp.step(istep, 0)
                sm.step(istep, 0)
            ev, fb = curvature_stats(sm)
            print("R = 16, 20 steps: spurious max|u| stencil %.3e, network %.3e; fallback fraction %.3f"
                  % (sp.max_vel_at_center(), sm.max_vel_at_center(), fb / max(ev, 1)))
            assert np.isfinite(sm.max_vel_at_center())
    assert res[5][1] < 1.5 * res[5][0]
    assert res[16][1] < 0.01 * (2.0 / 16)


def test_fp32_form_with_learned_curvature(trained_net):
    """The combined form (FP32 bulk, FP64 Poisson/volume/jumps, network
    curvature with per-cell fallback) on the 64^3 static drop of radius 16
    cells for 20 steps, against the plain FP64 stencil run: drop volume
    within 1e-6, interface curvature within 1% of kappa, velocities finite."""
    from icls_gpu import CURV_MLP, FP32, Solver, init_drops, initial_velocity, static_drop
    from icls_gpu.binding import curvature_stats
    from icls_gpu.config import IclsConfig
    wl = static_drop(64, steps=20)
    cf = IclsConfig.from_buffer_copy(wl.cfg)
    cf.precision = FP32
    cf.curvature_model = CURV_MLP
    ls = init_drops(wl.cfg, wl.centres, wl.radii, wl.all_images)
    u, v, w = initial_velocity(wl.cfg, wl.shear_v)
    sp, sf = Solver(wl.cfg), Solver(cf)
    trained_net.attach(sf)
    for s in (sp, sf):
        s.setup(ls, u, v, w)
        for istep in range(1, 21):
            s.step(istep, 0)
    h = 1.0 / 64
    ep, ef = _shell_error(sp, h, 16), _shell_error(sf, h, 16)
    vp, vf = sp.volumes()[0][0], sf.volumes()[0][0]
    ev, fb = curvature_stats(sf)
    print("\nFP32 + network, 20 steps: kappa*dx rms vs -2/r stencil(FP64) %.3e, form %.3e; volume rel diff %.2e; "
          "spurious max|u| FP64 %.3e, form %.3e; fallback fraction %.3f"
          % (ep, ef, abs(vf - vp) / vp, sp.max_vel_at_center(), sf.max_vel_at_center(), fb / max(ev, 1)))
    assert ev > 0
    assert np.isfinite(sf.max_vel_at_center())
    assert abs(vf - vp) / vp <= 1e-6
    assert ef < 0.01 * (2.0 / 16)


def test_combined_form_96(trained_net):
    """The combined configuration's kinds of input at 96^3 (FFT lines of
    16 x 6 points, 12 seeded drops of 7-10 cells, a seeded solenoidal
    velocity): FP32 with the network curvature against the plain FP64
    stencil run for 10 steps.  Bounds: finite velocities, per-drop volume
    within 1e-6 of FP64, drop volumes conserved to 1e-5 over the run in
    both."""
    from icls_gpu import CURV_MLP, FP32, Solver, combined, init_drops, workload_velocity
    from icls_gpu.binding import curvature_stats
    from icls_gpu.config import IclsConfig
    wl = combined(96, 12, rmin=0.07, rmax=0.1)
    ls = init_drops(wl.cfg, wl.centres, wl.radii, wl.all_images)
    u, v, w = workload_velocity(wl)
    cf = IclsConfig.from_buffer_copy(wl.cfg)
    cf.precision = FP32
    cf.curvature_model = CURV_MLP
    sp, sf = Solver(wl.cfg), Solver(cf)
    trained_net.attach(sf)
    for s in (sp, sf):
        s.setup(ls, u, v, w)
        for istep in range(1, 11):
            s.step(istep, 0)
    vp, vp0 = sp.volumes()
    vf, vf0 = sf.volumes()
    ev, fb = curvature_stats(sf)
    du = float(np.linalg.norm(sf.download("u") - sp.download("u")) / np.linalg.norm(sp.download("u")))
    print("\ncombined 96^3 x 12, 10 steps: volume vs FP64 %.2e, drift FP64 %.2e form %.2e, u rel L2 %.2e, "
          "max|u| FP64 %.3e form %.3e, fallback %.3f"
          % (np.max(np.abs(vf - vp) / vp), np.max(np.abs(vp - vp0) / vp0), np.max(np.abs(vf - vf0) / vf0), du,
             sp.max_vel_at_center(), sf.max_vel_at_center(), fb / max(ev, 1)))
    assert np.isfinite(sf.max_vel_at_center()) and np.isfinite(sp.max_vel_at_center())
    assert np.max(np.abs(vf - vp) / vp) <= 1e-6
    assert np.max(np.abs(vp - vp0) / vp0) <= 1e-5 and np.max(np.abs(vf - vf0) / vf0) <= 1e-5
    assert ev > 0


# bounds of the decomposition test below (relative L2 after 43 steps;
# measured: total u 2.4e-2, v 1.4e-5, w 1.0e-2; precision u 1.3e-4)
BOUND_TOTAL = {"u": 5e-2, "v": 5e-5, "w": 2.5e-2}
BOUND_PRECISION = 5e-4
BOUND_BIAS = 2e-3     # measured 4.6e-4
BOUND_RMS = 1e-2      # spurious-current magnitude change, measured 1.3e-3


def _seeded_shells(wl):
    """Per drop, the shape-C cells with ||x - c| - R| <= 1.5 dx (minimum
    image in x and y): flat Fortran-order indices and distances |x - c|."""
    cfg = wl.cfg
    n1, n2, n3 = cfg.itot + 2, cfg.jtot + 2, cfg.ktot + 2
    h = cfg.lz / cfg.ktot
    x = (np.arange(n1) - 0.5) * h
    y = (np.arange(n2) - 0.5) * h
    z = (np.arange(n3) - 0.5) * h
    out = []
    for c, R in zip(wl.centres, wl.radii):
        dx = x - c[0]
        dx -= cfg.lx * np.round(dx / cfg.lx)
        dy = y - c[1]
        dy -= cfg.ly * np.round(dy / cfg.ly)
        X, Y, Z = np.meshgrid(dx, dy, z - c[2], indexing="ij")
        r = np.sqrt(X * X + Y * Y + Z * Z)
        m = (np.abs(r - R) <= 1.5 * h)
        m[0, :, :] = m[-1, :, :] = False
        m[:, 0, :] = m[:, -1, :] = False
        out.append((np.flatnonzero(m.ravel(order="F")), r.ravel(order="F")[np.flatnonzero(m.ravel(order="F"))]))
    return out


def test_learned_form_velocity_error_decomposed(trained_net):
    """The velocity error of the FP32 + learned-curvature form against the
    plain FP64 run, split into its two causes, on the 128^3 box with 12
    seeded drops of 7.7-15 cells (the bench's drop sizes), 43 steps:

      network    FP64 with the network's curvature vs the FP64 stencil
      precision  the FP32 form with the network vs FP64 with the network

    The network accounts for nearly all of it.  It is no bias: the spurious
    currents keep their magnitude (rms of u, w within 1%), and the network's
    curvature on the drops' shells is shifted from the stencil's by under
    0.2% on average; what moves the velocity is its 0.26% rms cell-to-cell
    difference from the stencil, which the surface-tension-driven u and w
    (spurious currents, O(1e-4)) follow.  On these drops the network's
    curvature is also the closer of the two to the analytic -2/r."""
    from icls_gpu import CURV_MLP, FP32, Solver, init_drops, workload_velocity
    from icls_gpu.config import IclsConfig, multi_drop
    from conftest import rel_l2
    wl = multi_drop(n=128, ndrop=12, seed=2024, steps=43, rmin=0.06, rmax=0.12)
    ls = init_drops(wl.cfg, wl.centres, wl.radii, wl.all_images)
    u, v, w = workload_velocity(wl)

    def make(prec, curv):
        c = IclsConfig.from_buffer_copy(wl.cfg)
        c.precision, c.curvature_model = prec, curv
        s = Solver(c)
        if curv == CURV_MLP:
            trained_net.attach(s)
        s.setup(ls, u, v, w)
        return s

    runs = {"fp64": make(0, 0), "fp64_net": make(0, CURV_MLP), "form": make(FP32, CURV_MLP)}
    for istep in range(1, 44):
        for s in runs.values():
            s.step(istep, 0)
    f = {k: {n: s.download(n) for n in ("u", "v", "w")} for k, s in runs.items()}
    err = {pair: {n: rel_l2(f[a][n], f[b][n]) for n in ("u", "v", "w")}
           for pair, (a, b) in {"total": ("form", "fp64"), "network": ("fp64_net", "fp64"),
                                "precision": ("form", "fp64_net")}.items()}
    rms = {k: {n: float(np.sqrt(np.mean(f[k][n] ** 2))) for n in ("u", "w")} for k in f}
    # the curvature gfm4p uses, on every drop's seeded shell
    shells = _seeded_shells(wl)
    kap, rr = {}, np.concatenate([r for _, r in shells])
    for k, s in runs.items():
        vals = []
        for l, (flat, _r) in enumerate(shells, start=1):
            s.get_curvature(l)
            vals.append(s.download("curv").ravel(order="F")[flat])
        kap[k] = np.concatenate(vals)
    bias = float(np.mean(kap["fp64_net"] - kap["fp64"]) / np.mean(np.abs(kap["fp64"])))
    ana = {k: float(np.sqrt(np.mean((kv + 2.0 / rr) ** 2)) / np.sqrt(np.mean((2.0 / rr) ** 2)))
           for k, kv in kap.items()}
    print("\nlearned form, 128^3 x 12 drops, 43 steps, relative L2 of u, v, w: " +
          "; ".join("%s %.2e %.2e %.2e" % (k, e["u"], e["v"], e["w"]) for k, e in err.items()) +
          "; rms u, w: " + "; ".join("%s %.4e %.4e" % (k, r["u"], r["w"]) for k, r in rms.items()) +
          "; network's mean curvature shift vs the stencil %.2e; kappa rms vs -2/r: stencil %.4e, network %.4e"
          % (bias, ana["fp64"], ana["fp64_net"]))
    for n in ("u", "v", "w"):
        assert err["total"][n] <= BOUND_TOTAL[n], (n, err["total"][n])
        assert err["precision"][n] <= BOUND_PRECISION, (n, err["precision"][n])
    for n in ("u", "w"):
        assert abs(rms["fp64_net"][n] / rms["fp64"][n] - 1.0) <= BOUND_RMS, n
    assert abs(bias) <= BOUND_BIAS
    assert ana["fp64_net"] < ana["fp64"]
