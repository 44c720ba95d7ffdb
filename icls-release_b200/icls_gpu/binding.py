"""ctypes binding of the C ABI (include/icls_gpu.h).

``Solver`` exposes the subroutines that the reference driver
(src/main.f90:103-291) calls, under the reference's names, on top of an
``icls_ctx``.  Any non-zero status raises ``IclsError``: the reference stops
the program at the same points (main.f90:207-210, chkdiv.f90:60-87).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .config import (FIELD_ID, IclsConfig, IclsScalars, STATUS_NAMES, field_lo,
                     field_shape)

_PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG_DIR, "libicls_gpu.so")


class IclsError(RuntimeError):
    def __init__(self, code: int, where: str):
        self.code = code
        super().__init__("%s failed with %s (%d)" % (where, STATUS_NAMES.get(code, "?"), code))


_P = C.c_void_p
_I = C.c_int
_D = C.c_double
_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int)

# name -> argtypes after the ctx pointer
_SIGS = {
    "init_program": [],
    "ls_main": [_I],
    "average_stream_vel": [_DP],
    "ab2": [],
    "fillps": [],
    "gfm4p": [],
    "add_pjump": [],
    "solver2d": [],
    "boundp": [_I],
    "correc": [],
    "bounduvw": [_I],
    "pressure_update": [_I, _I],
    "average_vel_at_center": [],
    "max_vel_at_center": [_DP],
    "set_inflow": [_DP],
    "download_plane_x": [_I, _I, _I, _DP],
    "timestep_record": [_I, _DP],
    "disp": [_I, _DP, _DP],
    "write_checkpoint": [C.c_char_p, _I, _I],
    "read_checkpoint": [C.c_char_p, _IP],
    "chkdiv": [_I, _DP, _DP, _IP],
    "chkdt": [_DP],
    "ipot": [_DP],
    "step": [_I, _I],
    "tube_construction": [_I],
    "ls_advection": [_I],
    "ls_mass_correction": [_I, _I],
    "ls_reinit_main": [_I, _I],
    "update_materials": [],
    "get_curvature": [_I],
    "band_count": [_I, C.POINTER(C.c_longlong)],
    "field_bounds": [_I, _IP, _IP],
    "upload_field": [_I, _I, _DP],
    "download_field": [_I, _I, _DP],
    "get_scalars": [C.POINTER(IclsScalars)],
    "get_volumes": [_DP, _DP],
    "destroy": [],
    "profile_enable": [_I],
    "profile_reset": [],
    "profile_count": [_IP],
    "profile_entry": [_I, C.c_char_p, _I, _DP, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)],
    "launch_count": [C.POINTER(C.c_longlong)],
    "get_stream": [C.POINTER(C.c_void_p)],
}


class Backend:
    """A loaded shared library exposing the C ABI under ``prefix``."""

    def __init__(self, path: str, prefix: str):
        if not os.path.exists(path):
            raise FileNotFoundError(
                "%s not found: build it first (python __graft_entry__.py build)" % path)
        self.path = path
        self.prefix = prefix
        self.lib = C.CDLL(path)
        create = getattr(self.lib, prefix + "create")
        create.argtypes = [C.POINTER(IclsConfig), C.POINTER(_P)]
        create.restype = _I
        for name, args in _SIGS.items():
            fn = getattr(self.lib, prefix + name, None)
            if fn is None:
                continue
            fn.argtypes = [_P] + args
            fn.restype = _I

    def fn(self, name):
        return getattr(self.lib, self.prefix + name)


_GPU_BACKEND = None


def gpu_backend() -> Backend:
    """The CUDA library.  Raises if it has not been built: there is no CPU
    fallback."""
    global _GPU_BACKEND
    if _GPU_BACKEND is None:
        _GPU_BACKEND = Backend(LIB_PATH, "icls_")
        st = _GPU_BACKEND.lib.icls_status_string
        st.argtypes = [_I, C.c_char_p, _I]
        st.restype = _I
    return _GPU_BACKEND


class Solver:
    """One context: the device-resident state of the reference's mod_common."""

    def __init__(self, cfg: IclsConfig, backend: Backend | None = None):
        self.be = backend if backend is not None else gpu_backend()
        self.cfg = cfg
        self._cfg_ref = IclsConfig.from_buffer_copy(cfg)
        h = _P()
        rc = self.be.fn("create")(C.byref(self._cfg_ref), C.byref(h))
        if rc:
            raise IclsError(rc, self.be.prefix + "create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.be.fn("destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ------------------------------------------------------------------
    def _call(self, name, *args):
        rc = self.be.fn(name)(self.h, *args)
        if rc:
            raise IclsError(rc, self.be.prefix + name)
        return rc

    def upload(self, name: str, arr, l: int = 1):
        shp = field_shape(self.cfg, name)
        a = np.asfortranarray(arr, dtype=np.float64)
        if a.shape != shp:
            raise ValueError("%s: expected shape %s, got %s" % (name, shp, a.shape))
        self._call("upload_field", FIELD_ID[name], l, a.ctypes.data_as(_DP))

    def upload_ptr(self, name: str, ptr: int, l: int = 1):
        """Upload from a raw host address (e.g. pinned memory) holding the
        field in Fortran order."""
        self._call("upload_field", FIELD_ID[name], l, C.cast(C.c_void_p(ptr), _DP))

    def download_ptr(self, name: str, ptr: int, l: int = 1):
        self._call("download_field", FIELD_ID[name], l, C.cast(C.c_void_p(ptr), _DP))

    def probe(self, name: str, i: int, j: int, k: int, l: int = 1) -> float:
        x = C.c_double()
        fn = self.be.fn("probe")
        fn.argtypes = [_P, _I, _I, _I, _I, _I, _DP]
        fn.restype = _I
        rc = fn(self.h, FIELD_ID[name], l, i, j, k, C.byref(x))
        if rc:
            raise IclsError(rc, self.be.prefix + "probe")
        return x.value

    def download(self, name: str, l: int = 1) -> np.ndarray:
        a = np.empty(field_shape(self.cfg, name), order="F")
        self._call("download_field", FIELD_ID[name], l, a.ctypes.data_as(_DP))
        return a

    def bounds(self, name: str):
        lo = (C.c_int * 3)()
        hi = (C.c_int * 3)()
        self._call("field_bounds", FIELD_ID[name], lo, hi)
        return tuple(lo), tuple(hi)

    def scalars(self) -> dict:
        s = IclsScalars()
        self._call("get_scalars", C.byref(s))
        return {n: getattr(s, n) for n, _ in IclsScalars._fields_}

    def volumes(self):
        L = self.cfg.lmax
        v = np.zeros(L)
        v0 = np.zeros(L)
        self._call("get_volumes", v.ctypes.data_as(_DP), v0.ctypes.data_as(_DP))
        return v, v0

    # --- the subroutines main.f90 calls -------------------------------
    def init_program(self):
        self._call("init_program")

    def ls_main(self, istep: int):
        self._call("ls_main", istep)

    def average_stream_vel(self) -> float:
        x = C.c_double()
        self._call("average_stream_vel", C.byref(x))
        return x.value

    def ab2(self):
        self._call("ab2")

    def fillps(self):
        self._call("fillps")

    def gfm4p(self):
        self._call("gfm4p")

    def add_pjump(self):
        self._call("add_pjump")

    def solver2d(self):
        self._call("solver2d")

    def boundp(self, name: str = "p"):
        self._call("boundp", FIELD_ID[name])

    def correc(self):
        self._call("correc")

    def bounduvw(self, name: str = "u"):
        self._call("bounduvw", FIELD_ID[name])

    def pressure_update(self, istep: int, begin: int = 0):
        self._call("pressure_update", istep, begin)

    def average_vel_at_center(self):
        self._call("average_vel_at_center")

    def max_vel_at_center(self) -> float:
        x = C.c_double()
        self._call("max_vel_at_center", C.byref(x))
        return x.value

    def download_plane_x(self, name: str, i: int, l: int = 1) -> np.ndarray:
        """The plane i = const of a field over its own (j, k) bounds, indexed
        [j - lo1, k - lo2]."""
        lo, hi = self.bounds(name)
        a = np.zeros((hi[1] - lo[1] + 1, hi[2] - lo[2] + 1), order="F")
        self._call("download_plane_x", FIELD_ID[name], l, i, a.ctypes.data_as(_DP))
        return a

    def timestep_record(self, istep: int) -> np.ndarray:
        """(istep, time, dt, massloss, dmin(1,2)/dz, maxchk_glb), the
        timestep.txt record of main.f90:243-256."""
        r = np.zeros(6)
        self._call("timestep_record", istep, r.ctypes.data_as(_DP))
        return r

    def set_inflow(self, v_inflow: np.ndarray):
        """v_inflow(0:i1,0:k1) of bc_y = INOUT (bound.f90:118-130)."""
        a = np.asfortranarray(v_inflow, dtype=np.float64)
        assert a.shape == (self.cfg.itot + 2, self.cfg.ktot + 2)
        self._call("set_inflow", a.ctypes.data_as(_DP))

    def disp(self, l: int = 1):
        """disp_cg and disp_speed of drop l: (centroid[3], velocity[3])"""
        cg, vel = np.zeros(3), np.zeros(3)
        self._call("disp", l, cg.ctypes.data_as(_DP), vel.ctypes.data_as(_DP))
        return cg, vel

    def chkdiv(self, istep: int, raise_on_error: bool = True):
        tot, mx = C.c_double(), C.c_double()
        ijk = (C.c_int * 3)()
        rc = self.be.fn("chkdiv")(self.h, istep, C.byref(tot), C.byref(mx), ijk)
        if rc and raise_on_error:
            raise IclsError(rc, self.be.prefix + "chkdiv")
        return tot.value, mx.value, tuple(ijk), rc

    def chkdt(self) -> float:
        x = C.c_double()
        self._call("chkdt", C.byref(x))
        return x.value

    def ipot(self) -> np.ndarray:
        L = self.cfg.lmax
        d = np.zeros((L, L), order="F")
        self._call("ipot", d.ctypes.data_as(_DP))
        return d

    def step(self, istep: int, begin: int = 0):
        self._call("step", istep, begin)

    def write_checkpoint(self, path: str, nr: int, history: bool = True):
        """loadflds('w', nr) (loadd.f90:28-103): u, v, w, pnew, lvset(1..L)
        and jiemian over the interior, then (time, nr, dt).  With
        ``history`` also ``path.hist``: the AB2 and pressure history, the
        pressure-normalisation mean and the initial drop volumes, which an
        exact continuation needs."""
        self._call("write_checkpoint", os.fsencode(path), nr, 1 if history else 0)

    def read_checkpoint(self, path: str) -> int:
        """loadflds('r') followed by init_program; restores ``path.hist``
        when it exists.  Returns nr.  Continue with ``step(istep, begin=0)``
        for istep > nr to reproduce the uninterrupted run."""
        nr = C.c_int()
        self._call("read_checkpoint", os.fsencode(path), C.byref(nr))
        return nr.value

    # --- the routines those subroutines are built from ----------------
    def tube_construction(self, l: int):
        self._call("tube_construction", l)

    def ls_advection(self, l: int):
        self._call("ls_advection", l)

    def ls_mass_correction(self, istep: int, l: int):
        self._call("ls_mass_correction", istep, l)

    def ls_reinit_main(self, istep: int, l: int):
        self._call("ls_reinit_main", istep, l)

    def update_materials(self):
        self._call("update_materials")

    def get_curvature(self, l: int):
        self._call("get_curvature", l)

    def band_count(self, l: int) -> int:
        n = C.c_longlong()
        self._call("band_count", l, C.byref(n))
        return n.value

    # --- instrumentation (CUDA library only) ---------------------------
    def profile(self, on: bool = True):
        self._call("profile_enable", 1 if on else 0)

    def profile_reset(self):
        self._call("profile_reset")

    def profile_table(self) -> dict:
        n = C.c_int()
        self._call("profile_count", C.byref(n))
        out = {}
        buf = C.create_string_buffer(64)
        for i in range(n.value):
            ms, la, ti = C.c_double(), C.c_longlong(), C.c_longlong()
            self._call("profile_entry", i, buf, 64, C.byref(ms), C.byref(la), C.byref(ti))
            out[buf.value.decode()] = {"ms": ms.value, "launches": la.value, "timed": ti.value}
        return out

    def launch_count(self) -> int:
        n = C.c_longlong()
        self._call("launch_count", C.byref(n))
        return n.value

    def stream_ptr(self) -> int:
        s = C.c_void_p()
        self._call("get_stream", C.byref(s))
        return s.value or 0

    # --- convenience ---------------------------------------------------
    def setup(self, lvsets: np.ndarray, u=None, v=None, w=None, p=None):
        """Upload velocity, pressure and level sets, then init_program."""
        shp = field_shape(self.cfg, "u")
        z = np.zeros(shp, order="F")
        self.upload("u", z if u is None else u)
        self.upload("v", z if v is None else v)
        self.upload("w", z if w is None else w)
        self.upload("pnew", z if p is None else p)
        for l in range(self.cfg.lmax):
            self.upload("lvset", lvsets[..., l], l + 1)
        self.init_program()

    def interior(self, name: str, l: int = 1) -> np.ndarray:
        a = self.download(name, l)
        lo = field_lo(name)
        s = 1 - lo
        return a[s:s + self.cfg.itot, s:s + self.cfg.jtot, s:s + self.cfg.ktot]


def chkdiv_noalloc(u_ptr: int, v_ptr: int, w_ptr: int, imax: int, jmax: int, kmax: int,
                   dxi: float, dyi: float, dzi: float, result_ptr: int, stream: int = 0) -> int:
    """icls_chkdiv_noalloc on caller-owned device arrays (raw device
    addresses).  The library allocates nothing for this call; it returns the
    status code and leaves [divtot, divmax, i, j, k] in the 5-double device
    buffer at result_ptr."""
    lib = gpu_backend().lib
    fn = lib.icls_chkdiv_noalloc
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                   C.c_double, C.c_double, C.c_double, C.c_void_p, C.c_void_p]
    fn.restype = C.c_int
    return fn(u_ptr, v_ptr, w_ptr, imax, jmax, kmax, dxi, dyi, dzi, result_ptr, stream or None)


class Mlp:
    """The learned-curvature network (icls_mlp_* of the C ABI): 27-128-128-64-1
    SiLU MLP trained and evaluated on the GPU's tensor cores."""

    NPARAMS = 29057

    def __init__(self, seed: int = 2024):
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
            "icls_set_curvature_net": [P, P],
            "icls_curvature_stats": [P, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong), C.c_int],
        }
        for name, args in sig.items():
            getattr(lib, name).argtypes = args
            getattr(lib, name).restype = C.c_int
        self.lib = lib
        h = P()
        rc = lib.icls_mlp_create(C.byref(h), seed)
        if rc:
            raise IclsError(rc, "icls_mlp_create")
        self.h = h

    def _ok(self, rc, where):
        if rc:
            raise IclsError(rc, where)

    def make_data(self, seed: int, n_train: int, n_hold: int):
        self._ok(self.lib.icls_mlp_make_data(self.h, seed, n_train, n_hold), "icls_mlp_make_data")

    def train(self, epochs: int = 20, batch: int = 8192, lr: float = 1e-3, lr_final: float = 1e-5, seed: int = 5):
        losses = (C.c_double * epochs)()
        self._ok(self.lib.icls_mlp_train(self.h, epochs, batch, lr, lr_final, seed, losses), "icls_mlp_train")
        return list(losses)

    def evaluate(self) -> dict:
        st = (C.c_double * 8)()
        self._ok(self.lib.icls_mlp_eval(self.h, st), "icls_mlp_eval")
        keys = ("rms_mlp_label", "rms_mlp_analytic", "rms_plain_analytic", "rms_label_analytic",
                "max_mlp_analytic", "max_plain_analytic", "rms_analytic", "samples")
        return dict(zip(keys, list(st)))

    def params(self) -> np.ndarray:
        a = np.zeros(self.NPARAMS, dtype=np.float32)
        self._ok(self.lib.icls_mlp_params(self.h, a.ctypes.data_as(C.POINTER(C.c_float)), 1), "icls_mlp_params")
        return a

    def set_params(self, a):
        a = np.ascontiguousarray(a, dtype=np.float32)
        self._ok(self.lib.icls_mlp_params(self.h, a.ctypes.data_as(C.POINTER(C.c_float)), 0), "icls_mlp_params")

    def grad(self, x_ptr: int, label_ptr: int, n: int, scale: float):
        """gradient of the parameters for n FP32 samples [n][32] and labels
        (device addresses; n a power of two, at least 128, one 128-sample
        tile per block): dy = scale * (y - label) per sample; returns
        (gradient [NPARAMS], sum of squared errors)"""
        g = np.zeros(self.NPARAMS, dtype=np.float32)
        loss = C.c_double()
        self._ok(self.lib.icls_mlp_grad(self.h, x_ptr, label_ptr, n, scale, g.ctypes.data_as(C.POINTER(C.c_float)),
                                        C.byref(loss)), "icls_mlp_grad")
        return g, loss.value

    def attach(self, solver: "Solver"):
        """use this network for the solver's curvature (curvature_model MLP)"""
        self._ok(self.lib.icls_set_curvature_net(solver.h, self.h), "icls_set_curvature_net")
        solver._net = self

    def close(self):
        if getattr(self, "h", None):
            self.lib.icls_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def curvature_stats(solver: "Solver", reset: bool = False):
    """(cells the network evaluated, fallbacks to the stencil) of a solver"""
    lib = gpu_backend().lib
    fn = lib.icls_curvature_stats
    fn.argtypes = [C.c_void_p, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong), C.c_int]
    fn.restype = C.c_int
    e, f = C.c_longlong(), C.c_longlong()
    rc = fn(solver.h, C.byref(e), C.byref(f), 1 if reset else 0)
    if rc:
        raise IclsError(rc, "icls_curvature_stats")
    return e.value, f.value
