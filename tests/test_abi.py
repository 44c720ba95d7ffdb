"""The C ABI without a GPU: the library loads, exports every entry point that
include/icls_gpu.h declares, and rejects bad arguments and configurations on
the host before any CUDA call (the validation the reference does at start-up
in param.f90 / initsolver.f90 becomes status codes here)."""
import ctypes as C
import os
import re

import pytest

from conftest import ROOT
from icls_gpu.binding import LIB_PATH
from icls_gpu.config import IclsConfig, STATUS_NAMES, make_config

HEADER = os.path.join(ROOT, "include", "icls_gpu.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|void)\s+(icls_\w+)\s*\(", text, flags=re.M)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB_PATH):
        pytest.fail("%s missing: run python __graft_entry__.py build" % LIB_PATH)
    return C.CDLL(LIB_PATH)


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 40, names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings(lib):
    f = lib.icls_status_string
    f.argtypes = [C.c_int, C.c_char_p, C.c_int]
    f.restype = C.c_int
    buf = C.create_string_buffer(96)
    seen = set()
    for code in sorted(STATUS_NAMES):
        assert f(code, buf, 96) == 0
        assert buf.value, code
        seen.add(buf.value)
    assert len(seen) == len(STATUS_NAMES)
    assert f(12345, buf, 96) == 0 and buf.value == b"unknown status"


def test_config_default_matches_python_defaults(lib):
    c = IclsConfig()
    lib.icls_config_default.argtypes = [C.POINTER(IclsConfig)]
    lib.icls_config_default.restype = None
    lib.icls_config_default(C.byref(c))
    ref = make_config()
    for name, _ in IclsConfig._fields_:
        a, b = getattr(c, name), getattr(ref, name)
        if hasattr(a, "__len__"):
            assert list(a) == list(b), name
        else:
            assert a == b, name


def test_config_layout_matches_header(tmp_path):
    """The ctypes mirror of icls_config has the header's size and offsets
    (a C program built against include/icls_gpu.h prints them)."""
    import shutil
    import subprocess
    if not shutil.which("gcc"):
        pytest.skip("no C compiler")
    names = [n for n, _ in IclsConfig._fields_]
    src = tmp_path / "layout.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "%s"\nint main(void) {\n'
                   '  printf("%%zu\\n", sizeof(icls_config));\n%s  return 0;\n}\n'
                   % (HEADER, "".join('  printf("%%zu\\n", offsetof(icls_config, %s));\n' % n for n in names)))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-o", str(exe), str(src)], check=True)
    out = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    assert out[0] == C.sizeof(IclsConfig)
    assert out[1:] == [getattr(IclsConfig, n).offset for n in names]


@pytest.mark.parametrize("change,code", [
    (dict(itot=24), "E_CONFIG"),            # radix-2 FFT in x
    (dict(jtot=40), "E_CONFIG"),               # no FFT of that length
    (dict(itot=40), "E_CONFIG"),
    (dict(jtot=100), "E_CONFIG"),
    (dict(itot=8, jtot=384), "E_CONFIG"),      # 384-point y lines tile at least 16 columns            # radix-2 FFT in y
    (dict(itot=8192), "E_CONFIG"),
    (dict(ktot=4), "E_CONFIG"),
    (dict(lmax=0), "E_CONFIG"),
    (dict(lx=0.0), "E_CONFIG"),
    (dict(timestep=-1e-4), "E_CONFIG"),
    (dict(reinit_step=0), "E_CONFIG"),
    (dict(ls_adv_space=7), "E_CONFIG"),
    (dict(precision=5), "E_CONFIG"),        # neither ICLS_FP64 nor ICLS_FP32
    (dict(curvature_model=2), "E_CONFIG"),      # neither stencil nor network
    (dict(curvature_model=1, lx=2.0), "E_UNSUPPORTED"),  # the network needs isotropic spacing
    (dict(curvature_model=1, mlp_fallback_tol=0.0), "E_CONFIG"),
    (dict(mass_threshold=-1e-6), "E_CONFIG"),
    (dict(mass_gain_one=2), "E_CONFIG"),
])
def test_create_rejects_bad_configs_on_host(lib, change, code):
    cfg = make_config(itot=32, jtot=32, ktot=32, lmax=1)
    for k, v in change.items():
        setattr(cfg, k, v)
    lib.icls_create.argtypes = [C.POINTER(IclsConfig), C.POINTER(C.c_void_p)]
    lib.icls_create.restype = C.c_int
    h = C.c_void_p(1)
    rc = lib.icls_create(C.byref(cfg), C.byref(h))
    assert STATUS_NAMES.get(rc) == code, (change, rc)
    assert not h.value
    assert STATUS_NAMES.get(lib.icls_create(None, C.byref(h))) == "E_ARG"


@pytest.mark.parametrize("ni,nj", [(48, 48), (96, 32), (32, 96), (384, 16), (16, 384), (192, 64), (8, 4096)])
def test_create_accepts_fft_lengths(lib, ni, nj):
    """lengths with a transform pass the configuration check (without a GPU
    the allocation that follows fails instead)"""
    cfg = make_config(itot=ni, jtot=nj, ktot=8, lmax=1)
    lib.icls_create.argtypes = [C.POINTER(IclsConfig), C.POINTER(C.c_void_p)]
    lib.icls_create.restype = C.c_int
    h = C.c_void_p()
    rc = lib.icls_create(C.byref(cfg), C.byref(h))
    if rc == 0:
        lib.icls_destroy(h)
    assert STATUS_NAMES.get(rc) != "E_CONFIG", (ni, nj, rc)


def test_null_context_is_an_argument_error(lib):
    for name in ("icls_init_program", "icls_ab2", "icls_fillps", "icls_gfm4p", "icls_solver2d",
                 "icls_correc", "icls_update_materials", "icls_synchronize"):
        fn = getattr(lib, name)
        fn.argtypes = [C.c_void_p]
        fn.restype = C.c_int
        assert STATUS_NAMES.get(fn(None)) == "E_ARG", name


def test_noalloc_argument_checks_run_before_cuda(lib):
    fn = lib.icls_chkdiv_noalloc
    fn.argtypes = [C.c_void_p] * 3 + [C.c_int] * 3 + [C.c_double] * 3 + [C.c_void_p, C.c_void_p]
    fn.restype = C.c_int
    dummy = 0x1000  # never dereferenced: both checks return before any CUDA call
    assert STATUS_NAMES.get(fn(None, dummy, dummy, 8, 8, 8, 1., 1., 1., dummy, None)) == "E_ARG"
    assert STATUS_NAMES.get(fn(dummy, dummy, dummy, 0, 8, 8, 1., 1., 1., dummy, None)) == "E_ARG"
    assert STATUS_NAMES.get(fn(dummy, dummy, dummy, 2048, 2048, 2048, 1., 1., 1., dummy, None)) == "E_SIZE"
    # the limit itself: 2^31 cells (one above ICLS_NOALLOC_MAX_CELLS) is refused on the host
    assert 2048 * 1024 * 1024 == 2**31
    assert STATUS_NAMES.get(fn(dummy, dummy, dummy, 2048, 1024, 1024, 1., 1., 1., dummy, None)) == "E_SIZE"


def test_config_beyond_32bit_indexing_is_rejected(lib):
    """A grid whose level set with halos exceeds 2^30 elements is refused by
    icls_create before any allocation (the kernels' 32-bit grid-stride
    loops stay below INT_MAX); one just inside the limit passes validation."""
    lib.icls_create.argtypes = [C.POINTER(IclsConfig), C.POINTER(C.c_void_p)]
    lib.icls_create.restype = C.c_int
    h = C.c_void_p()
    cfg = make_config(itot=1024, jtot=1024, ktot=1024, lmax=1)  # 1030^3 > 2^30
    assert STATUS_NAMES.get(lib.icls_create(C.byref(cfg), C.byref(h))) == "E_CONFIG"
    cfg = make_config(itot=1024, jtot=1024, ktot=8, lmax=1)
    rc = lib.icls_create(C.byref(cfg), C.byref(h))
    if rc == 0:
        lib.icls_destroy(h)
    assert STATUS_NAMES.get(rc) != "E_CONFIG"
