"""Host-side output of the reference driver, single process:

* post2d (output.f90:179-432): the mid-yz plane file ``yz_mid%07d.dat``;
* the ``timestep.txt`` record (main.f90:243-256).

The device work is a plane gather (``icls_download_plane_x``) and the
record's reductions (``icls_timestep_record``); this module only formats
and writes, with the reference's Fortran edit descriptors.
"""
from __future__ import annotations

import os

import numpy as np


def fortran_e(x: float, w: int = 15, d: int = 7) -> str:
    """Fortran ``Ew.d``: 0.ddddddd E+xx, right-aligned in w columns."""
    x = float(x)
    if x == 0.0:
        body = "0." + "0" * d + "E+00"
        return body.rjust(w)
    s = "{:.{p}E}".format(abs(x), p=d - 1)      # d significant digits
    mant, exp = s.split("E")
    digits = mant.replace(".", "")
    e = int(exp) + 1
    body = "0." + digits + "E" + ("+" if e >= 0 else "-") + "{:02d}".format(abs(e))
    if x < 0:
        body = "-" + body
    return body.rjust(w)


def fortran_es(x: float, w: int = 16, d: int = 8) -> str:
    """Fortran ``ESw.d``: d.dddddddd E+xx, right-aligned in w columns."""
    return "{:{w}.{d}E}".format(float(x), w=w, d=d)


def append_timestep(path: str, rec) -> None:
    """One line of timestep.txt, format (6ES16.8) (main.f90:253-255)."""
    with open(path, "a") as f:
        f.write("".join(fortran_es(v) for v in rec) + "\n")


def post2d(solver, istep: int, datadir: str = ".") -> str:
    """Write the mid-yz plane (i = itot/2) as output.f90:179-432 does on one
    process: y, z, u averaged to the cell centre in x, v and w averaged to
    the cell centre in y and z (v periodic in y, w = 0 below k = 1), p, the
    first level set, jiemian and fixhv (the static Heaviside of riblets,
    zero without them).  Returns the file path."""
    cfg = solver.cfg
    jtot, kmax = cfg.jtot, cfg.ktot
    dyi, dzi = jtot / cfg.ly, kmax / cfg.lz
    iloc = cfg.itot // 2
    # planes over the C bounds (0:j1, 0:k1); L planes over (-2:j1+2, -2:k1+2)
    u0 = solver.download_plane_x("u", iloc)
    um = solver.download_plane_x("u", iloc - 1)
    v = solver.download_plane_x("v", iloc)
    w = solver.download_plane_x("w", iloc)
    p = solver.download_plane_x("pnew", iloc)
    ls = solver.download_plane_x("lvset", iloc, 1)[2:-2, 2:-2]
    jm = solver.download_plane_x("jiemian", iloc)
    path = os.path.join(datadir, "yz_mid%07d.dat" % istep)
    with open(path, "w") as f:
        f.write(' VARIABLES = "y","z","u","v","w","p","s","indie","fixhv"\n')
        f.write(' ZONE T="Zone1" I=%12d J=%12d , F=POINT\n' % (jtot, kmax))
        for k in range(1, kmax + 1):
            for j in range(1, jtot + 1):
                jmm = j - 1 if j > 1 else jtot
                w_km = w[j, k - 1] if k > 1 else 0.0
                row = ((j - 0.5) / dyi, (k - 0.5) / dzi,
                       0.5 * (u0[j, k] + um[j, k]),
                       0.5 * (v[j, k] + v[jmm, k]),
                       0.5 * (w[j, k] + w_km),
                       p[j, k], ls[j, k], jm[j, k], 0.0)
                f.write("".join(fortran_e(x) for x in row) + "\n")
    return path
