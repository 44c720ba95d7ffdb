"""Generates the golden fixtures of tests/golden/ (run from the repo root).

  fft_vfftpack.npz   seeded input rows and the VRFFTF output defined by the
                     reference's fft.f:1123-1142 (half-complex layout,
                     sqrt(1/N) scaling), evaluated by direct O(N^2) sums in
                     numpy -- independent of the oracle's FFT.
  oracle_static16.json  a regression record of the CPU oracle on a 16^3
                     static drop (3 steps): norms and probe values.

The reference itself cannot be built in this image (no Fortran compiler,
MPI or LAPACK), so the FFT vectors come from the transform's documented
definition and the oracle record pins the restatement against drift.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "icls-release_b200"))


def vrfftf_direct(x):
    """VRFFTF of one row by its definition (fft.f:1123-1142)."""
    n = x.size
    j = np.arange(n)
    s = np.sqrt(1.0 / n)
    out = np.zeros(n)
    out[0] = s * x.sum()
    for k in range(1, (n + 1) // 2):
        out[2 * k - 1] = s * np.sum(x * np.cos(2.0 * np.pi * j * k / n))
        out[2 * k] = -s * np.sum(x * np.sin(2.0 * np.pi * j * k / n))
    if n % 2 == 0:
        out[n - 1] = s * np.sum(x * (-1.0) ** j)
    return out


def make_fft():
    rng = np.random.default_rng(12345)
    data = {}
    for n in (8, 16, 64, 256):
        x = rng.standard_normal((3, n))
        data["x%d" % n] = x
        data["f%d" % n] = np.stack([vrfftf_direct(r) for r in x])
    np.savez(os.path.join(HERE, "fft_vfftpack.npz"), **data)


def make_oracle_record():
    from oracle.oracle import Oracle, set_threads
    from icls_gpu import init_drops, initial_velocity, static_drop
    set_threads(1)
    wl = static_drop(16, steps=3)
    o = Oracle(wl.cfg)
    o.setup(init_drops(wl.cfg, wl.centres, wl.radii), *initial_velocity(wl.cfg, 0.0))
    for s in range(1, 4):
        o.step(s, 0)
    rec = {"config": "static_drop_16", "steps": 3}
    for name in ("lvset", "u", "v", "w", "pnew"):
        a = o.download(name)
        rec[name + "_l2"] = float(np.linalg.norm(a.ravel()))
        rec[name + "_probe"] = float(a[8, 8, 8])
    rec["volume"] = float(o.volumes()[0][0])
    with open(os.path.join(HERE, "oracle_static16.json"), "w") as f:
        json.dump(rec, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    make_fft()
    make_oracle_record()
    print("golden fixtures written to", HERE)
