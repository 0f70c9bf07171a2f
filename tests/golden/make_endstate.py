"""Generates the end-state fixtures of the simple-spin scenario from the
compiled reference (oracle/_ref/ref_ftest: the reference's own fluid_2d::solve
and output writers, built with the clean-room TGMG shim):

  sspin_128_t2pi.npz   ftest simple-spin at 128 x 128 run to t = 2 pi with 120
                       frames (fluid_2d::solve(2 pi, 120); frame interval pi/60,
                       the coded solve(4 pi, 240)'s): frame 120 of w, p, phi,
                       X, Y and frames 12 and 60 of w and phi as written
                       (float32 gnuplot matrices, the solid fields cropped to
                       the solid's box + 2) and the whole track.dat.
  sspin_1024_f12.npz   the same scenario at 1024 x 1024 to frame 12 (t = pi/5,
                       about 1.65e4 steps): frame 12 of w, p, phi, X, Y,
                       block-averaged 4 x 4 (w, p) and 2 x 2 (the cropped
                       solid fields) to keep the fixture small, and
                       track.dat.

Each run takes the rel_tol of the solver from INCRMT_MG_RTOL (default 1e-9).
Usage, from the repository root after `make -C oracle`:
    python tests/golden/make_endstate.py 128 [<existing output dir>]
    python tests/golden/make_endstate.py 1024 [<existing output dir>]
An existing output directory (<base>.odr of a finished ref_ftest run) is read
instead of running the reference again (the 1024 run takes hours on the host).
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

OUT = os.path.dirname(os.path.abspath(__file__))
FIELDS = ("w", "p", "phi", "X", "Y")
# size: (duration, frames, {frame: fields kept}, block of w and p, block of
# the solid fields, fixture name)
CASES = {128: (2 * np.pi, 120, {12: ("w", "phi"), 60: ("w", "phi"), 120: FIELDS}, 1, 1, "sspin_128_t2pi.npz"),
         1024: (np.pi / 5, 12, {12: FIELDS}, 4, 2, "sspin_1024_f12.npz")}


def read_frame(path):
    """A gnuplot binary matrix: (coordinate row, coordinate column, values)."""
    a = np.fromfile(path, dtype=np.float32)
    si = int(a[0])
    a = a.reshape(-1, si + 1)
    return a[0, 1:].copy(), a[1:, 0].copy(), a[1:, 1:].copy()


def block_average(v, f):
    """Averages f x f blocks (float64); a ragged edge keeps its partial
    blocks, averaged over the cells they hold."""
    if f == 1:
        return v.astype(np.float64)
    ny, nx = v.shape
    by, bx = -(-ny // f), -(-nx // f)
    s = np.zeros((by, bx))
    c = np.zeros((by, bx))
    iy, ix = np.arange(ny) // f, np.arange(nx) // f
    np.add.at(s, (iy[:, None], ix[None, :]), v.astype(np.float64))
    np.add.at(c, (iy[:, None], ix[None, :]), 1.0)
    return s / c


def reduce_frame(path, f):
    x, y, v = read_frame(path)
    return block_average(x[None, :], f)[0], block_average(y[:, None], f)[:, 0], block_average(v, f)


def fixture(m, odr):
    T, frames, keep, fw, fs, name = CASES[m]
    d = {"m": m, "duration": T, "frames": frames, "block_w": fw, "block_solid": fs}
    for k, fields in keep.items():
        for f in fields:
            x, y, v = reduce_frame(os.path.join(odr, f"{f}.{k}"), fw if f in ("w", "p") else fs)
            d[f"{f}_{k}"] = v.astype(np.float32)
            d[f"{f}_{k}_x"] = x
            d[f"{f}_{k}_y"] = y
    d["track"] = np.fromfile(os.path.join(odr, "track.dat"), dtype=np.float64).reshape(-1, 4)
    np.savez_compressed(os.path.join(OUT, name), **d)
    return name


def run(m, workdir):
    from oracle import refsim
    if not refsim.available():
        refsim.build()
    T, frames = CASES[m][:2]
    base = os.path.join(workdir, f"sspin_{m}")
    subprocess.run([refsim.FTEST, str(m), repr(T), str(frames), base], check=True, cwd=workdir,
                   stdout=subprocess.DEVNULL)
    return base + ".odr"


if __name__ == "__main__":
    m = int(sys.argv[1])
    if len(sys.argv) > 2:
        print(fixture(m, sys.argv[2]))
    else:
        with tempfile.TemporaryDirectory() as td:
            print(fixture(m, run(m, td)))
