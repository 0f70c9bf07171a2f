"""The C++ host (incrmt_b200/host: fluid_2d and the object classes over the
C ABI, driven by ftest_gpu) against the reference's own ftest run and output
writers (oracle/_ref/ref_ftest: fluid_2d::solve, write_files, output,
output_tracers, obj_simple_spin::file_output; fluid_2d.cc:254-295,
fluid_2d_io.cc:13-179, object.cc:202-219).

Both runs write a simple-spin output directory at 64 x 64 for a short
duration; every file is compared:
  - header: identical text;
  - frames (gnuplot float32 matrices): identical shape, identical coordinate
    row and column (the cropped solid box is the same), values within 1e-6
    of the field's magnitude for p and w and 1e-6 for X, Y, phi (the state
    agrees to ~1e-9 after ~100 steps; the frames are float32), except phi of
    frame 0: the band built at initialisation differs from the reference's
    fast march at a few kinks by up to 0.015 dx (the march there accepts a
    point below an already accepted neighbour), so frame 0's phi is held to
    0.02 dx; the first pinning of the next step removes the difference;
  - trace.K: tracer positions seeded by the same C rand() sequence, 1e-6;
  - track.dat: same number of records; time exact, position and unwrapped
    angle 1e-8.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, oracle_available

pytestmark = pytest.mark.gpu

FTEST_GPU = os.path.join(ROOT, "incrmt_b200", "host", "ftest_gpu")


def _read_frame(path):
    a = np.fromfile(path, dtype=np.float32)
    si = int(a[0])
    a = a.reshape(-1, si + 1)
    return a


@pytest.fixture(scope="module")
def runs(tmp_path_factory, gpu):
    from oracle import refsim
    if not oracle_available() or not os.path.exists(refsim.FTEST):
        pytest.skip("oracle/_ref not built")
    assert os.path.exists(FTEST_GPU), "ftest_gpu not built (make -C incrmt_b200/host)"
    d = tmp_path_factory.mktemp("host")
    gdir, rdir = d / "gpu", d / "ref"
    gdir.mkdir()
    rdir.mkdir()
    dur, frames = "0.1", "2"
    g = subprocess.run([FTEST_GPU, "simple-spin", "64", "-d", dur, "-n", frames], cwd=gdir,
                       capture_output=True, text=True, timeout=600)
    assert g.returncode == 0, g.stderr
    r = subprocess.run([refsim.FTEST, "64", dur, frames, str(rdir / "sspin_64")], cwd=rdir,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return gdir / "sspin_64.odr", rdir / "sspin_64.odr", g.stdout, r.stdout


def test_same_files(runs):
    g, r, _, _ = runs
    assert sorted(os.listdir(g)) == sorted(os.listdir(r))


def test_header(runs):
    g, r, _, _ = runs
    assert (g / "header").read_text() == (r / "header").read_text()


@pytest.mark.parametrize("name", ["p", "w", "X", "Y", "phi"])
@pytest.mark.parametrize("k", [0, 1, 2])
def test_frames(runs, name, k):
    g, r, _, _ = runs
    a, b = _read_frame(g / f"{name}.{k}"), _read_frame(r / f"{name}.{k}")
    assert a.shape == b.shape
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[:, 0], b[:, 0])
    scale = max(float(np.abs(b[1:, 1:]).max()), 1.0) if name in ("p", "w") else 1.0
    err = float(np.abs(a[1:, 1:] - b[1:, 1:]).max()) / scale
    tol = 0.02 * (2.0 / 64) if (name, k) == ("phi", 0) else 1e-6
    assert err < tol, f"{name}.{k}: {err}"


@pytest.mark.parametrize("k", [0, 1, 2])
def test_tracers(runs, k):
    g, r, _, _ = runs
    a = np.fromfile(g / f"trace.{k}", dtype=np.float32)
    b = np.fromfile(r / f"trace.{k}", dtype=np.float32)
    assert a.shape == b.shape == (1024,)
    assert float(np.abs(a - b).max()) < 1e-6


def test_track(runs):
    g, r, _, _ = runs
    a = np.fromfile(g / "track.dat", dtype=np.float64).reshape(-1, 4)
    b = np.fromfile(r / "track.dat", dtype=np.float64).reshape(-1, 4)
    assert a.shape == b.shape
    np.testing.assert_array_equal(a[:, 0], b[:, 0])
    assert float(np.abs(a[:, 1:] - b[:, 1:]).max()) < 1e-8


def test_stdout_frames(runs):
    _, _, gout, rout = runs
    gl = [l.split("[")[0] for l in gout.splitlines() if l.startswith("# Output frame")]
    rl = [l.split("[")[0] for l in rout.splitlines() if l.startswith("# Output frame")]
    assert gl == rl
    assert "# Non-constant density" in gout
