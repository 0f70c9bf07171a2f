"""Grid convergence on the GPU (conv_test's study, conv_test.cc:95-194, with
fluid_2d::l_comparison on the GPU): conv_test type 4 (a circle of density 3
in sim_velocity_pulses) at 128^2, 64^2 and 32^2, stepped together over five
intervals of 0.02 with the test's time steps and padding.

- the velocity and pressure errors against the finest grid shrink with
  resolution (32^2 worse than 64^2, in L1, L2 and max);
- mixed precision (FP32 V-cycles in FP64 defect correction) gives the same
  errors as FP64 to 1e-6 relative: its projections reach the same 1e-9
  residual, so the discretisation error is unchanged;
- the conv_test_gpu driver writes cnv_<type>.dat in the reference's layout
  (per interval: index, time, then 32 norms per coarser grid).
"""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RES = (128, 64, 32)
HOST = os.path.join(os.path.dirname(__file__), os.pardir, "incrmt_b200", "host")


def _study(precision, intervals=5):
    from incrmt_b200 import capi
    sims, steps = [], []
    for m in RES:
        s = capi.Simulation(m, m, visc=1e-3, ntrace=0, x_prd=True, y_prd=True, pulses=True, precision=precision)
        s.add_circle(-0.1, 0.0, 0.6, 1.0, 3.0, set_velocity=False)
        dt_reg = s.initialize(0.4, 0.4 * RES[-1] / m, 0.8 * RES[-1] / m)
        l = int(0.02 / dt_reg) + 1
        sims.append(s)
        steps.append((0.02 / l, l))
    for _ in range(intervals):
        for s, (dt, l) in zip(sims, steps):
            s.step(dt, l)
    errs = [s.l_comparison(sims[0]) for s in sims[1:]]
    for s in sims:
        s.close()
    return np.array(errs)


def test_errors_shrink_and_mixed_matches(gpu):
    from incrmt_b200 import capi
    e64 = _study(capi.PREC_FP64)
    # norms: 8..11 velocity L2, 12..15 pressure L2, 16..19 velocity L1,
    # 20..23 pressure L1, 24..27 velocity max, 28..31 pressure max (totals at +3)
    for col in (11, 15, 19, 23, 27, 31):
        assert e64[1, col] > e64[0, col] > 0, (col, e64[:, col])
    emx = _study(capi.PREC_MIXED)
    for col in (11, 15, 19, 23, 27, 31):
        assert np.allclose(emx[:, col], e64[:, col], rtol=1e-6, atol=0), (col, emx[:, col], e64[:, col])


def test_driver_output(gpu, tmp_path):
    exe = os.path.abspath(os.path.join(HOST, "conv_test_gpu"))
    r = subprocess.run([exe, "4", "-res", "64,32", "-n", "2"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = (tmp_path / "cnv_04.dat").read_text().strip().split("\n")
    assert len(lines) == 3
    for i, line in enumerate(lines):
        v = [float(x) for x in line.split()]
        assert len(v) == 2 + 32 and v[0] == i and abs(v[1] - 0.02 * i) < 1e-12
        assert all(np.isfinite(v))
    assert (tmp_path / "cnv_04_1.odr").is_dir()


def test_driver_full_solid(gpu, tmp_path):
    """Type 2: the full solid with periodic reference maps (conv_test.cc:78-80,
    116-120) runs and writes finite norms, X and Y among the frames."""
    exe = os.path.abspath(os.path.join(HOST, "conv_test_gpu"))
    r = subprocess.run([exe, "2", "-res", "64,32", "-n", "2"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = (tmp_path / "cnv_02.dat").read_text().strip().split("\n")
    assert len(lines) == 3
    for line in lines:
        v = [float(x) for x in line.split()]
        assert len(v) == 2 + 32 and all(np.isfinite(v))
    names = os.listdir(tmp_path / "cnv_02_1.odr")
    assert any(f.startswith("X.") for f in names) and any(f.startswith("Y.") for f in names)
