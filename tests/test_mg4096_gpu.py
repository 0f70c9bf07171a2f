"""The benchmark's standalone 4096 x 4096 MAC solve against the oracle's
solution of the same system (tests/golden/mg_mac_4096.npz, written by
tests/golden/make_mg4096.py: the reference's MAC callbacks with the
clean-room TGMG shim, from zero to a 1e-9 relative residual).

The GPU solves the same seeded system in FP64 from zero to the same
tolerance. Both solutions meet the residual bound; the pure-Neumann system
fixes them only up to a constant, so both are compared with their means
removed, on the fixture's 16 x 16 block averages and its three full rows and
columns: within 1e-8 of the largest |value| (rounding differences only, the
bound of the smaller FP64 parity cases in test_mg_gpu.py), and the V-cycle
counts within one. Mixed precision meets the same residual, within 1e-6.
"""
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(GOLDEN, "mg_mac_4096.npz")
sys.path.insert(0, GOLDEN)


@pytest.mark.skipif(not os.path.exists(FIXTURE), reason="the 4096 x 4096 fixture has not been generated")
@pytest.mark.parametrize("prec,tol", [(0, 1e-8), (1, 1e-6)])
def test_mac4096_matches_oracle(gpu, prec, tol):
    from incrmt_b200 import capi, workloads
    from make_mg4096 import M, reduce
    g = np.load(FIXTURE)
    rho, b = workloads.standalone_mac_problem(M)
    s = capi.MGSolver(capi.SYS_MAC, M, M)
    s.set_density(rho.numpy())
    z = np.zeros(M * M)
    st = s.solve(b.numpy().ravel(), z, rel_tol=1e-9, precision=prec)
    s.close()
    assert st.rel_res <= 1e-9
    d = reduce(z.reshape(M, M))
    scale = max(np.abs(g[k]).max() for k in ("blocks", "rows", "cols"))
    for key in ("blocks", "rows", "cols"):
        err = np.abs(d[key] - g[key]).max() / scale
        assert err <= tol, (key, err)
    if prec == 0:
        assert abs(st.vcycles - int(g["vcycles"])) <= 1, (st.vcycles, int(g["vcycles"]))
