"""The tile-fused smoothers (two Gauss-Seidel sweeps per launch in
shared-memory tiles) against one launch per colour (incrmt_mg_set_tiles):
identical iterates, bit for bit, after three FP64 V-cycles and after a whole
mixed-precision solve, on grids of several launch waves (where blocks that
start late would see their neighbours' finished tiles if the sweeps worked
in place) and with periodic directions (whose halos hold periodic images).
The density is set again after each switch, so the Galerkin coarse operators
are rebuilt by the tiled kernel (shared-memory staging) and by the
one-thread-per-unknown kernel, and must agree bit for bit as well.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [
    # sys, m, n, x_prd, y_prd, zpr, whole solve (the doubly periodic system is
    # singular with a periodic null space: V-cycles only)
    (0, 1024, 1024, False, False, False, True),
    (1, 1024, 1024, False, False, False, True),
    (0, 768, 512, False, True, True, True),
    (1, 768, 512, False, True, True, True),
    (0, 512, 384, True, True, False, False),
    # large enough for the 64 x 32 tiles of the fine levels (at least two
    # blocks per SM), with periodic seams and the zero-pressure column
    (0, 1024, 1024, False, True, True, True),
    (1, 1024, 1024, False, True, True, True),
    (0, 1024, 768, True, True, False, False),
    (1, 1024, 768, True, True, False, False),
]


@pytest.mark.parametrize("sys_,m,n,xp,yp,zpr,solve", CASES)
def test_tiles_identical_to_colour_launches(gpu, sys_, m, n, xp, yp, zpr, solve):
    import torch
    from incrmt_b200 import capi, workloads
    s = capi.MGSolver(sys_, m, n, x_prd=xp, y_prd=yp, zpr=zpr)
    circ = workloads.circles(seed=m + n, count=8, rmin=0.05, rmax=0.2)
    rho = workloads.circle_density(m, n, circ).numpy()
    s.set_density(rho)
    rng = np.random.default_rng(m * 7 + n)
    N = s.m_sys * s.n_sys
    b = rng.standard_normal(N)
    b -= b.mean()
    z0 = rng.standard_normal(N)
    dev = torch.device("cuda")
    bd = torch.tensor(b, device=dev)
    out = {}
    for tiles in (True, False):
        s.set_tiles(tiles)
        s.set_density(rho)
        z = torch.tensor(z0, device=dev)
        torch.cuda.synchronize()
        for _ in range(3):
            s.vcycle_device(bd.data_ptr(), z.data_ptr())
        torch.cuda.synchronize()
        zm = torch.zeros(N, dtype=torch.float64, device=dev)
        vc = 0
        if solve:
            vc = s.solve_device(bd.data_ptr(), zm.data_ptr(), precision=capi.PREC_MIXED).vcycles
        torch.cuda.synchronize()
        out[tiles] = (z.cpu().numpy(), zm.cpu().numpy(), vc)
    assert np.array_equal(out[True][0], out[False][0])
    assert out[True][2] == out[False][2]
    assert np.array_equal(out[True][1], out[False][1])
    s.close()
