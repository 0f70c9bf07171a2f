"""The allocation-free operator application (incrmt_mg_apply_noalloc).

Callers that cannot allocate device memory (a framework arena that forbids
cudaMalloc, a real-time loop) get A z from device pointers, with the library's
fixed scratch array instead of a solver handle's buffers. The result must
match the handle-based incrmt_mg_apply within the operator tolerance of the
other tests (1e-12 relative), on two calls in a row (the second call reuses
the scratch the first one left behind). Grids above the 256 x 256 limit are
rejected with a clear error. This file is collected last on purpose.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("sys_,zpr,m,n", [(0, False, 48, 40), (0, True, 256, 256),
                                          (1, False, 64, 48), (1, True, 256, 200)])
def test_noalloc_apply_matches_handle_apply(gpu, sys_, zpr, m, n):
    import torch
    from incrmt_b200 import capi
    rng = np.random.default_rng(7 + m + n)
    rho = 1 + 2 * rng.random((n + 4, m + 4))
    h = capi.MGSolver(sys_, m, n, zpr=zpr)
    h.set_density(rho)
    dev = torch.device("cuda", 0)
    d_rho = torch.from_numpy(rho).to(dev)
    for call in range(2):
        z = rng.standard_normal(h.m_sys * h.n_sys)
        ref = h.apply(z)
        d_z = torch.from_numpy(z).to(dev)
        d_out = torch.full_like(d_z, float("nan"))
        torch.cuda.synchronize()
        capi.mg_apply_noalloc(sys_, m, n, d_rho.data_ptr(), d_z.data_ptr(), d_out.data_ptr(), zpr=zpr,
                              stream=torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        out = d_out.cpu().numpy()
        assert np.abs(out - ref).max() <= 1e-12 * np.abs(ref).max(), (call, np.abs(out - ref).max())
    h.close()


def test_noalloc_rejects_oversized_grid(gpu):
    import torch
    from incrmt_b200 import capi
    dev = torch.device("cuda", 0)
    buf = torch.zeros(4, dtype=torch.float64, device=dev)
    with pytest.raises(capi.IncrmtError) as e:
        capi.mg_apply_noalloc(0, 257, 64, buf.data_ptr(), buf.data_ptr(), buf.data_ptr())
    assert e.value.code == capi.ERR_BADARG
    assert "exceeds" in str(e.value)
