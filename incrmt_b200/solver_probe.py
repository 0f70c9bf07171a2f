"""Timing probe of one pressure solver (include/incrmt.h), for profiling the
multigrid kernels on a chosen grid without a simulation around it.

    python -m incrmt_b200.solver_probe --sys 0 --m 3456 --n 1152 \
        --box -1 5 -1 1 --y-prd --zpr --vcycles 2

builds the solver, sets a seeded density (8 circles, rho 3, blended as
fluid_2d::set_rho does), runs --vcycles V-cycles on a seeded right-hand side
from zero, then the same number again with the fine-level smoothing launches
timed by CUDA events, and prints their count, mean duration and algorithmic
bandwidth.
"""
import argparse

import numpy as np
import torch

from . import capi, workloads


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--sys", type=int, default=capi.SYS_MAC, choices=[capi.SYS_MAC, capi.SYS_FEM])
    ap.add_argument("--m", type=int, default=1024)
    ap.add_argument("--n", type=int, default=1024)
    ap.add_argument("--box", type=float, nargs=4, default=[-1.0, 1.0, -1.0, 1.0])
    ap.add_argument("--x-prd", action="store_true")
    ap.add_argument("--y-prd", action="store_true")
    ap.add_argument("--zpr", action="store_true")
    ap.add_argument("--vcycles", type=int, default=2)
    ap.add_argument("--no-tiles", action="store_true", help="one launch per colour")
    a = ap.parse_args()
    box = tuple(a.box)
    s = capi.MGSolver(a.sys, a.m, a.n, *box, x_prd=a.x_prd, y_prd=a.y_prd, zpr=a.zpr)
    if a.no_tiles:
        s.set_tiles(False)
    circ = workloads.circles(seed=3, count=8, rmin=0.05, rmax=0.2, box=box)
    s.set_density(workloads.circle_density(a.m, a.n, circ, box=box).numpy())
    N = s.m_sys * s.n_sys
    rng = np.random.default_rng(0)
    b = torch.tensor(rng.standard_normal(N), device="cuda")
    z = torch.zeros(N, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    for _ in range(a.vcycles):
        s.vcycle_device(b.data_ptr(), z.data_ptr())
    torch.cuda.synchronize()
    s.set_profiling(True)
    for _ in range(a.vcycles):
        s.vcycle_device(b.data_ptr(), z.data_ptr())
    torch.cuda.synchronize()
    ms, by, nl = s.profile()
    print(f"fine-level smoothing: {nl} launches, {1000 * ms / max(nl, 1):.1f} us each, "
          f"{by / (ms / 1e3) / 1e9 if ms > 0 else 0:.0f} GB/s algorithmic")
    s.close()


if __name__ == "__main__":
    main()
