"""Generates tests/golden/mg_mac_4096.npz: the oracle's solution of the
standalone 4096 x 4096 MAC system (workloads.standalone_mac_problem(4096),
seed 3, the benchmark's problem; walls, no zero-pressure column) solved to a
1e-9 relative residual by the oracle (the reference's MAC callbacks,
mgs_mac.hh:64-102, with the clean-room TGMG shim), from zero.

The full solution (134 MB) is not kept: the fixture holds its 16 x 16 block
averages (256 x 256), rows 0, 2047 and 4095 and columns 0, 2048 and 4095 at
full resolution, the mean, and the V-cycle count. The system is pure
Neumann, so every array is stored with the solution's mean removed.

Usage, from the repository root after `make -C oracle` (about half a minute
on eight host threads): python tests/golden/make_mg4096.py
"""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "mg_mac_4096.npz")
M = 4096
ROWS = (0, 2047, 4095)
COLS = (0, 2048, 4095)


def reduce(z):
    """The fixture's view of a solution z (M x M, any gauge)."""
    z = z - z.mean()
    return {"blocks": z.reshape(M // 16, 16, M // 16, 16).mean(axis=(1, 3)),
            "rows": np.stack([z[r] for r in ROWS]), "cols": np.stack([z[:, c] for c in COLS])}


def main():
    from incrmt_b200 import workloads
    from oracle import refsim
    rho, b = workloads.standalone_mac_problem(M)
    rho, b = rho.numpy(), b.numpy().ravel()
    t0 = time.perf_counter()
    z, _, st = refsim.mg_solve(0, M, M, rho, b)
    secs = time.perf_counter() - t0
    d = reduce(z.reshape(M, M))
    np.savez_compressed(OUT, m=M, vcycles=int(st[0]), oracle_seconds=secs, rows_at=np.array(ROWS),
                        cols_at=np.array(COLS), **d)
    print(f"{OUT}: {int(st[0])} V-cycles, {secs:.1f} s")


if __name__ == "__main__":
    main()
