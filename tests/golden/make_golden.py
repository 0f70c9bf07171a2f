"""Generates the golden fixtures in tests/golden from the compiled reference
(oracle/_ref: the reference's own sources built with the clean-room TGMG
shim). Run from the repository root after `make -C oracle`:
    python tests/golden/make_golden.py
The GPU parity tests use these when oracle/_ref is not present.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from incrmt_b200 import workloads  # noqa: E402
from oracle import refsim  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def mg_cases():
    cases = []
    for sys_, m, zpr in [(0, 64, False), (1, 64, False), (1, 64, True)]:
        if sys_ == 0:
            rho, b = workloads.standalone_mac_problem(m)
        else:
            rho, b = workloads.standalone_fem_problem(m)
        rho, b = rho.numpy(), b.numpy().ravel()
        z, bu, st = refsim.mg_solve(sys_, m, m, rho, b, zpr=zpr)
        name = f"mg_{'mac' if sys_ == 0 else 'fem'}_{m}{'_zpr' if zpr else ''}.npz"
        np.savez_compressed(os.path.join(OUT, name), rho=rho, b=b, b_used=bu, z=z,
                            vcycles=st[0], rel_res=st[1], sys=sys_, m=m, zpr=int(zpr))
        cases.append((name, st))
    return cases


if __name__ == "__main__":
    for name, st in mg_cases():
        print(name, st)
