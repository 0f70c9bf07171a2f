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


def sspin_cases():
    """Simple-spin end states after a few steps from the scenario's own
    initialisation (ftest.cc:116-143), interior cells only."""
    out = []
    for m, steps in [(64, 20), (128, 50)]:
        r = refsim.RefSim(m, ntrace=16)
        tr0 = r.tracers()[:, :2].copy()
        dt, _ = refsim.frame_dt(r.scalars()["dt_reg"])
        r.step(dt, steps)
        d = {f: r.get(f)[2:-2, 2:-2] for f in ["u", "v", "p", "X", "Y", "phi"]}
        d["tracers0"] = tr0
        d["tracers"] = r.tracers()[:, :2]
        d["objtr"] = r.obj_tracers()[:, :2]
        name = f"sspin_{m}_{steps}.npz"
        np.savez_compressed(os.path.join(OUT, name), **d)
        r.close()
        out.append(name)
    return out


if __name__ == "__main__":
    for name, st in mg_cases():
        print(name, st)
    for name in sspin_cases():
        print(name)
