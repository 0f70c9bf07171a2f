"""The learned warm start inside the simulation's projections
(incrmt_sim_set_learned, incrmt_sim_learned_capture; include/incrmt_unet.h).

- capture: a captured sample's target is exactly the block average of the
  projection's solution minus its warm start (to float rounding), and the
  input's third channel is zero;
- training on the simulation's own samples lowers the loss;
- with the guess on, every projection counts as applied, fallen back or
  skipped (after eight rejections in a row the next 32 projections skip the
  guess), every projection still converges to the same 1e-9 residual, and after 10
  steps the fields agree with the plain run to 1e-6 of their maximum (the
  two runs differ only in where each solve stopped within its tolerance);
- under the residual rule (0) a guess is applied only if it does not raise
  the residual, so rule 0 never applies more guesses than rule 1.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SED_BOX = (-0.75, 0.75, -1.5, 1.5)
M, FACTOR = 128, 4


def _sim(seed=5):
    from incrmt_b200 import capi, workloads
    ax, bx, ay, by = SED_BOX
    sim = capi.Simulation(M, 2 * M, ax=ax, bx=bx, ay=ay, by=by, visc=2e-3, ntrace=0)
    for o in workloads.sediment_bodies(seed=seed, count=8):
        if o["kind"] == "circle":
            sim.add_circle(o["cx"], o["cy"], o["r"], 1.0, o["rhos"], grav=o["grav"])
        else:
            sim.add_ellipse(o["cx"], o["cy"], o["r"], o["b"], o["theta"], 1.0, o["rhos"], grav=o["grav"])
    dt = sim.initialize()
    return sim, dt


def _rel(a, b):
    # a non-finite value where the other array is finite fails the comparison
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    fa, fb = np.isfinite(a), np.isfinite(b)
    if not np.array_equal(fa, fb):
        return float("inf")
    if not fb.any():
        return 0.0
    d = np.abs(a[fb] - b[fb])
    s = np.abs(b[fb]).max()
    return float(d.max() / (s if s > 0 else 1.0))


def test_capture_target_is_the_correction(gpu):
    import torch
    from incrmt_b200 import capi
    sim, dt = _sim()
    sim.step(dt, 3)
    dev = torch.device("cuda")
    before = {capi.SYS_MAC: ["normal_derivatives_velocity", "godunov_tang", "tangential_derivatives",
                             "half_time_edge_velocities", "godunov"],
              capi.SYS_FEM: ["update_reference_map", "pin", "set_boundaries", "compute_stress", "compute_ustar"]}
    for sys, stage, (m, n) in [(capi.SYS_MAC, "mac_projection", (M, 2 * M)),
                               (capi.SYS_FEM, "finite_element_projection", (M + 1, 2 * M + 1))]:
        # the step's stages in order up to the projection; its warm start is
        # the previous step's solution
        for st in before[sys]:
            sim.stage(st, dt)
        H, W = sim.learned_grid(sys, FACTOR)
        X = torch.zeros(1, H, W, 3, device=dev)
        T = torch.zeros(1, H, W, device=dev)
        z0 = sim.get_mg(sys).reshape(n, m)
        torch.cuda.synchronize()
        sim.learned_capture(sys, FACTOR, X.data_ptr(), T.data_ptr(), 1)
        sim.stage(stage, dt)
        assert sim.learned_stats(sys).captured == 1
        sim.learned_capture(sys, FACTOR, 0, 0, 0)
        z1 = sim.get_mg(sys).reshape(n, m)
        d = z1 - z0
        hc, wc = -(-n // FACTOR), -(-m // FACTOR)
        pad = np.zeros((hc * FACTOR, wc * FACTOR))
        cnt = np.zeros_like(pad)
        pad[:n, :m] = d
        cnt[:n, :m] = 1
        ref = pad.reshape(hc, FACTOR, wc, FACTOR).sum((1, 3)) / cnt.reshape(hc, FACTOR, wc, FACTOR).sum((1, 3))
        got = T[0].cpu().numpy()
        assert np.abs(got[:hc, :wc] - ref).max() <= 1e-5 * np.abs(ref).max() + 1e-30
        assert np.all(got[hc:, :] == 0) and np.all(got[:, wc:] == 0)
        assert torch.all(X[..., 2] == 0)
        assert torch.all(X[0, :hc, :wc, 1] > 0)  # reciprocal density inside the image
    sim.close()


def _trained_nets(dev):
    from incrmt_b200 import capi, learned
    sim, dt = _sim(seed=6)
    sim.step(dt, 3)
    data = learned.capture(sim, FACTOR, 48, dt, dev)
    sim.close()
    nets = {}
    for sys, (X, T) in data.items():
        Xn, Tn, V = learned.normalise(X, T)
        net = capi.UNet(3, 16, seed=3 + sys)
        first = learned.train(net, Xn, Tn, V, 1)
        last = learned.train(net, Xn, Tn, V, 300, seed=1)
        assert last < first, (sys, first, last)
        nets[sys] = net
    return nets, dt


def test_learned_warm_start_in_the_step(gpu):
    import torch
    from incrmt_b200 import capi
    dev = torch.device("cuda")
    nets, _ = _trained_nets(dev)
    runs = {}
    for mode in ["plain", 0, 1]:
        sim, dt = _sim()
        sim.step(dt, 3)
        if mode != "plain":
            for sys in (capi.SYS_MAC, capi.SYS_FEM):
                sim.set_learned(sys, nets[sys], FACTOR, mode)
        s0 = sim.stats()
        sim.step(dt, 10)
        s1 = sim.stats()
        runs[mode] = dict(u=sim.get("u"), v=sim.get("v"), p=sim.get("p"),
                          lst=[sim.learned_stats(s) for s in (capi.SYS_MAC, capi.SYS_FEM)],
                          solves=(s1.solves_mac - s0.solves_mac, s1.solves_fem - s0.solves_fem))
        sim.close()
    for mode in (0, 1):
        r = runs[mode]
        for k in range(2):
            st = r["lst"][k]
            assert st.applied + st.fallback + st.skipped == r["solves"][k]
            # a skip follows eight rejections in a row
            assert st.skipped == 0 or st.fallback >= 8
        for f in "uvp":
            e = _rel(r[f][2:-2, 2:-2], runs["plain"][f][2:-2, 2:-2])
            assert e <= 1e-6, (mode, f, e)
    for k in range(2):
        assert runs[0]["lst"][k].applied <= runs[1]["lst"][k].applied
    for net in nets.values():
        net.close()
