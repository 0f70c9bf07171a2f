"""Benchmark of incrmt_b200 on one node; prints ONE JSON line on rank 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload flag2048|flag3456|sed2048|sed1024|sspin1024|mac4096]
                    [--precision fp64|mixed] [--guess previous|learned]
                    [--coarse-refresh R] [--also W1,W2]

The metric: steps per second of fluid_2d::step_forward (fluid_2d.cc:298-369)
and V-cycles per projection at a 1e-9 relative residual, with the learned
warm start and mixed precision against the plain FP64 multigrid started from
the previous step's pressure (the reference's warm start, mgs_common.cc:15-21).

Default run (N=1): workload "flag2048", the flag scenario (ftest.cc:335-378:
y-periodic channel, uniform inflow, zero-pressure outlet, FEM projection with
its fixed column) on the literal 2048 x 2048 grid of [-1,5]x[-1,1] (cells
three times as wide as high), mass ratio 1, bending rigidity 0.1, Re 100,
aspect ratio 10. Before timing, the learned warm starts of both projections
are trained on a training run of the same workload (the flag with a
perturbed tail) with the library's own U-Net kernels. Then, from the same
initial state, W + K steps with the learned guess and mixed precision
(`value`, the K timed) and W + K steps of the plain FP64 method (`plain_fp64`):
steps/s, V-cycles per projection, the learned guess's fallback rate and the
difference of the end fields (u, v, p, every phi) of the two runs. A second
workload (--also, default sed2048 at N=1) repeats the comparison.

Workloads: flag3456 (the isotropic 3456 x 1152 flag), sed2048 / sed1024 (32
seeded circles and ellipses, size 0.03-0.06, density 1.5-3, G 1, gravity
(rho_s-1)/rho_s, settling in the walled [-0.75,0.75]x[-1.5,1.5] box of the
reference's sediment driver at 2048 x 4096 / 1024 x 2048), sspin1024 (ftest
simple-spin at 1024 x 1024), mac4096 (the standalone variable-density MAC
solve at 4096 x 4096: 8 seeded circles at density ratio 3, right-hand side
from 64 seeded Gaussian velocity blobs, incrmt_b200/workloads.py; one step =
coefficients and hierarchy rebuilt from the density, then V-cycles from zero
to 1e-9). The simulation arrays of every workload exceed the 126 MB L2 and
each step streams them, so no flush is added.

The projections rebuild their Galerkin coarse levels on every density
change by default (--coarse-refresh 1), as the reference's solver setup
does (mgs_mac.cc:62-63, mgs_fem.cc:108-109); the line also reports the
lagged rebuild (every 16 projections) of the timed configuration.

The timed region is bracketed by cudaProfilerStart/Stop, so
`ncu --profile-from-start off` lists exactly the timed launches.

Multi-GPU: the path does not shard; N ranks run N independent replicas
(weak scaling), timed on the device as the maximum over ranks.

--impl reference times the reference's own CPU code (oracle/_ref: the
reference's sources built with the clean-room TGMG shim) on the same
workload with all host threads, a bounded number of steps.
"""
import argparse
import faulthandler
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "steps/s, V-cycles/projection @1e-9 residual: learned+mixed vs plain GPU MG"


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi during a region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.tmp, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        self.tmp.flush()
        rows = []
        with open(self.tmp.name) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) >= 9:
                    rows.append(p)
        os.unlink(self.tmp.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def _traffic(key):
    """DRAM bytes per launch of a roofline kernel from the committed ncu
    summary (profiles/traffic.json: dram__bytes_read.sum + dram__bytes_write.sum
    of one captured launch), or None."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        return json.load(f).get(key)


def vcycle_pass_bytes(m, n, c0, w=8, tail=1024):
    """Compulsory bytes of one FP64 V-cycle as the kernels run it on an
    isotropic grid (standard coarsening): on a level of N unknowns with c
    coefficient words each (c0 on the fine level, 9 on the Galerkin levels),
    two tile-fused smoothing launches read z, b and the coefficients and write
    z ((3 + c) words each), the restriction reads z, b, the coefficients and
    four prolongation weights (6 + c) and writes b and z of the coarse level,
    the prolongation reads the weights and z and writes z (6) and reads each
    coarse value once: (18 + 3c) N + 3 N_coarse words; the fine level adds the
    residual norm (2 + c) N. Levels of at most `tail` unknowns run in one
    block from shared memory and are not counted."""
    total, c, first = 0.0, c0, True
    while m * n > tail:
        mc, nc = (m + 1) // 2, (n + 1) // 2
        total += (18 + 3 * c) * m * n + 3 * mc * nc
        if first:
            total += (2 + c) * m * n
            first = False
        m, n, c = mc, nc, 9
    return total * w


def _roofline(key, ms, nbytes, launches, kernel, rule):
    """Roofline object of a kernel timed live with CUDA events: achieved =
    algorithmic bytes / device time, against the measured copy bandwidth."""
    if not launches or ms <= 0:
        return None
    peak, peak_kind = _peaks()
    achieved = (nbytes / (ms / 1e3)) / 1e9
    t = _traffic(key)
    return {"bound": "hbm", "kernel": kernel, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_kind": peak_kind,
            "traffic": t["bytes_per_launch"] if t else None,
            "traffic_source": t["source"] if t else None,
            "algorithmic_bytes_per_launch": nbytes / launches,
            "avg_launch_us": 1e3 * ms / launches, "launches": launches, "bytes_rule": rule}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _maybe_init(ws, local):
    import torch
    if ws > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        return dist
    return None


def _max_over_ranks(dist, v):
    if dist is None:
        return v
    import torch
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(dist):
    if dist is not None:
        dist.barrier()


# ---------------------------------------------------------------------------
# Workloads

SED_BOX = (-0.75, 0.75, -1.5, 1.5)
FLAG_BOX = (-1.0, 5.0, -1.0, 1.0)
# flag scenario constants (none fixed by the reference for these grids):
# mass ratio 1, bending rigidity 0.1, Re 100, aspect ratio 10
FLAG_MU, FLAG_KB, FLAG_RE, FLAG_AR = 1.0, 0.1, 100.0, 10.0
SIM_WORKLOADS = {
    "flag2048": ("flag", 2048, 2048),
    "flag3456": ("flag", 3456, 1152),
    "sed2048": ("sed", 2048, 4096),
    "sed1024": ("sed", 1024, 2048),
    "sspin1024": ("sspin", 1024, 1024),
}


def describe(workload):
    kind, m, n = SIM_WORKLOADS[workload]
    if kind == "flag":
        return (f"flag {m}x{n} on [-1,5]x[-1,1] (mu {FLAG_MU:g}, k_B {FLAG_KB:g}, Re {FLAG_RE:g}, ar {FLAG_AR:g}), "
                f"FEM with zero-pressure outlet, y-periodic; fluid_2d::step_forward, dt of 900 frames over T=30")
    if kind == "sed":
        return (f"sediment {m}x{n}: 32 seeded circles and ellipses (r 0.03-0.06, rho 1.5-3, G 1) settling, "
                f"fluid_2d::step_forward, dt of 0.1 frames")
    return f"simple-spin {m}x{n} fluid_2d::step_forward, dt of solve(2pi,120)"


def frame_interval(workload):
    kind = SIM_WORKLOADS[workload][0]
    return {"flag": 30.0 / 900, "sed": 0.1, "sspin": 2 * np.pi / 120}[kind]


def _flag_params(training):
    w = 1.0 / FLAG_AR
    # the training run's tail is perturbed (ftest's optional perturb_v), a
    # different trajectory
    return (0.0, 0.0, 1.0, w, 0.25 * w, 0.2 if training else 0.0, 17), 4 * FLAG_KB / w ** 3, FLAG_MU / w


def make_sim(workload, rank, prec, training=False):
    """The GPU simulation of a workload (capi.Simulation), initialised."""
    from incrmt_b200 import capi, workloads
    kind, m, n = SIM_WORKLOADS[workload]
    if kind == "sspin":
        sim = capi.Simulation(m, n, ntrace=512, precision=prec)
        sim.add_simple_spin()
        sim.initialize()
        rng = np.random.default_rng(1 + rank)
        sim.set_tracers(rng.uniform(-1, 1, size=(512, 2)))
        return sim
    if kind == "flag":
        (cx, cy, fl, fw, fa, pv, nt), G, rhos = _flag_params(training)
        ax, bx, ay, by = FLAG_BOX
        sim = capi.Simulation(m, n, ax=ax, bx=bx, ay=ay, by=by, visc=1.0 / FLAG_RE, ntrace=0,
                              precision=prec, y_prd=True, horiz_flow=1.0)
        sim.add_flag(cx, cy, fl, fw, fa, G, rhos, perturb_v=pv, ntrace=nt)
        sim.initialize()
        return sim
    ax, bx, ay, by = SED_BOX
    sim = capi.Simulation(m, n, ax=ax, bx=bx, ay=ay, by=by, visc=2e-3, ntrace=512, precision=prec)
    for o in workloads.sediment_bodies(seed=(1011 if training else 11) + rank):
        if o["kind"] == "circle":
            sim.add_circle(o["cx"], o["cy"], o["r"], 1.0, o["rhos"], grav=o["grav"])
        else:
            sim.add_ellipse(o["cx"], o["cy"], o["r"], o["b"], o["theta"], 1.0, o["rhos"], grav=o["grav"])
    sim.initialize()
    rng = np.random.default_rng(1 + rank)
    sim.set_tracers(np.stack([rng.uniform(ax, bx, 512), rng.uniform(ay, by, 512)], axis=1))
    return sim


def frame_dt(dt_reg, interval):
    """fluid_2d::solve's step: the frame interval split into equal steps no
    longer than dt_reg (fluid_2d.cc:266-270)."""
    return interval / (int(interval / dt_reg) + 1)


# ---------------------------------------------------------------------------
# CPU reference (the reference's own code, oracle/_ref)

def cpu_reference_mac(m, steps, warmup, seed=3):
    from incrmt_b200 import workloads
    from oracle import refsim
    if not refsim.available():
        refsim.build()
    rho, b = workloads.standalone_mac_problem(m, seed=seed)
    rho, b = rho.numpy(), b.numpy().ravel()
    for _ in range(warmup):
        refsim.mg_solve(0, m, m, rho, b)
    t0 = time.perf_counter()
    vc = []
    for _ in range(steps):
        _, _, st = refsim.mg_solve(0, m, m, rho, b)
        vc.append(st[0])
    dt = time.perf_counter() - t0
    return steps / dt, dt, float(np.mean(vc)) if vc else 0.0


def cpu_reference_sspin(m, steps, warmup):
    """The reference's own step on the host cores: oracle/_ref/ref_run."""
    from oracle import refsim
    if not refsim.available():
        refsim.build()
    with tempfile.TemporaryDirectory() as td:
        out = subprocess.run([refsim.RUN, str(m), str(steps), str(warmup), os.path.join(td, "sspin")],
                             capture_output=True, text=True, check=True).stdout
    last = [l for l in out.splitlines() if l and not l.startswith("#")][-1].split()
    nsteps, secs, vm, vf, threads = int(last[0]), float(last[1]), int(last[2]), int(last[3]), int(last[4])
    return nsteps / secs, secs, (vm + vf) / (2.0 * nsteps), threads


def _sed_reference_objects(seed=11):
    """The sediment bodies as reference objects: circles as obj_circle, the
    ellipses as the oracle harness's obj_ellipse (an obj_standard subclass
    compiled against the reference; the reference has no ellipse)."""
    from incrmt_b200 import workloads
    objs = []
    for o in workloads.sediment_bodies(seed=seed):
        if o["kind"] == "circle":
            objs.append(("circle", (o["cx"], o["cy"], o["r"], 0, 0, 0, o["grav"]), 1.0, o["rhos"]))
        else:
            objs.append(("ellipse", (o["cx"], o["cy"], o["r"], o["b"], o["theta"], o["grav"]), 1.0, o["rhos"]))
    return objs


def cpu_reference_sim(workload, steps, warmup):
    """The reference's own step on a simulation workload (oracle/_ref), with
    the projections' V-cycles per projection. Returns (steps/s, seconds,
    V-cycles per projection, threads)."""
    from oracle import refsim
    kind, m, n = SIM_WORKLOADS[workload]
    if kind == "sspin":
        return cpu_reference_sspin(m, steps, warmup)
    if not refsim.available():
        refsim.build()
    if kind == "flag":
        p, G, rhos = _flag_params(False)
        r = refsim.RefSim(m, ntrace=0, n=n, objects=[("flag", p, G, rhos)], geom=FLAG_BOX, visc=1.0 / FLAG_RE,
                          flow_u=1.0)
    else:
        r = refsim.RefSim(m, ntrace=512, n=n, objects=_sed_reference_objects(), geom=SED_BOX, visc=2e-3)
    dt = frame_dt(r.scalars()["dt_reg"], frame_interval(workload))
    r.step(dt, warmup)
    r.vcycles(0)  # the counters restart (ref_vcycles reads and resets them)
    r.vcycles(1)
    t0 = time.perf_counter()
    r.step(dt, steps)
    secs = time.perf_counter() - t0
    vc = (r.vcycles(0) + r.vcycles(1)) / (2.0 * steps)
    r.close()
    return steps / secs, secs, vc, int(os.environ.get("OMP_NUM_THREADS", os.cpu_count()))


def cpu_steps(workload):
    """A bounded sample for the CPU reference: about 10-30 s of host work
    (the 2048-wide flag and sediment run at about one step per second on
    16 threads)."""
    kind, m, n = SIM_WORKLOADS[workload]
    return {"sspin": 40, "flag": 12, "sed": 12}[kind] if m * n > 2e6 else 40


def run_reference(args, ws, rank):
    if rank != 0:
        return
    threads = os.cpu_count()
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    if args.workload in SIM_WORKLOADS:
        nref = max(1, min(args.steps, cpu_steps(args.workload)))
        nwarm = min(args.warmup, 1 if nref < 10 else 2)
        try:
            sps, dt, vc, thr = cpu_reference_sim(args.workload, nref, nwarm)
        except Exception as e:
            print(json.dumps({"impl": "reference", "unavailable": f"reference build/run failed: {e}"}))
            return
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": sps, "unit": "steps/s",
            "n_gpus": args.gpus, "steps": nref, "warmup": nwarm,
            "ms_per_step": 1e3 * dt / nref, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": describe(args.workload), "flush": "working set larger than L2",
                       "coarse_refresh": 1, "krylov": False},
            "vcycles_per_projection": vc,
            "cpu_baseline": {"value": sps, "unit": "steps/s", "cores": thr, "kind": "reference",
                             "sample": f"{nref} steps after {nwarm} warm-up steps (reference sources + TGMG-API "
                                       f"shim, Galerkin setup on every projection), OMP threads = {thr}"},
            "e2e": {"value": sps, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return
    m = 4096
    # A 4096^2 solve takes seconds on the host: time at most 8 of them.
    nref = max(1, min(args.steps, 8))
    try:
        sps, dt, vc = cpu_reference_mac(m, nref, min(args.warmup, 1))
    except Exception as e:  # the reference could not be built here
        print(json.dumps({"impl": "reference", "unavailable": f"reference build/run failed: {e}"}))
        return
    line = {
        "impl": "reference", "metric": METRIC, "value": sps, "unit": "steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * dt / nref, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"standalone MAC solve {m}x{m} (8 circles rho 3, 64 blobs), 1e-9",
                   "flush": "inputs larger than L2"},
        "vcycles_per_projection": vc,
        "cpu_baseline": {"value": sps, "unit": "steps/s", "cores": threads, "kind": "reference",
                         "sample": f"{nref} full solves at {m}x{m} after {min(args.warmup, 1)} warm-up"},
        "e2e": {"value": sps, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# GPU path: simulation workloads

LEARNED_SIM_FACTOR = 8     # network grid: the projection's unknowns restricted by 8
LEARNED_SIM_SAMPLES = 400  # projections captured per system from the training run
LEARNED_SIM_STEPS = 2000   # Adam steps per network
LEARNED_SIM_BASE = 32      # channels at the finest level of the U-Net


def train_learned_sim(workload, rank, dev, guess=0):
    """The learned warm start of the MAC and FEM projections, trained with
    this library's own U-Net kernels on samples the method generates: a
    training run of the workload (another seed; for the flag a perturbed
    tail) captures every projection's input and correction."""
    import torch
    from incrmt_b200 import capi, learned
    t0 = time.perf_counter()
    sim = make_sim(workload, rank, capi.PREC_FP64, training=True)
    sim.set_guess(guess)  # the corrections the networks learn are to this warm start
    dt = frame_dt(sim.dt_reg, frame_interval(workload))
    sim.step(dt, 10)
    data = learned.capture(sim, LEARNED_SIM_FACTOR, LEARNED_SIM_SAMPLES, dt, dev)
    sim.close()
    t_data = time.perf_counter() - t0
    nets, losses = {}, {}
    t1 = time.perf_counter()
    for sys, (X, T) in data.items():
        Xn, Tn, V = learned.normalise(X, T)
        net = capi.UNet(4, LEARNED_SIM_BASE, seed=11 + sys)
        losses["mac" if sys == capi.SYS_MAC else "fem"] = learned.train(net, Xn, Tn, V, LEARNED_SIM_STEPS, seed=rank)
        nets[sys] = net
    torch.cuda.synchronize()
    H, W = data[capi.SYS_MAC][0].shape[1:3]
    info = {"network": f"two U-Nets (MAC, FEM), 4 levels, base {LEARNED_SIM_BASE} channels, "
                       f"{nets[0].num_params()} parameters each, BF16 activations",
            "grid": f"{H}x{W} (projection restricted by {LEARNED_SIM_FACTOR})",
            "train_samples_per_system": LEARNED_SIM_SAMPLES, "train_steps": LEARNED_SIM_STEPS, "batch": 8,
            "final_loss": losses, "data_seconds": t_data, "train_seconds": time.perf_counter() - t1}
    return nets, info


SNAP_FIELDS = ("u", "v", "p")


def _snapshot(sim):
    """End fields of a run: u, v, p and every object's level set (interior)."""
    d = {f: sim.get(f)[2:-2, 2:-2].copy() for f in SNAP_FIELDS}
    for k in range(sim.objects):
        d[f"phi{k}"] = sim.get("phi", k)[2:-2, 2:-2].copy()
    return d


def _snap_errors(a, b):
    """Largest difference of each field relative to the FP64 run's largest
    magnitude (u, v, p) or to its grid spacing h (the level sets: max over
    the objects, in units of h)."""
    out = {}
    for f in SNAP_FIELDS:
        out[f] = float(np.abs(a[f] - b[f]).max() / max(np.abs(b[f]).max(), 1e-300))
    phis = [k for k in b if k.startswith("phi")]
    if phis:
        out["phi_max_over_objects"] = max(float(np.abs(a[k] - b[k]).max()) for k in phis)
    return out


def _vcycles(st0, st1, steps):
    return ((st1.vcycles_mac - st0.vcycles_mac) / max(1, st1.solves_mac - st0.solves_mac),
            (st1.vcycles_fem - st0.vcycles_fem) / max(1, st1.solves_fem - st0.solves_fem))


def projection_roofline(sim, workload, prec, vc_mac, vc_fem, phases):
    """V-cycle-level roofline of the two projections: the algorithmic bytes
    of the V-cycles they ran, (4/3) N w [(nu1+nu2+1)(3+c) + 3.5] per V-cycle
    (w = 8 FP64; in mixed precision w = 4 for the FP32 cycle plus the FP64
    outer residual and update, 68 B MAC / 60 B FEM per unknown), over the
    device time of the mac and fem phases."""
    peak, peak_kind = _peaks()
    kind, m, n = SIM_WORKLOADS[workload]
    nm, nf = m * n, (m + 1) * (n if kind == "flag" else n + 1)
    if prec == 0:
        bm, bf = 304.0, 251.0
    else:
        bm, bf = 152.0 + 68.0, 125.0 + 60.0
    bytes_ = vc_mac * nm * bm + vc_fem * nf * bf
    ms = phases.get("mac", 0.0) + phases.get("fem", 0.0)
    if ms <= 0:
        return None
    achieved = bytes_ / (ms / 1e3) / 1e9
    return {"achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
            "algorithmic_bytes_per_step": bytes_, "ms_per_step": ms,
            "bytes_rule": "V-cycles x (4/3) N w [(nu1+nu2+1)(3+c)+3.5], nu1=nu2=2; c=2 MAC, 1 FEM; "
                          "mixed: w=4 plus 68/60 B per unknown of FP64 outer residual and update"}


def sim_run(workload, rank, dev, prec, nets, steps, warmup, coarse_refresh, dist, clocks=None, extras=True, guess=0,
            e2e_steps=0, learned_rule=0, krylov=False):
    """One run of a simulation workload: warm-up, K timed steps (CUDA events
    on the simulation stream, max over ranks), end snapshot, then (extras)
    the phase breakdown and the live smoother roofline over further steps
    and (e2e_steps) the end-to-end rate through the C ABI with one frame of
    fields copied to host. Returns a dict."""
    import torch
    from incrmt_b200 import capi
    sim = make_sim(workload, rank, prec)
    sim.set_coarse_refresh(coarse_refresh)
    sim.set_guess(guess)
    sim.set_krylov(krylov)
    dt = frame_dt(sim.dt_reg, frame_interval(workload))
    if nets is not None:
        for sys, net in nets.items():
            sim.set_learned(sys, net, LEARNED_SIM_FACTOR, learned_rule)
    ext = torch.cuda.ExternalStream(sim.stream(), device=dev)
    sim.step(dt, warmup)
    torch.cuda.synchronize()
    _barrier(dist)
    torch.cuda.synchronize()
    st0 = sim.stats()
    nl0 = sum(n.launches() for n in nets.values()) if nets else 0
    lst0 = {s: sim.learned_stats(s) for s in nets} if nets else {}
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with (clocks if clocks is not None else _NullCtx()):
        torch.cuda.cudart().cudaProfilerStart()
        e0.record(ext)
        sim.step(dt, steps)
        e1.record(ext)
        torch.cuda.synchronize()
        torch.cuda.cudart().cudaProfilerStop()
    ms = _max_over_ranks(dist, e0.elapsed_time(e1))
    st1 = sim.stats()
    out = {"ms": ms, "steps_per_s": steps / (ms / 1e3), "dt": dt}
    out["vc_mac"], out["vc_fem"] = _vcycles(st0, st1, steps)
    out["launches"] = int(st1.launches - st0.launches) + \
        ((sum(n.launches() for n in nets.values()) - nl0) if nets else 0)
    out["coarse_builds_per_step"] = (st1.coarse_builds - st0.coarse_builds) / steps
    out["coarse_retries"] = int(st1.coarse_retries - st0.coarse_retries)
    out["mixed_fallbacks"] = int(st1.mixed_fallbacks - st0.mixed_fallbacks)
    out["krylov_fallbacks"] = int(st1.krylov_fallbacks - st0.krylov_fallbacks)
    out["march_sweeps_per_step"] = (st1.march_sweeps - st0.march_sweeps) / steps
    out["extrap_sweeps_per_step"] = (st1.extrap_sweeps - st0.extrap_sweeps) / steps
    if nets:
        lst1 = {s: sim.learned_stats(s) for s in nets}
        nm = lambda s: "mac" if s == capi.SYS_MAC else "fem"  # noqa: E731
        out["learned"] = {nm(s): {"applied": int(lst1[s].applied - lst0[s].applied),
                                  "fallback": int(lst1[s].fallback - lst0[s].fallback),
                                  "skipped": int(lst1[s].skipped - lst0[s].skipped)} for s in nets}
        for v in out["learned"].values():
            v["fallback_rate"] = v["fallback"] / max(1, v["applied"] + v["fallback"])
    out["snapshot"] = _snapshot(sim)
    if extras:
        n_extra = min(steps, 10)
        sim.set_profiling(True)
        sim.step(dt, n_extra)
        out["phases"] = {k: v / n_extra for k, v in sim.profile().items()}
        sim.set_profiling(False, smoothers=True)
        sim.step(dt, n_extra)
        sm = [0.0, 0.0, 0]
        for which in (capi.SYS_MAC, capi.SYS_FEM):
            a, b, c = sim.smoother_profile(which)
            sm = [sm[0] + a, sm[1] + b, sm[2] + c]
        out["smoother"] = sm
        sim.set_profiling(False)
    if e2e_steps:
        # End to end through the C ABI as fluid_2d::solve drives it: the
        # steps of one frame, then the frame's fields copied to host buffers
        # (p, u, v for the vorticity, X, Y, phi; fluid_2d::write_files,
        # fluid_2d_io.cc:60-102).
        # the frame lands in pinned host buffers allocated once, as an output
        # loop would keep them
        names = ("p", "u", "v", "X", "Y", "phi")
        pinned = [torch.empty(sim.nl * sim.ml, dtype=torch.float64).pin_memory() for _ in names]
        _barrier(dist)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sim.step(dt, e2e_steps)
        host = [sim.get(f, out=b.numpy()) for f, b in zip(names, pinned)]
        secs = _max_over_ranks(dist, time.perf_counter() - t0)
        out["e2e_steps_per_s"] = e2e_steps / secs
        out["e2e_d2h_bytes_per_step"] = int(sum(h.nbytes for h in host) / e2e_steps)
    out["objects"], out["cells"] = sim.objects, (sim.m + 4) * (sim.n + 4)
    sim.close()
    return out


class _NullCtx:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


def compare_workload(workload, args, ws, rank, dev, dist, clocks=None, extras=True, e2e=True):
    """The metric on one workload: the timed configuration (learned guess
    and/or mixed precision) against the plain FP64 method, same steps from
    the same initial state. Returns (timed run, plain run, learned info)."""
    from incrmt_b200 import capi
    prec = capi.PREC_MIXED if args.precision == "mixed" else capi.PREC_FP64
    nets, info = (None, None)
    if args.guess == "learned":
        nets, info = train_learned_sim(workload, rank, dev, args.extrapolate)
    a = sim_run(workload, rank, dev, prec, nets, args.steps, args.warmup, args.coarse_refresh, dist, clocks=clocks,
                extras=extras, guess=args.extrapolate, e2e_steps=args.steps if e2e else 0,
                learned_rule=args.learned_rule, krylov=bool(args.krylov))
    plain = None
    if nets is not None or prec != capi.PREC_FP64 or args.extrapolate:
        plain = sim_run(workload, rank, dev, capi.PREC_FP64, None, args.steps, args.warmup, args.coarse_refresh,
                        dist, extras=extras)
        a["errors_vs_fp64"] = _snap_errors(a["snapshot"], plain["snapshot"])
    if args.coarse_refresh == 1 and extras:
        # the timed configuration with the Galerkin coarse levels rebuilt
        # every 16 projections instead of on every one (the reference's
        # policy, kept for the headline)
        c = sim_run(workload, rank, dev, prec, nets, args.steps, args.warmup, 16, dist, extras=False,
                    guess=args.extrapolate, learned_rule=args.learned_rule, krylov=bool(args.krylov))
        a["coarse_refresh_16"] = {"steps_per_s": ws * c["steps_per_s"],
                                  "vcycles_per_projection": {"mac": c["vc_mac"], "fem": c["vc_fem"]},
                                  "errors_vs_fp64": _snap_errors(c["snapshot"], plain["snapshot"])
                                  if plain is not None else None}
    # the timed configuration with the flexible CG around the V-cycle
    # switched the other way (incrmt_sim_set_krylov)
    kv = sim_run(workload, rank, dev, prec, nets, args.steps, args.warmup, args.coarse_refresh, dist,
                 extras=False, guess=args.extrapolate, learned_rule=args.learned_rule, krylov=not args.krylov)
    a["with_krylov" if not args.krylov else "without_krylov"] = {
        "steps_per_s": ws * kv["steps_per_s"],
        "vcycles_per_projection": {"mac": kv["vc_mac"], "fem": kv["vc_fem"]},
        "krylov_fallbacks": kv["krylov_fallbacks"], "mixed_fallbacks": kv["mixed_fallbacks"],
        "errors_vs_fp64": _snap_errors(kv["snapshot"], plain["snapshot"]) if plain is not None else None}
    if nets is not None:
        for net in nets.values():
            net.close()
        # the same configuration without the networks: what the learned
        # correction adds or costs on top of the rest
        b = sim_run(workload, rank, dev, prec, None, args.steps, args.warmup, args.coarse_refresh, dist,
                    extras=False, guess=args.extrapolate, krylov=bool(args.krylov))
        a["without_learned"] = {"steps_per_s": ws * b["steps_per_s"],
                                "vcycles_per_projection": {"mac": b["vc_mac"], "fem": b["vc_fem"]},
                                "mixed_fallbacks": b["mixed_fallbacks"],
                                "errors_vs_fp64": _snap_errors(b["snapshot"], plain["snapshot"])
                                if plain is not None else None}
    return a, plain, info


def run_ours_sim(args, ws, rank, local, dist):
    """Simulation steps on the GPU through the simulation C ABI."""
    import torch
    from incrmt_b200 import capi

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    prec = capi.PREC_MIXED if args.precision == "mixed" else capi.PREC_FP64
    with ClockSampler(local) as clk:
        a, plain, info = compare_workload(args.workload, args, ws, rank, dev, dist, clocks=None)
    # the clock record covers the whole comparison (the timed steps are a
    # few percent of it; the sampler runs throughout)
    clocks = clk.summary()
    value = ws * a["steps_per_s"]
    also = {}
    for w in [x for x in args.also.split(",") if x] if ws == 1 else []:
        if w == args.workload or w not in SIM_WORKLOADS:
            continue
        b, bplain, binfo = compare_workload(w, args, ws, rank, dev, dist, extras=False, e2e=False)
        also[w] = {"workload": describe(w), "steps_per_s": b["steps_per_s"],
                   "vcycles_per_projection": {"mac": b["vc_mac"], "fem": b["vc_fem"]},
                   "mixed_fallbacks": b["mixed_fallbacks"]}
        if bplain is not None:
            also[w]["plain_fp64"] = {"steps_per_s": bplain["steps_per_s"],
                                     "vcycles_per_projection": {"mac": bplain["vc_mac"], "fem": bplain["vc_fem"]}}
            also[w]["speedup_vs_plain_fp64"] = b["steps_per_s"] / bplain["steps_per_s"]
            also[w]["errors_vs_fp64"] = b["errors_vs_fp64"]
        if "learned" in b:
            also[w]["learned"] = b["learned"]
        for key in ("with_krylov", "without_krylov"):
            if key in b:
                also[w][key] = b[key]
    if rank != 0:
        return
    cpu = None
    if ws == 1 and not args.no_cpu_baseline:
        try:
            n = cpu_steps(args.workload)
            w_ = 2 if n >= 10 else 0
            sps, dts, vcr, thr = cpu_reference_sim(args.workload, n, w_)
            cpu = {"value": sps, "unit": "steps/s", "cores": thr, "kind": "reference",
                   "sample": f"{n} steps after {w_} warm-up of the same workload (reference sources + "
                             f"TGMG-API shim, {vcr:.2f} V-cycles per projection), OMP threads = {thr}"}
        except Exception as e:
            cpu = {"value": None, "unit": "steps/s", "cores": 0, "kind": "reference",
                   "sample": f"unavailable: {e}"}
    sm_ms, sm_bytes, sm_launch = a["smoother"]
    roof = _roofline(f"{args.workload}_smooth", sm_ms, sm_bytes, sm_launch,
                     "k_smooth_rb / k_smooth_tile on the fine level of the MAC and FEM projections "
                     "(two Gauss-Seidel sweeps per launch)",
                     "updated unknowns x 2 sweeps x (3+c) x w; c=2 MAC, 1 FEM")
    if roof is not None:
        roof["projection"] = projection_roofline(None, args.workload, prec, a["vc_mac"], a["vc_fem"], a["phases"])
        if plain is not None and "phases" in plain:
            roof["projection_plain_fp64"] = projection_roofline(None, args.workload, capi.PREC_FP64, plain["vc_mac"],
                                                                plain["vc_fem"], plain["phases"])
    start = {0: "the previous solution", 1: "the extrapolation 2 z(n-1) - z(n-2) of the last two solutions",
             2: "the extrapolation 3 z(n-1) - 3 z(n-2) + z(n-3) of the last three solutions"}[args.extrapolate]
    guess = f"learned warm start on {start}" if args.guess == "learned" else start
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": a["ms"] / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if prec == capi.PREC_FP64 else "f64 state, f32 V-cycles in f64 defect correction",
        "data": "synthetic",
        "config": {"workload": describe(args.workload), "precision": args.precision, "initial_guess": guess,
                   "flush": "working set larger than L2", "parallelism": f"replicas x{ws}",
                   "coarse_refresh": args.coarse_refresh, "krylov": bool(args.krylov)},
        "vcycles_per_projection": {"mac": a["vc_mac"], "fem": a["vc_fem"]},
        "mixed_fallbacks": a["mixed_fallbacks"],
        "krylov_fallbacks": a["krylov_fallbacks"],
        "coarse_builds_per_step": a["coarse_builds_per_step"],
        "phase_ms_per_step": a["phases"],
        "march_sweeps_per_step": a["march_sweeps_per_step"],
        "extrap_sweeps_per_step": a["extrap_sweeps_per_step"],
        "roofline": roof,
        "cpu_baseline": cpu,
        "e2e": {"value": ws * a["e2e_steps_per_s"], "unit": "steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": a["e2e_d2h_bytes_per_step"],
                "note": "state resident on the device; one frame of fields (p,u,v,X,Y,phi) copied to host per "
                        "timed run of K steps"},
        "gpu_launches": a["launches"],
        "clocks": clocks,
    }
    if plain is not None:
        line["plain_fp64"] = {"value": ws * plain["steps_per_s"], "unit": "steps/s",
                              "vcycles_per_projection": {"mac": plain["vc_mac"], "fem": plain["vc_fem"]},
                              "phase_ms_per_step": plain.get("phases")}
        line["speedup_vs_plain_fp64"] = a["steps_per_s"] / plain["steps_per_s"]
        line["errors_vs_fp64"] = a["errors_vs_fp64"]
    if info is not None:
        info.update(a.get("learned", {}))
        line["learned"] = info
    if "without_learned" in a:
        line["without_learned"] = a["without_learned"]
    if "coarse_refresh_16" in a:
        line["coarse_refresh_16"] = a["coarse_refresh_16"]
    for key in ("with_krylov", "without_krylov"):
        if key in a:
            line[key] = a[key]
    if also:
        line["also"] = also
    print(json.dumps(line))


LEARNED_FACTOR = 8      # the network runs on the 4096^2 solve restricted to 512^2
LEARNED_SAMPLES = 128   # training problems (seeds disjoint from the benchmarked one)
LEARNED_STEPS = 1500


def _train_learned_mac(s, m, dev, rank):
    """Trains the learned initial guess on GPU-generated 4096^2 MAC problems
    with this library's own U-Net kernels: inputs from incrmt_mg_learned_input
    (zero start), targets the FP64 multigrid solutions restricted by block
    averages and normalised. Returns the network and a summary."""
    import torch
    from incrmt_b200 import capi, workloads
    t0 = time.perf_counter()
    H, W = capi.learned_grid(m, m, LEARNED_FACTOR)
    X = torch.empty(LEARNED_SAMPLES, H, W, 3, dtype=torch.float32, device=dev)
    T = torch.empty(LEARNED_SAMPLES, H, W, dtype=torch.float32, device=dev)
    z = torch.zeros(m * m, dtype=torch.float64, device=dev)
    z0 = torch.zeros(m * m, dtype=torch.float64, device=dev)
    for k in range(LEARNED_SAMPLES):
        rho, b = workloads.standalone_mac_problem(m, seed=1000 + 97 * rank + k, device=dev)
        rho, b = rho.contiguous(), b.contiguous().view(-1)
        z.zero_()
        torch.cuda.synchronize()
        s.set_density_device(rho.data_ptr())
        s.solve_device(b.data_ptr(), z.data_ptr())
        capi.learned_input(s, b.data_ptr(), z0.data_ptr(), LEARNED_FACTOR, X[k].data_ptr())
        zt = torch.nn.functional.avg_pool2d(z.view(1, 1, m, m).float(), LEARNED_FACTOR)[0, 0]
        T[k] = (zt - zt.mean()) / zt.std()
    t_data = time.perf_counter() - t0
    V = torch.ones(8, H, W, dtype=torch.float32, device=dev)
    net = capi.UNet(4, 16, seed=11)
    g = torch.Generator(device="cpu").manual_seed(rank)
    t1 = time.perf_counter()
    loss = None
    for it in range(LEARNED_STEPS):
        idx = torch.randperm(LEARNED_SAMPLES, generator=g)[:8]
        xb, tb = X[idx].contiguous(), T[idx].contiguous()
        loss = net.train_step(8, H, W, xb.data_ptr(), tb.data_ptr(), V.data_ptr(),
                              2e-3 if it < 0.75 * LEARNED_STEPS else 5e-4)
    torch.cuda.synchronize()
    info = {"network": f"U-Net, 4 levels, base 16 channels, {net.num_params()} parameters, BF16 activations, "
                       f"mma.sync tensor-core convolutions",
            "grid": f"{H}x{W} (solve restricted by {LEARNED_FACTOR})", "train_samples": LEARNED_SAMPLES,
            "train_steps": LEARNED_STEPS, "batch": 8, "final_loss": loss,
            "data_seconds": t_data, "train_seconds": time.perf_counter() - t1}
    return net, info


def run_ours(args, ws, rank, local, dist):
    import torch
    from incrmt_b200 import capi, workloads
    if args.workload in SIM_WORKLOADS:
        return run_ours_sim(args, ws, rank, local, dist)

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    m = 4096
    prec = capi.PREC_MIXED if args.precision == "mixed" else capi.PREC_FP64
    rho, b = workloads.standalone_mac_problem(m, seed=3 + rank, device=dev)
    rho = rho.contiguous()
    b = b.contiguous().view(-1)
    z = torch.zeros_like(b)
    s = capi.MGSolver(capi.SYS_MAC, m, m)
    ext = torch.cuda.ExternalStream(s.stream(), device=dev)
    torch.cuda.synchronize()
    net, learned_info = None, None
    if args.learned:
        net, learned_info = _train_learned_mac(s, m, dev, rank)
        # Plain FP64 solves of the same problem, for the comparison line.
        vc_plain, t_plain = [], []
        for _ in range(5):
            s.set_density_device(rho.data_ptr())
            with torch.cuda.stream(ext):
                z.zero_()
            st = s.solve_device(b.data_ptr(), z.data_ptr(), precision=capi.PREC_FP64)
            vc_plain.append(st.vcycles)
        zstar = z.clone()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        for _ in range(5):
            s.set_density_device(rho.data_ptr())
            with torch.cuda.stream(ext):
                z.zero_()
            s.solve_device(b.data_ptr(), z.data_ptr(), precision=capi.PREC_FP64)
        e1.record(ext)
        torch.cuda.synchronize()
        learned_info["plain_fp64"] = {"value": 5 / (e0.elapsed_time(e1) / 1e3), "unit": "steps/s",
                                      "vcycles_per_projection": float(np.mean(vc_plain))}
        with torch.cuda.stream(ext):
            z.zero_()
        torch.cuda.synchronize()
        st = capi.learned_guess(s, net, b.data_ptr(), z.data_ptr(), LEARNED_FACTOR)
        dz, ds = z - z.mean(), zstar - zstar.mean()
        learned_info["guess_relative_error"] = float((dz - ds).norm() / ds.norm())
        learned_info["guess_alpha"] = st.alpha

    s.set_krylov(bool(args.krylov))

    def step():
        s.set_density_device(rho.data_ptr())
        with torch.cuda.stream(ext):
            z.zero_()
        if net is not None:
            capi.learned_guess(s, net, b.data_ptr(), z.data_ptr(), LEARNED_FACTOR, stats=False)
        st = s.solve_device(b.data_ptr(), z.data_ptr(), precision=prec)
        return st.vcycles

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    _barrier(dist)
    torch.cuda.synchronize()
    s.set_profiling(True)
    l0 = s.launches()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    vcs = []
    with ClockSampler(local) as clk:
        torch.cuda.cudart().cudaProfilerStart()
        e0.record(ext)
        for _ in range(args.steps):
            vcs.append(step())
        e1.record(ext)
        torch.cuda.synchronize()
        torch.cuda.cudart().cudaProfilerStop()
    ms = e0.elapsed_time(e1)
    launches = s.launches() - l0
    kms, kbytes, klaunch = s.profile()
    s.set_profiling(False)
    _barrier(dist)
    torch.cuda.synchronize()
    ms_max = _max_over_ranks(dist, ms)
    value = ws * args.steps / (ms_max / 1e3)

    # End to end through the C ABI with pinned host buffers: density and
    # right-hand side in, zero guess in, solution out, every step.
    rho_h = rho.cpu().pin_memory()
    b_h = b.cpu().pin_memory()
    z_h = torch.zeros_like(b_h).pin_memory()
    rho_np, b_np, z_np = rho_h.numpy(), b_h.numpy(), z_h.numpy()

    def e2e_step():
        if net is None:
            s.set_density(rho_np)
            z_np[:] = 0
            s.solve(b_np, z_np, precision=prec)
            return
        # With the learned guess: host buffers in on the solver's stream, the
        # guess and the solve on the device, the solution back to the host.
        with torch.cuda.stream(ext):
            rho.copy_(rho_h, non_blocking=True)
            b.copy_(b_h, non_blocking=True)
            z.zero_()
        s.set_density_device(rho.data_ptr())
        capi.learned_guess(s, net, b.data_ptr(), z.data_ptr(), LEARNED_FACTOR, stats=False)
        s.solve_device(b.data_ptr(), z.data_ptr(), precision=prec)
        with torch.cuda.stream(ext):
            z_h.copy_(z, non_blocking=True)
        ext.synchronize()

    for _ in range(min(args.warmup, 1)):
        e2e_step()
    _barrier(dist)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_s = time.perf_counter() - t0
    e2e_s = _max_over_ranks(dist, e2e_s)
    e2e = ws * args.steps / e2e_s

    # Release in order: the pinned host tensors were copied on the solver's
    # stream (non-blocking copies under torch.cuda.stream(ext) in e2e_step),
    # and when one is freed torch's pinned-memory allocator records an event
    # on every stream that used it, so they go first, while the solver (which
    # owns the stream) is still alive.
    h2d_bytes = int(rho_h.numel() * 8 + (1 if net is not None else 2) * b_h.numel() * 8)
    d2h_bytes = int(b_h.numel() * 8)
    del rho_np, b_np, z_np, rho_h, b_h, z_h
    torch.cuda.synchronize()
    import gc
    gc.collect()

    def release():
        torch.cuda.synchronize()
        s.close()
        if net is not None:
            net.close()

    if rank != 0:
        release()
        return
    cpu = None
    if ws == 1 and not args.no_cpu_baseline:
        try:
            threads = os.cpu_count()
            sps, dt, _ = cpu_reference_mac(m, 4, 0)
            cpu = {"value": sps, "unit": "steps/s", "cores": threads, "kind": "reference",
                   "sample": f"4 full {m}x{m} solves (reference callbacks + TGMG-API shim), "
                             f"OMP threads = {threads}"}
        except Exception as e:
            cpu = {"value": None, "unit": "steps/s", "cores": 0, "kind": "reference",
                   "sample": f"unavailable: {e}"}
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if prec == capi.PREC_FP64 else "f32 V-cycles in f64 defect correction",
        "data": "synthetic",
        "learned": learned_info,
        "config": {"workload": f"standalone MAC solve {m}x{m} (8 circles rho 3, 64 blobs), "
                               f"setup + V-cycles to 1e-9 from " +
                               ("the learned guess" if args.learned else "zero"), "precision": args.precision,
                   "flush": "inputs larger than L2 (each array 134 MB)", "parallelism": f"replicas x{ws}",
                   "krylov": bool(args.krylov)},
        "vcycles_per_projection": float(np.mean(vcs)),
        "roofline": _roofline("mac4096_smooth", kms, kbytes, klaunch,
                              "k_smooth_rb (fine-level red-black Gauss-Seidel, two sweeps per launch)",
                              "updated unknowns x 2 sweeps x (3+c) x w, c=2 (MAC)"),
        "cpu_baseline": cpu,
        "e2e": {"value": e2e, "unit": "steps/s",
                "h2d_bytes_per_step": h2d_bytes, "d2h_bytes_per_step": d2h_bytes},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if line["roofline"] is not None:
        # V-cycle level: the algorithmic bytes of the V-cycles run, (4/3) N w
        # [(nu1+nu2+1)(3+c) + 3.5] each (304 B per unknown FP64; FP32 cycle
        # 152 B plus the 68 B FP64 outer residual and update in mixed), over
        # the whole step, which also rebuilds the coefficients and the
        # Galerkin hierarchy (the reference's setup per solve)
        bpu = 304.0 if prec == capi.PREC_FP64 else 152.0 + 68.0
        if args.krylov:
            # the flexible CG's FP64 vector passes per iteration (dot
            # products, direction, A p, step: 124 B per unknown) instead of
            # the mixed path's 68 B outer residual and update
            bpu += 124.0 - (0.0 if prec == capi.PREC_FP64 else 68.0)
        ach = float(np.mean(vcs)) * m * m * bpu / (ms_max / args.steps / 1e3) / 1e9
        peak, kind = _peaks()
        line["roofline"]["vcycle_level"] = {"achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                                            "peak_kind": kind, "bytes_per_unknown_per_vcycle": bpu,
                                            "time": "whole step including the density setup"}
        if prec == capi.PREC_FP64:
            pb = vcycle_pass_bytes(m, m, 2)
            ach2 = float(np.mean(vcs)) * pb / (ms_max / args.steps / 1e3) / 1e9
            line["roofline"]["vcycle_passes"] = {
                "achieved": ach2, "peak": peak, "unit": "GB/s", "frac": ach2 / peak, "peak_kind": kind,
                "bytes_per_vcycle": pb, "time": "whole step including the density setup",
                "bytes_rule": "per level of N unknowns with c coefficient words (2 fine MAC, 9 Galerkin): "
                              "(18 + 3c) N w for two smoothing launches, the restriction and the prolongation "
                              "as implemented (each reading its arrays once), 3 w per coarse unknown, and the "
                              "fine residual norm (2 + c) N w"}
    print(json.dumps(line))
    release()


def main():
    # a crash in native code prints the Python stack it happened under
    faulthandler.enable()
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="flag2048", choices=list(SIM_WORKLOADS) + ["mac4096"])
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"],
                    help="arithmetic of the V-cycles (mixed: FP32 cycles inside FP64 defect correction)")
    ap.add_argument("--guess", default="learned", choices=["previous", "learned"],
                    help="initial guess of each projection: the previous solution, or the learned warm start "
                         "trained first on a training run of the workload")
    ap.add_argument("--learned", action="store_true", help="same as --guess learned")
    ap.add_argument("--extrapolate", type=int, default=2, choices=[0, 1, 2],
                    help="1: the projections start from 2 z(n-1) - z(n-2), 2: from 3 z(n-1) - 3 z(n-2) + "
                         "z(n-3) (incrmt_sim_set_guess); the plain FP64 comparison run always starts from the "
                         "previous solution")
    ap.add_argument("--coarse-refresh", type=int, default=1,
                    help="rebuild the projections' Galerkin coarse operators every K projections "
                         "(1: on every density change, as the reference)")
    ap.add_argument("--also", default="sed2048",
                    help="further simulation workloads compared the same way (comma-separated; N=1 only)")
    ap.add_argument("--krylov", type=int, default=0, choices=[0, 1],
                    help="1: flexible conjugate gradients with the V-cycle as preconditioner in the timed "
                         "configuration (incrmt_sim_set_krylov); the plain FP64 comparison run never uses it")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--learned-rule", type=int, default=0, choices=[0, 1],
                    help="fallback rule of the simulation's learned warm start (0: when the guess raises the "
                         "residual, 1: when the energy-optimal step is not positive)")
    ap.set_defaults(steps=20, warmup=5)
    args = ap.parse_args()
    if args.learned:
        args.guess = "learned"
    args.learned = args.guess == "learned"
    ws, rank, local = _dist()
    if args.impl == "reference":
        run_reference(args, ws, rank)
        return
    dist = _maybe_init(ws, local)
    try:
        run_ours(args, ws, rank, local, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()
    sys.stdout.flush()


if __name__ == "__main__":
    main()
