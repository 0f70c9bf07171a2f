"""Benchmark of incrmt_b200 on one node; prints ONE JSON line on rank 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload sspin1024|mac4096|sed1024|flag2048] [--precision fp64|mixed]
                    [--learned]

Workload "sspin1024" (default): the ftest simple-spin scenario (three-pronged
neo-Hookean rotor in a walled [-1,1]^2 box, ftest.cc:116-143) on a 1024 x 1024
grid. One step = fluid_2d::step_forward (fluid_2d.cc:298-369) with the step
size solve(2*pi,120) uses; the state starts from the scenario's own
initialisation. Every field array is 8.4 MB (the ~60 arrays together exceed
the 126 MB L2), and each step streams them, so no flush is added.

Workload "mac4096": the standalone variable-density MAC pressure solve on a
4096 x 4096 cell grid (8 seeded circles at density ratio 3, right-hand side
from 64 seeded Gaussian velocity blobs; incrmt_b200/workloads.py). One step =
one projection as the reference performs it: rebuild the coefficients and
the multigrid hierarchy from the density (mgs_mac.cc:62-63), then V-cycles
from a zero guess until ||b-Az||_2 <= 1e-9 ||b||_2. Every array is larger
than the 126 MB L2, so no flush is needed between steps.

The timed region is bracketed by cudaProfilerStart/Stop, so
`ncu --profile-from-start off` lists exactly the timed launches.

Workload "sed1024": the sediment configuration, 32 seeded bodies
(alternately circles and ellipses, size 0.03-0.06, density 1.5-3, G 1,
gravity (rho_s-1)/rho_s) settling in the walled [-0.75,0.75]x[-1.5,1.5] box of
the reference's sediment driver on a 1024 x 2048 grid; one step =
fluid_2d::step_forward. The reference arm runs the same bodies with each
ellipse replaced by a rounded rod, the reference having no ellipse.

Workload "flag2048": the flag scenario (ftest.cc:335-378; y-periodic channel,
uniform inflow, zero-pressure outlet, FEM projection with its fixed column) on
3456 x 1152 square cells of [-1,5]x[-1,1] (about 2048^2 cells), mass ratio 1,
bending rigidity 0.1, Re 100, aspect ratio 10.

--learned (mac4096): before timing, the learned initial guess is trained on
128 GPU-generated problems of the same kind (other seeds) with the library's
own U-Net kernels; every timed solve then starts from the network's guess
instead of zero. The line adds the training summary and plain FP64 solves of
the same problem for comparison.

Multi-GPU: the path does not shard; N ranks run N independent replicas
(weak scaling), timed on the device as the maximum over ranks.

--impl reference times the reference's own CPU code on the same workload:
the reference's mgs_mac_varying_rho callbacks driven by the clean-room TGMG
shim (oracle/_ref), with all host threads.
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


def cpu_reference_sed(steps, warmup):
    """The reference's own step on the sediment workload (oracle/_ref)."""
    from oracle import refsim
    if not refsim.available():
        refsim.build()
    r = refsim.RefSim(SED_M, ntrace=512, n=2 * SED_M, objects=_sed_reference_objects(), geom=SED_BOX, visc=2e-3)
    dt_reg = r.scalars()["dt_reg"]
    dt = 0.1 / (int(0.1 / dt_reg) + 1)
    r.step(dt, warmup)
    t0 = time.perf_counter()
    r.step(dt, steps)
    secs = time.perf_counter() - t0
    r.close()
    return steps / secs, secs, None, int(os.environ.get("OMP_NUM_THREADS", os.cpu_count()))


def cpu_reference_flag(steps, warmup):
    """The reference's own step on the flag workload (oracle/_ref)."""
    from oracle import refsim
    if not refsim.available():
        refsim.build()
    w = 0.1
    flag = ("flag", (0.0, 0.0, 1.0, w, 0.25 * w, 0.0, 17), 4 * 0.1 / w ** 3, 1.0 / w)
    r = refsim.RefSim(3 * FLAG_N, ntrace=0, n=FLAG_N, objects=[flag], geom=(-1.0, 5.0, -1.0, 1.0), visc=0.01,
                      flow_u=1.0)
    dt_reg = r.scalars()["dt_reg"]
    iv = 30.0 / 900
    dt = iv / (int(iv / dt_reg) + 1)
    r.step(dt, warmup)
    t0 = time.perf_counter()
    r.step(dt, steps)
    secs = time.perf_counter() - t0
    r.close()
    return steps / secs, secs, None, int(os.environ.get("OMP_NUM_THREADS", os.cpu_count()))


def run_reference(args, ws, rank):
    if rank != 0:
        return
    threads = os.cpu_count()
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    if args.workload in ("sed1024", "flag2048"):
        nref = max(1, min(args.steps, 3))
        try:
            fn = cpu_reference_sed if args.workload == "sed1024" else cpu_reference_flag
            sps, dt, _, thr = fn(nref, min(args.warmup, 1))
        except Exception as e:
            print(json.dumps({"impl": "reference", "unavailable": f"reference build/run failed: {e}"}))
            return
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": sps, "unit": "steps/s",
            "n_gpus": args.gpus, "steps": nref, "warmup": min(args.warmup, 1),
            "ms_per_step": 1e3 * dt / nref, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": (f"sediment {SED_M}x{2 * SED_M}, 32 bodies, ellipses as rounded rods"
                                    if args.workload == "sed1024" else
                                    f"flag {3 * FLAG_N}x{FLAG_N} (mu 1, k_B 0.1, Re 100, ar 10)"),
                       "flush": "working set larger than L2"},
            "cpu_baseline": {"value": sps, "unit": "steps/s", "cores": thr, "kind": "reference",
                             "sample": f"{nref} steps (a step takes seconds on the host)"},
            "e2e": {"value": sps, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return
    if args.workload == "sspin1024":
        m = 1024
        try:
            sps, dt, vc, thr = cpu_reference_sspin(m, args.steps, args.warmup)
        except Exception as e:
            print(json.dumps({"impl": "reference", "unavailable": f"reference build/run failed: {e}"}))
            return
        line = {
            "impl": "reference", "metric": METRIC, "value": sps, "unit": "steps/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * dt / max(args.steps, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"simple-spin {m}x{m} fluid_2d::step_forward, dt of solve(2pi,120)",
                       "flush": "working set larger than L2"},
            "vcycles_per_projection": vc,
            "cpu_baseline": {"value": sps, "unit": "steps/s", "cores": thr, "kind": "reference",
                             "sample": f"{args.steps} steps after {args.warmup} warm-up steps at {m}x{m}, "
                                       f"reference sources + TGMG-API shim, OMP threads = {thr}"},
            "e2e": {"value": sps, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line))
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
# GPU path

SED_M = 1024
SED_BOX = (-0.75, 0.75, -1.5, 1.5)
FLAG_N = 1152


def _make_sim(workload, rank, prec, training=False):
    """The simulation of a step workload and its frame interval:
    sspin1024 (ftest simple-spin, solve(2pi,120) frames) or sed1024 (32
    seeded circles and ellipses settling in the sediment box at 1024 x 2048,
    frame interval 0.1 as sediment.cc's 1600 frames over T=160)."""
    from incrmt_b200 import capi, workloads
    if workload == "sspin1024":
        m = 1024
        sim = capi.Simulation(m, m, ntrace=512, precision=prec)
        sim.add_simple_spin()
        sim.initialize()
        rng = np.random.default_rng(1 + rank)
        sim.set_tracers(rng.uniform(-1, 1, size=(512, 2)))
        return sim, 2 * np.pi / 120, f"simple-spin {m}x{m} fluid_2d::step_forward, dt of solve(2pi,120)"
    if workload == "flag2048":
        # The flag scenario (ftest.cc:335-378) on 3456 x 1152 square cells of
        # [-1,5]x[-1,1] (about 2048^2 cells; 1152 = 9 x 2^7 lets the periodic
        # direction halve seven times); mass ratio 1, bending rigidity 0.1,
        # Re 100, aspect ratio 10.
        n = FLAG_N
        m = 3 * n
        mu, k_B, Re, ar = 1.0, 0.1, 100.0, 10.0
        w = 1.0 / ar
        sim = capi.Simulation(m, n, ax=-1.0, bx=5.0, ay=-1.0, by=1.0, visc=1.0 / Re, ntrace=0,
                              precision=prec, y_prd=True, horiz_flow=1.0)
        # the learned warm start trains on a run whose tail is perturbed
        # (ftest's optional perturb_v), a different trajectory
        sim.add_flag(0.0, 0.0, 1.0, w, 0.25 * w, 4 * k_B / w ** 3, mu / w, perturb_v=0.2 if training else 0.0,
                     ntrace=17)
        sim.initialize()
        return sim, 30.0 / 900, (f"flag {m}x{n} on [-1,5]x[-1,1] (mu 1, k_B 0.1, Re 100, ar 10), FEM with "
                                 f"zero-pressure outlet, y-periodic; fluid_2d::step_forward, dt of 900 frames over T=30")
    m, n = SED_M, 2 * SED_M
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
    return sim, 0.1, (f"sediment {m}x{n}: 32 seeded circles and ellipses (r 0.03-0.06, rho 1.5-3, G 1) "
                      f"settling, fluid_2d::step_forward, dt of 0.1 frames")


LEARNED_SIM_FACTOR = 8     # network grid: the projection's unknowns restricted by 8
LEARNED_SIM_SAMPLES = 200  # projections captured per system from the training run
LEARNED_SIM_STEPS = 1500   # Adam steps per network


def _frame_dt(sim, interval):
    l = int(interval / sim.dt_reg) + 1
    return interval / l


def _train_learned_sim(workload, rank, dev):
    """The learned warm start of the MAC and FEM projections, trained with
    this library's own U-Net kernels on samples the method generates: a
    training run of the workload (another seed; for the flag a perturbed
    tail) captures every projection's input and correction."""
    import torch
    from incrmt_b200 import capi, learned
    t0 = time.perf_counter()
    sim, interval, _ = _make_sim(workload, rank, capi.PREC_FP64, training=True)
    dt = _frame_dt(sim, interval)
    sim.step(dt, 10)
    data = learned.capture(sim, LEARNED_SIM_FACTOR, LEARNED_SIM_SAMPLES, dt, dev)
    sim.close()
    t_data = time.perf_counter() - t0
    nets, losses = {}, {}
    t1 = time.perf_counter()
    for sys, (X, T) in data.items():
        Xn, Tn, V = learned.normalise(X, T)
        net = capi.UNet(4, 16, seed=11 + sys)
        losses["mac" if sys == capi.SYS_MAC else "fem"] = learned.train(net, Xn, Tn, V, LEARNED_SIM_STEPS,
                                                                       seed=rank)
        nets[sys] = net
    torch.cuda.synchronize()
    H, W = data[capi.SYS_MAC][0].shape[1:3]
    info = {"network": f"two U-Nets (MAC, FEM), 4 levels, base 16 channels, {nets[0].num_params()} parameters "
                       f"each, BF16 activations, mma.sync tensor-core convolutions",
            "grid": f"{H}x{W} (projection restricted by {LEARNED_SIM_FACTOR})",
            "train_samples_per_system": LEARNED_SIM_SAMPLES, "train_steps": LEARNED_SIM_STEPS, "batch": 8,
            "final_loss": losses, "data_seconds": t_data, "train_seconds": time.perf_counter() - t1}
    return nets, info


def _plain_fp64_rate(workload, rank, steps, warmup, dev, coarse_refresh=1):
    """Steps/s and V-cycles per projection of the plain FP64 method on the
    same workload (the comparison of the learned + mixed line)."""
    import torch
    from incrmt_b200 import capi
    sim, interval, _ = _make_sim(workload, rank, capi.PREC_FP64)
    sim.set_coarse_refresh(coarse_refresh)
    dt = _frame_dt(sim, interval)
    ext = torch.cuda.ExternalStream(sim.stream(), device=dev)
    sim.step(dt, warmup)
    torch.cuda.synchronize()
    st0 = sim.stats()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    sim.step(dt, steps)
    e1.record(ext)
    torch.cuda.synchronize()
    st1 = sim.stats()
    sim.close()
    vc = ((st1.vcycles_mac - st0.vcycles_mac) + (st1.vcycles_fem - st0.vcycles_fem)) / (2.0 * steps)
    return steps / (e0.elapsed_time(e1) / 1e3), vc


def run_ours_sspin(args, ws, rank, local, dist):
    """Simulation steps on the GPU through the simulation C ABI."""
    import torch
    from incrmt_b200 import capi

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    prec = capi.PREC_MIXED if args.precision == "mixed" else capi.PREC_FP64
    nets, learned_info = None, None
    if args.learned:
        if args.workload not in ("sed1024", "flag2048"):
            raise SystemExit("--learned: the simulation workloads with a learned warm start are sed1024, flag2048")
        nets, learned_info = _train_learned_sim(args.workload, rank, dev)
    sim, interval, wl = _make_sim(args.workload, rank, prec)
    sim.set_coarse_refresh(args.coarse_refresh)
    dt = _frame_dt(sim, interval)
    if nets is not None:
        for sys, net in nets.items():
            sim.set_learned(sys, net, LEARNED_SIM_FACTOR, args.learned_rule)
    ext = torch.cuda.ExternalStream(sim.stream(), device=dev)
    sim.step(dt, args.warmup)
    torch.cuda.synchronize()
    _barrier(dist)
    torch.cuda.synchronize()
    st0 = sim.stats()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.cudart().cudaProfilerStart()
        e0.record(ext)
        sim.step(dt, args.steps)
        e1.record(ext)
        torch.cuda.synchronize()
        torch.cuda.cudart().cudaProfilerStop()
    ms = e0.elapsed_time(e1)
    st1 = sim.stats()
    _barrier(dist)
    torch.cuda.synchronize()
    ms_max = _max_over_ranks(dist, ms)
    value = ws * args.steps / (ms_max / 1e3)
    vc = ((st1.vcycles_mac - st0.vcycles_mac) + (st1.vcycles_fem - st0.vcycles_fem)) / (2.0 * args.steps)

    # Phase breakdown of a few extra steps, timed by CUDA events on the stream
    # (outside the timed region).
    sim.set_profiling(True)
    sim.step(dt, min(args.steps, 10))
    phases = {k: v / min(args.steps, 10) for k, v in sim.profile().items()}
    # Roofline of the projections' fine-level smoothing (the HBM-bound kernel
    # with the largest time share): every launch bracketed by CUDA events on
    # the simulation stream over a few more steps.
    sim.set_profiling(False, smoothers=True)
    sim.step(dt, min(args.steps, 10))
    sm_ms, sm_bytes, sm_launch = 0.0, 0.0, 0
    for which in (capi.SYS_MAC, capi.SYS_FEM):
        a, b, c = sim.smoother_profile(which)
        sm_ms, sm_bytes, sm_launch = sm_ms + a, sm_bytes + b, sm_launch + c
    sim.set_profiling(False)

    # End to end through the C ABI as fluid_2d::solve drives it: the steps of
    # one frame, then the frame's fields copied to host buffers (p, u, v for
    # the vorticity, X, Y, phi; fluid_2d::write_files, fluid_2d_io.cc:60-102).
    frame_fields = ["p", "u", "v", "X", "Y", "phi"]
    _barrier(dist)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sim.step(dt, args.steps)
    host = [sim.get(f) for f in frame_fields]
    e2e_s = time.perf_counter() - t0
    e2e_s = _max_over_ranks(dist, e2e_s)
    e2e = ws * args.steps / e2e_s
    d2h = sum(h.nbytes for h in host)

    if nets is not None:
        lst = {("mac" if s == capi.SYS_MAC else "fem"): sim.learned_stats(s) for s in nets}
        sim.close()
        for net in nets.values():
            net.close()
        plain_sps, plain_vc = _plain_fp64_rate(args.workload, rank, args.steps, args.warmup, dev, args.coarse_refresh)
        learned_info.update({
            "rule": "fall back to the previous solution when the guess raises the residual" if args.learned_rule == 0
                    else "fall back only when the energy-optimal step is not positive",
            "applied": {k: v.applied for k, v in lst.items()},
            "fallback": {k: v.fallback for k, v in lst.items()},
            "fallback_rate": {k: v.fallback / max(1, v.applied + v.fallback) for k, v in lst.items()},
            "plain_fp64_steps_per_s": plain_sps, "plain_fp64_vcycles_per_projection": plain_vc,
            "speedup_vs_plain_fp64": value / ws / plain_sps})
    if rank != 0:
        sim.close()
        return
    cpu = None
    if ws == 1 and not args.no_cpu_baseline:
        try:
            if args.workload == "sspin1024":
                sps, dts, vcr, thr = cpu_reference_sspin(1024, 40, 2)
                sample = (f"40 steps after 2 warm-up steps at 1024x1024 (reference sources + "
                          f"TGMG-API shim), OMP threads = {thr}")
            elif args.workload == "flag2048":
                sps, dts, vcr, thr = cpu_reference_flag(2, 0)
                sample = f"2 steps of the flag workload (reference sources + TGMG-API shim), OMP threads = {thr}"
            else:
                sps, dts, vcr, thr = cpu_reference_sed(2, 0)
                sample = (f"2 steps of the sediment workload with each ellipse replaced by a "
                          f"rounded rod (the reference has no ellipse), OMP threads = {thr}")
            cpu = {"value": sps, "unit": "steps/s", "cores": thr, "kind": "reference", "sample": sample}
        except Exception as e:
            cpu = {"value": None, "unit": "steps/s", "cores": 0, "kind": "reference",
                   "sample": f"unavailable: {e}"}
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if prec == capi.PREC_FP64 else "f64 state, f32 V-cycles in f64 defect correction",
        "data": "synthetic",
        "config": {"workload": wl, "precision": args.precision, "flush": "working set larger than L2",
                   "parallelism": f"replicas x{ws}", "coarse_refresh": args.coarse_refresh},
        "vcycles_per_projection": vc,
        "coarse_builds_per_step": (st1.coarse_builds - st0.coarse_builds) / args.steps,
        "phase_ms_per_step": phases,
        "march_sweeps_per_step": (st1.march_sweeps - st0.march_sweeps) / args.steps,
        "march_monotone_rebuilds": int(st1.march_monotone - st0.march_monotone),
        "extrap_sweeps_per_step": (st1.extrap_sweeps - st0.extrap_sweeps) / args.steps,
        # level-set points in the objects' rebuild windows over all objects' full grids
        "window_fraction": st1.window_points / max(1, sim.objects * (sim.m + 4) * (sim.n + 4)),
        "roofline": _roofline(f"{args.workload}_smooth", sm_ms, sm_bytes, sm_launch,
                              "k_smooth_rb / k_smooth_tile on the fine level of the MAC and FEM projections "
                              "(two Gauss-Seidel sweeps per launch)",
                              "updated unknowns x 2 sweeps x (3+c) x 8 B; c=2 MAC, 1 FEM"),
        "cpu_baseline": cpu,
        "e2e": {"value": e2e, "unit": "steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": int(d2h / args.steps),
                "note": "one frame of fields (p,u,v,X,Y,phi) copied to host per timed run"},
        "gpu_launches": int(st1.launches - st0.launches),
        "clocks": clk.summary(),
    }
    if learned_info is not None:
        line["learned"] = learned_info
        line["config"]["initial_guess"] = "learned warm start on the previous solution"

    print(json.dumps(line))
    sim.close()


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
    if args.workload in ("sspin1024", "sed1024", "flag2048"):
        return run_ours_sspin(args, ws, rank, local, dist)

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
                   "flush": "inputs larger than L2 (each array 134 MB)", "parallelism": f"replicas x{ws}"},
        "vcycles_per_projection": float(np.mean(vcs)),
        "roofline": _roofline("mac4096_smooth", kms, kbytes, klaunch,
                              "k_smooth_rb (fine-level red-black Gauss-Seidel, two sweeps per launch)",
                              "updated unknowns x 2 sweeps x (3+c) x 8 B, c=2 (MAC)"),
        "cpu_baseline": cpu,
        "e2e": {"value": e2e, "unit": "steps/s",
                "h2d_bytes_per_step": int(rho_h.numel() * 8 + (1 if net is not None else 2) * b_h.numel() * 8),
                "d2h_bytes_per_step": int(b_h.numel() * 8)},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
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
    ap.add_argument("--workload", default="sspin1024", choices=["sspin1024", "mac4096", "sed1024", "flag2048"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--coarse-refresh", type=int, default=16,
                    help="rebuild the projections' Galerkin coarse operators every K projections "
                         "(1: on every density change)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--learned", action="store_true",
                    help="mac4096: train the learned initial guess first and start every solve from it; "
                         "sed1024, flag2048: train the learned warm start of both projections on a training "
                         "run and apply it in every projection")
    ap.add_argument("--learned-rule", type=int, default=0, choices=[0, 1],
                    help="fallback rule of the simulation's learned warm start (0: when the guess raises the "
                         "residual, 1: when the energy-optimal step is not positive)")
    args = ap.parse_args()
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
