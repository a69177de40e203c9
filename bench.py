"""Benchmark: node-stage updates per second of the fdfault time-stepping path.

Workload (default): the 3D planar strike-slip rupture -- two blocks of
401x201x201 nodes (h = 0.1 km) split by a vertical y-normal fault, slip
weakening with a seeded log-normal static-friction field (mean 0.677, sd 0.03,
2 km correlation length), 20x15 km frictional region, 2x2 km nucleation patch,
RK3 -- in FP32 fields with FP64 friction.  One "step" is one full RK3 time step
(3 stages) over all 32,401,602 nodes.  Inputs are synthetic (seeded); no
dataset is involved.

Usage:  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                        [--decomp replicas|slabs]
Under torchrun each rank runs by default its own replica of the problem on its
own GPU, so ``value`` is the sum over ranks of node-stage updates divided by the
slowest rank's time (weak scaling).  With ``--decomp slabs`` the ranks split
one problem into x slabs and swap ghost planes over NCCL after every stage
(fdfault_b200.slabs): ``value`` is the whole grid's node-stages over the
slowest rank's time (strong scaling).
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "node-stage updates/s"
WORKLOAD = dict(nx=401, ny=201, nz=201, h=0.1)
# reduced instance of the same problem for ncu captures: the full-size cross-section
# (the same 26 x 7 tiles per plane) over half the planes; 16.2M nodes, 2.4 GB
PROFILE_WORKLOAD = dict(nx=201, ny=201, nz=201, h=0.1)
CPU_SAMPLE = dict(nx=101, ny=51, nz=51, h=0.4)
PROFILE_TRAFFIC = {1: os.path.join(HERE, "profiles", "volume_fast3d_planar3d.md"),
                   3: os.path.join(HERE, "profiles", "volume_regwindow3d_planar3d.md")}
# steps of the end-to-end run (the workload itself runs 1500; the state upload
# at its start is spread over these steps in h2d_bytes_per_step)
E2E_STEPS = 300
PLANAR_WORKLOAD_NAME = "planar3d: 2 blocks 401x201x201, slip weakening, log-normal mus, RK3 at CFL 0.2"
KERNEL_NAMES = {0: "volume_exact", 1: "volume_tiled3d", 2: "volume_staged3d", 3: "volume_regwindow3d"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=0)
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the other workloads (FP64 planar, 2D FP64, STZ, ensemble, rough) that a full-size "
                         "single-GPU run records under 'extras'")
    ap.add_argument("--size", default="full", choices=["full", "profile"],
                    help="profile: 2x201x101x101 instance for ncu captures")
    ap.add_argument("--config", default="planar", choices=["planar", "stz", "mode2", "ensemble", "rough"],
                    help="stz: planar STZ fault, plain vs learned Newton start; mode2: 2D mode-II "
                         "rupture in FP64; ensemble: 256 2D ruptures of uneven sizes, batched; rough: "
                         "rough fault with plasticity, two blocks of 601x301x301, FP32")
    ap.add_argument("--members", type=int, default=256, help="ensemble members (all ranks together)")
    ap.add_argument("--decomp", default="replicas", choices=["replicas", "slabs"],
                    help="planar workload on N GPUs: replicas (each rank its own copy, weak scaling) or "
                         "slabs (one problem split along x, ghost planes exchanged over NCCL after every "
                         "stage, strong scaling)")
    ap.add_argument("--volume-kernel", type=int, default=3, choices=[0, 1, 2, 3],
                    help="FP32 3D volume kernel: 0 reference order, 1 tiled, 2 staged (TMA), "
                         "3 register window (TMA-staged planes, default)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


REF_TIMEOUT_S = 300   # a reference run in a CPU-baseline sample never holds the GPU longer than this


def wait_bounded(proc, timeout=REF_TIMEOUT_S):
    """Wait for a reference process; kill it and raise if it runs past `timeout` seconds."""
    try:
        proc.wait(timeout=timeout)
    except subprocess.TimeoutExpired:
        proc.kill()
        proc.wait()
        raise RuntimeError("reference sample ran longer than %d s" % timeout)


def build_problem(workdir, nt, **size):
    from fdfault_b200 import problems as P

    prob = P.planar3d(nt=nt, name="planar3d", datadir=workdir + "/", workdir=workdir, seed=1234, cfl=P.WORKLOAD_CFL_3D,
                      nx=size["nx"], ny=size["ny"], nz=size["nz"], h=size["h"])
    return prob.write(os.path.join(workdir, "planar3d.in")), prob


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    path = os.path.join(HERE, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            v = json.load(fh)["hbm_gbs"]
        return float(v), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(kind):
    """DRAM bytes per node-stage of volume kernel `kind` from its committed ncu summary, or None."""
    try:
        with open(PROFILE_TRAFFIC[kind]) as fh:
            for line in fh:
                if line.startswith("traffic_bytes_per_node_stage:"):
                    return float(line.split(":")[1].split()[0])
    except Exception:
        pass
    return None


def cpu_reference_sample(workdir, nsteps, nproc):
    """Runs the reference solver (or, without its binary, the C oracle) on a
    bounded sample of the workload: nproc concurrent single-process runs of a
    101x51x51-per-block instance of the same problem, each timing only its
    time-stepping loop.  Returns (node-stage/s aggregate, kind, cores, seconds)."""
    import oracle

    runs = []
    for r in range(nproc):
        d = os.path.join(workdir, "cpu%d" % r)
        os.makedirs(d, exist_ok=True)
        infile, prob = build_problem(d, nsteps, **CPU_SAMPLE)
        runs.append((d, infile, prob))
    nodes = CPU_SAMPLE["nx"] * (2 * CPU_SAMPLE["ny"]) * CPU_SAMPLE["nz"]
    if os.path.exists(oracle.REF_BIN):
        kind = "reference"
        procs = []
        for d, infile, _ in runs:
            tf = os.path.join(d, "timing.txt")
            env = dict(os.environ, FDF_REF_TIMING=tf)
            procs.append((subprocess.Popen([oracle.REF_BIN, infile], cwd=d, env=env, stdout=subprocess.DEVNULL,
                                           stderr=subprocess.DEVNULL), tf))
        secs = []
        for p, tf in procs:
            wait_bounded(p)
            with open(tf) as fh:
                secs.append(float(fh.read().split()[-1]))
    else:
        kind = "port"
        code = ("import sys,time; sys.path.insert(0,%r); import oracle; o=oracle.Oracle(sys.argv[1]); "
                "t=time.perf_counter(); o.run(int(sys.argv[2])); print(time.perf_counter()-t)") % HERE
        procs = [subprocess.Popen([sys.executable, "-c", code, infile, str(nsteps)], stdout=subprocess.PIPE,
                                  text=True) for _, infile, _ in runs]
        secs = [float(p.communicate(timeout=REF_TIMEOUT_S)[0].split()[-1]) for p in procs]
    total = nodes * 3 * nsteps * nproc
    return total / max(secs), kind, nproc, max(secs)


def cpu_workers(bytes_per_run=512 << 20):
    """Host threads to use: all cores, bounded by memory (bytes_per_run per sample run)."""
    n = os.cpu_count() or 1
    try:
        mem = os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_PHYS_PAGES")
        n = min(n, max(1, int(0.8 * mem // bytes_per_run)))
    except (ValueError, OSError):
        pass
    return max(1, min(n, 128))


REF_FULL_BYTES = 10 << 30   # resident memory of one reference process on the full planar grid (9.0 GB measured)


def run_reference_arm(args, rank, world):
    """The reference solver on the host cores, on the same workload as the GPU
    arm: the full planar grid (two blocks of 401x201x201, the identical .in
    file), one process per core (bounded by memory), each timing one RK3 step
    of its own copy; the value is all processes' node-stages over the slowest
    process's time-stepping loop.  A full-grid step takes about a minute per
    process, so the arm times one sample whatever --steps is."""
    if rank != 0:
        return
    import oracle

    nproc = cpu_workers(REF_FULL_BYTES)
    tmp = tempfile.mkdtemp(prefix="fdf_refarm_")
    nodes = WORKLOAD["nx"] * 2 * WORKLOAD["ny"] * WORKLOAD["nz"]
    runs = []
    for r in range(nproc):
        d = os.path.join(tmp, "r%d" % r)
        os.makedirs(d, exist_ok=True)
        infile, _ = build_problem(d, 1, **WORKLOAD)
        runs.append((d, infile))
    if os.path.exists(oracle.REF_BIN):
        kind = "reference"
        procs = []
        for d, infile in runs:
            tf = os.path.join(d, "timing.txt")
            procs.append((subprocess.Popen([oracle.REF_BIN, infile], cwd=d, env=dict(os.environ, FDF_REF_TIMING=tf),
                                           stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL), tf))
        secs = []
        for pr, tf in procs:
            wait_bounded(pr, timeout=900)
            with open(tf) as fh:
                secs.append(float(fh.read().split()[-1]))
    else:
        kind = "port"
        code = ("import sys,time; sys.path.insert(0,%r); import oracle; o=oracle.Oracle(sys.argv[1]); "
                "t=time.perf_counter(); o.run(1); print(time.perf_counter()-t)") % HERE
        procs = [subprocess.Popen([sys.executable, "-c", code, infile], stdout=subprocess.PIPE, text=True)
                 for _, infile in runs]
        secs = [float(pr.communicate(timeout=900)[0].split()[-1]) for pr in procs]
    value = nodes * 3 * nproc / max(secs)
    sample = ("%d concurrent single-process runs of the full workload (2x401x201x201, the same input file), one "
              "RK3 step each; time-stepping loop only (slowest %.1f s)" % (nproc, max(secs)))
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": "node-stage/s", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * max(secs),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": PLANAR_WORKLOAD_NAME, "nodes": nodes, "stages_per_step": 3,
                      "timed_rk3_steps_per_process": 1, "processes": nproc},
           "cpu_baseline": {"value": value, "unit": "node-stage/s", "cores": nproc, "kind": kind, "sample": sample},
           "e2e": {"value": value, "unit": "node-stage/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def run_stz(args, local):
    """Planar STZ workload (two blocks of 401x201x201, per-node f0 and chi0):
    samples from a plain run, GPU training of the initial-guess network, then
    the same steps timed with the plain and with the learned Newton start,
    each compared with the FP64 plain run."""
    import torch

    from fdfault_b200 import problems as P
    from fdfault_b200 import solver as fs

    torch.cuda.set_device(local)
    size = WORKLOAD if args.size == "full" else PROFILE_WORKLOAD
    ncollect, epochs = 24, 20
    nrun = args.warmup + args.steps + 2
    tmp = tempfile.mkdtemp(prefix="fdf_stz_")
    prob = P.stz3d(nt=max(ncollect, nrun) + 2, name="stz3d", datadir=tmp + "/", workdir=tmp, cfl=P.WORKLOAD_CFL_3D,
                   **size)
    infile = prob.write(os.path.join(tmp, "stz3d.in"))
    with fs.Problem(infile, precision=fs.FP32, device=local) as p:
        p.stz_collect(2_400_000)
        p.step(ncollect)
        cnt = p.stz_sample_count()
        p.mlp_init(7)
        t0 = time.perf_counter()
        tr, va = p.mlp_train(epochs=epochs, batch=8192, lr=2e-3, seed=3)
        p.synchronize()
        train_s = time.perf_counter() - t0
        params = p.mlp_params()
    runs = {}
    keys = (fs.U, fs.V, fs.S, fs.STATE)
    # the learned start and its judges: the reference's midpoint start, a warm
    # start from each node's previous root, and the exact derivative
    starts = {"plain": fs.Problem.STZ_MIDPOINT, "learned": fs.Problem.STZ_LEARNED, "warm": fs.Problem.STZ_WARM,
              "exact_derivative": fs.Problem.STZ_EXACT_DERIVATIVE}
    for mode, code in starts.items():
        with fs.Problem(infile, precision=fs.FP32, device=local) as q:
            q.mlp_set_params(params)
            q.stz_start(code)
            q.step(args.warmup)
            q.synchronize()
            q.profile(True)
            ms = q.time_steps(args.steps)
            if_ms, if_n = q.profile_read(1)
            vol_ms, vol_n = q.profile_read(0)
            q.profile(False)
            q.stz_counting(True)
            q.step(2)
            solves, iters, mid = q.stz_counts()
            runs[mode] = dict(ms_per_step=ms / args.steps, interface_ms_per_stage=if_ms / max(if_n, 1),
                              volume_ms_per_launch=vol_ms / max(vol_n, 1), newton_solves=solves,
                              newton_iterations_per_solve=iters / max(solves, 1), midpoint_starts=mid,
                              fault={w: q.fault(0, w) for w in keys}, nodes=q.nxyz, nstages=q.nstages)
    with fs.Problem(infile, precision=fs.FP64, device=local) as r:
        r.step(nrun)
        ref = {w: r.fault(0, w) for w in keys}

    def rel(a, b):
        nb = float(np.linalg.norm(b))
        return float(np.linalg.norm(a - b)) / (nb if nb > 0 else 1.0)

    names = {fs.U: "slip", fs.V: "slip_rate", fs.S: "shear_stress", fs.STATE: "state"}
    for mode in runs:
        runs[mode]["rel_l2_vs_fp64"] = {names[w]: rel(runs[mode]["fault"][w], ref[w]) for w in keys}
    learned_vs_plain = {names[w]: rel(runs["learned"]["fault"][w], runs["plain"]["fault"][w]) for w in keys}
    for mode in runs:
        del runs[mode]["fault"]
    nodes, nst = runs["plain"]["nodes"], runs["plain"]["nstages"]
    out = {"metric": METRIC, "value": nodes * nst / (runs["learned"]["ms_per_step"] * 1e-3), "unit": "node-stage/s",
           "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32 fields, f64 friction", "data": "synthetic",
           "config": {"workload": "stz3d: 2 blocks %dx%dx%d, STZ per-node f0 and chi0, learned Newton start"
                                  % (size["nx"], size["ny"], size["nz"]), "nodes": nodes},
           "training": {"samples": cnt, "collected_over_steps": ncollect, "epochs": epochs, "seconds": train_s,
                        "train_loss": tr, "heldout_loss": va},
           "plain": runs["plain"], "learned": runs["learned"],
           "judges": {"warm": runs["warm"], "exact_derivative": runs["exact_derivative"]},
           "learned_vs_plain_rel_l2": learned_vs_plain}
    print(json.dumps(out), flush=True)


def run_mode2(args, local):
    """2D plane-strain mode-II rupture in FP64 (two blocks of 401x201, RK3, 1000
    steps in the reference's configuration): device time of --steps steps, the
    same steps through the C-ABI from host memory, and the reference solver on
    the host cores for a sample of the same problem."""
    import torch

    from fdfault_b200 import problems as P
    from fdfault_b200 import solver as fs

    torch.cuda.set_device(local)
    tmp = tempfile.mkdtemp(prefix="fdf_mode2_")
    nt = args.warmup + 2 * args.steps + 2
    prob = P.mode2_rupture(nx=401, ny=201, h=0.1, nt=nt, name="mode2", datadir=tmp + "/")
    infile = prob.write(os.path.join(tmp, "mode2.in"))
    with fs.Problem(infile, precision=fs.FP64, device=local) as p:
        nodes, nst = p.nxyz, p.nstages
        p.step(args.warmup)
        p.synchronize()
        clocks = ClockSampler(local)
        clocks.start()
        ms = p.time_steps(args.steps)   # default path: each step replayed from a one-step CUDA graph
        clk = clocks.stop()
        p.profile(True)   # per-kernel event times: a separate pass, launched kernel by kernel
        p.step(min(args.steps, 20))
        vol_ms, vol_n = p.profile_read(0)
        if_ms, if_n = p.profile_read(1)
        p.profile(False)
        # end to end: the state starts from host memory; the fault arrays come back every
        # step into pinned buffers, each copy queued behind its step
        state = [torch.from_numpy(p.field(c)).pin_memory() for c in range(p.nfields)]
        outs = [torch.empty(p.fault_count(0, w), dtype=torch.float64, pin_memory=True).numpy()
                for w in (fs.V, fs.S)]
        t0 = time.perf_counter()
        for c in range(p.nfields):
            p.set_field(c, state[c].numpy())
        for _ in range(args.steps):
            p.step(1)
            p.fault_async(0, fs.V, outs[0])
            p.fault_async(0, fs.S, outs[1])
        p.synchronize()
        te = time.perf_counter() - t0
    value = nodes * nst * args.steps / (ms * 1e-3)
    bps = 200
    out = {"metric": METRIC, "value": value, "unit": "node-stage/s", "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": "mode2: 2 blocks 401x201, slip weakening, RK3, FP64", "nodes": nodes,
                      "l2": "resident in L2 (32 MB per stage): not graded against HBM"},
           "clocks": clk,
           "e2e": {"value": nodes * nst * args.steps / te, "unit": "node-stage/s",
                   "h2d_bytes_per_step": 8.0 * nodes * len(state) / args.steps,
                   "d2h_bytes_per_step": 2 * 8 * 401},
           "kernel_ms": {"volume_avg": vol_ms / max(vol_n, 1), "volume_launches": vol_n,
                         "interface_avg_per_stage": if_ms / max(if_n, 1)},
           # all node-stages of the profiled pass over its total volume-kernel time (one launch
           # covers both blocks)
           "roofline": {"bound": "latency",
                        "achieved_gbs": bps * nodes * nst * min(args.steps, 20) / (vol_ms * 1e-3) / 1e9,
                        "algorithmic_bytes_per_node_stage": bps}}
    if not args.no_cpu_baseline:
        nproc = cpu_workers()
        runs = []
        for r in range(nproc):
            d = os.path.join(tmp, "cpu%d" % r)
            os.makedirs(d, exist_ok=True)
            pr = P.mode2_rupture(nx=401, ny=201, h=0.1, nt=60, name="mode2", datadir=d + "/")
            runs.append((d, pr.write(os.path.join(d, "mode2.in"))))
        import oracle
        if os.path.exists(oracle.REF_BIN):
            procs = []
            for d, f in runs:
                tf = os.path.join(d, "timing.txt")
                procs.append((subprocess.Popen([oracle.REF_BIN, f], cwd=d, env=dict(os.environ, FDF_REF_TIMING=tf),
                                               stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL), tf))
            secs = []
            for pp, tf in procs:
                wait_bounded(pp)
                with open(tf) as fh:
                    secs.append(float(fh.read().split()[-1]))
            out["cpu_baseline"] = {"value": nodes * 3 * 60 * nproc / max(secs), "unit": "node-stage/s",
                                   "cores": nproc, "kind": "reference",
                                   "sample": "%d concurrent single-process runs of the same problem, 60 RK3 steps "
                                             "each; time-stepping loop only (%.1f s)" % (nproc, max(secs))}
    print(json.dumps(out), flush=True)


def run_ensemble(args, rank, world, local):
    """256 2D mode-II slip-weakening ruptures, blocks of 101x51 ... 801x401
    nodes (log-uniform), per-member friction and nucleation: batched launches
    replayed from CUDA graphs, tiles from the autotuner.  Members are split
    across ranks (no collective); the aggregate is all members' node-stages
    over the slowest rank's device time."""
    import torch

    from fdfault_b200 import problems as P
    from fdfault_b200 import solver as fs

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    tune_steps = 2
    nt = tune_steps * 6 + args.warmup + args.steps + 24
    tmp = tempfile.mkdtemp(prefix="fdf_ens_%d_" % rank)
    allfiles = P.ensemble_members(n=args.members, seed=2024, workdir=tmp, nt=nt)
    from fdfault_b200 import replicas

    files = replicas.partition(allfiles, rank, world)
    t0 = time.perf_counter()
    ens = fs.Ensemble(files, device=local)
    setup_s = time.perf_counter() - t0
    threads, tile = ens.autotune(tune_steps)
    ens.run(args.warmup)
    per_step = ens.node_stages_per_step()
    clocks = ClockSampler(local)
    clocks.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ms = ens.time_steps(args.steps)
    torch.cuda.synchronize()
    clk = clocks.stop()
    total, ms = replicas.reduce_totals(float(per_step * args.steps), ms, device="cuda")
    ens.check_status()
    # the same members stepped one problem at a time through their own handles
    nsingle = 8
    t1 = time.perf_counter()
    for i in range(ens.size):
        ens.member(i).step(nsingle)
    for i in range(ens.size):
        ens.member(i).synchronize()
    single_s = time.perf_counter() - t1
    single_rate = per_step * nsingle / single_s
    out = {"metric": METRIC, "value": total / (ms * 1e-3), "unit": "node-stage/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32 fields, f64 friction",
           "data": "synthetic",
           "config": {"workload": "ensemble: %d 2D mode-II ruptures, blocks 101x51..801x401 log-uniform"
                                  % args.members, "members_per_rank": len(files),
                      "node_stages_per_step": per_step, "parallelism": "members split across ranks" if world > 1
                      else "single", "setup_s": setup_s, "autotuned": {"threads": threads, "tile": tile}},
           "clocks": clk,
           "one_problem_at_a_time": {"value": single_rate, "unit": "node-stage/s", "steps": nsingle,
                                     "note": "rank 0's members stepped one after another through their own "
                                             "handles (per-problem launches and graphs), wall clock"},
           "gpu_launches": args.steps * (3 * 2 + 1)}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        nproc = cpu_workers()
        procs = []
        import oracle
        sample = allfiles[:nproc]
        secs = []
        nodes_sample = 0
        if os.path.exists(oracle.REF_BIN):
            for f in sample:
                d = os.path.dirname(f)
                name = os.path.splitext(os.path.basename(f))[0]
                src = open(f).read().split("\n")
                src[3] = "20"   # [fdfault.problem] nt
                g = os.path.join(d, name + "_cpu.in")
                with open(g, "w") as fh:
                    fh.write("\n".join(src))
                tf = os.path.join(d, name + "_timing.txt")
                procs.append((subprocess.Popen([oracle.REF_BIN, g], cwd=d, env=dict(os.environ, FDF_REF_TIMING=tf),
                                               stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL), tf))
            for pp, tf in procs:
                wait_bounded(pp)
                with open(tf) as fh:
                    secs.append(float(fh.read().split()[-1]))
            for f in sample:
                src = open(f).read().split("\n")
                nxs = [int(v) for v in src[src.index("[fdfault.domain]") + 3].split()]
                nodes_sample += nxs[0] * nxs[1] * nxs[2]
            out["cpu_baseline"] = {"value": nodes_sample * 3 * 20 / max(secs), "unit": "node-stage/s", "cores": nproc,
                                   "kind": "reference",
                                   "sample": "the first %d members run concurrently by the reference solver, one "
                                             "process each, 20 RK3 steps; time-stepping loop only (%.1f s)"
                                             % (nproc, max(secs))}
    ens.close()
    if rank == 0:
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_rough(args, local):
    """Rough-fault rupture with Drucker-Prager plasticity and depth-dependent
    stress, two blocks of 601x301x301 nodes (109 M), FP32 fields: device time
    of --steps steps (graph replay), per-kernel times from a profiled pass,
    and the reference solver on the host cores for a reduced instance."""
    import torch

    from fdfault_b200 import problems as P
    from fdfault_b200 import solver as fs

    torch.cuda.set_device(local)
    size = dict(nx=601, ny=301, nz=301, h=0.1) if args.size == "full" else dict(nx=201, ny=101, nz=101, h=0.3)
    tmp = tempfile.mkdtemp(prefix="fdf_rough_")
    t0 = time.perf_counter()
    prob = P.rough3d(nt=args.warmup + args.steps + 8, name="rough3d", datadir=tmp + "/", workdir=tmp,
                     cfl=P.WORKLOAD_CFL_3D, **size)
    infile = prob.write(os.path.join(tmp, "rough3d.in"))
    gen_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    p = fs.Problem(infile, precision=fs.FP32, device=local)
    setup_s = time.perf_counter() - t0
    # the reference's return-map loop never ends on blocks deeper than
    # trunc(lambda + 2/3 G) + 1 = 54 z nodes (its z index holds the bulk
    # modulus, block.cpp:451-524): this workload runs the every-node rule
    p.set_plastic_rule(fs.Problem.PLASTIC_EVERY_NODE)
    vk = p.set_volume_kernel(args.volume_kernel)
    fast = vk != 0
    nodes, nst, nblocks = p.nxyz, p.nstages, int(np.prod(p.nblocks))
    p.step(args.warmup)
    p.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    ms = p.time_steps(args.steps)
    clk = clocks.stop()
    p.profile(True)
    p.step(min(args.steps, 6))
    vol_ms, vol_n = p.profile_read(0)
    if_ms, if_n = p.profile_read(1)
    p.profile(False)
    p.synchronize()
    bps = p.bytes_per_node_stage()
    vmax = float(np.max(p.fault(0, fs.V)))
    p.close()
    peak, peak_kind = measured_peak()
    vol_avg = vol_ms / max(vol_n, 1)
    achieved = bps * nodes / nblocks / (vol_avg * 1e-3) / 1e9
    out = {"metric": METRIC, "value": nodes * nst * args.steps / (ms * 1e-3), "unit": "node-stage/s", "n_gpus": 1,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32 fields, f64 friction", "data": "synthetic",
           "config": {"workload": "rough3d: 2 blocks %dx%dx%d, rough fault, Drucker-Prager plasticity, "
                                  "depth-dependent stress" % (size["nx"], size["ny"], size["nz"]), "nodes": nodes,
                      "generate_s": gen_s, "setup_s": setup_s, "max_slip_rate": vmax,
                      "plastic_rule": "every node, exact bulk modulus (the reference's own loop does not "
                                      "terminate on blocks of more than 54 z nodes)"},
           "clocks": clk,
           "kernel_ms": {"volume_avg": vol_avg, "volume_launches": vol_n,
                         "interface_avg_per_stage": if_ms / max(if_n, 1)},
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                        "peak_source": peak_kind, "kernel": KERNEL_NAMES[vk],
                        "algorithmic_bytes_per_node_stage": bps}}
    if not args.no_cpu_baseline:
        import oracle
        if os.path.exists(oracle.REF_BIN):
            nproc = min(cpu_workers(), 8)
            procs, secs = [], []
            # the reference finishes only on blocks of at most 54 z nodes (above,
            # its return-map loop does not terminate); at 61x31x31 it applies
            # the return map on the first z plane of each block
            small = dict(nx=61, ny=31, nz=31, h=1.0)
            for r in range(nproc):
                d = os.path.join(tmp, "cpu%d" % r)
                os.makedirs(d, exist_ok=True)
                pr = P.rough3d(nt=3, name="rough_cpu", datadir=d + "/", workdir=d, **small)
                f = pr.write(os.path.join(d, "rough_cpu.in"))
                tf = os.path.join(d, "timing.txt")
                procs.append((subprocess.Popen([oracle.REF_BIN, f], cwd=d, env=dict(os.environ, FDF_REF_TIMING=tf),
                                               stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL), tf))
            for pp, tf in procs:
                wait_bounded(pp)
                with open(tf) as fh:
                    secs.append(float(fh.read().split()[-1]))
            n_small = small["nx"] * 2 * small["ny"] * small["nz"]
            out["cpu_baseline"] = {"value": n_small * 3 * 3 * nproc / max(secs), "unit": "node-stage/s",
                                   "cores": nproc, "kind": "reference",
                                   "sample": "%d concurrent single-process runs of the workload at 61x31x31 per "
                                             "block, 3 RK3 steps each; time-stepping loop only (%.1f s); the "
                                             "reference's return map covers only the first z plane there"
                                             % (nproc, max(secs))}
    print(json.dumps(out), flush=True)


EXTRAS = [
    ("planar3d_fp64", ["--precision", "fp64", "--steps", "10", "--warmup", "3", "--e2e-steps", "20"]),
    ("mode2_fp64", ["--config", "mode2", "--steps", "100", "--warmup", "10"]),
    ("stz_learned", ["--config", "stz", "--steps", "10", "--warmup", "3"]),
    ("ensemble_256", ["--config", "ensemble", "--steps", "20", "--warmup", "3"]),
    ("rough_plastic", ["--config", "rough", "--steps", "6", "--warmup", "2"]),
]
EXTRA_KEYS = ("value", "unit", "ms_per_step", "dtype", "config", "roofline", "kernel_ms", "e2e", "plain", "learned",
              "learned_vs_plain_rel_l2", "training", "one_problem_at_a_time", "judges")


def run_extras():
    """The other workloads, each as its own bench.py process (one GPU, bounded
    time): their JSON lines, trimmed, keyed by workload; a failure is recorded
    and does not stop the others."""
    res = {}
    for name, argv in EXTRAS:
        cmd = [sys.executable, os.path.join(HERE, "bench.py"), "--no-cpu-baseline", "--no-extras"] + argv
        t0 = time.perf_counter()
        try:
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
            lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
            if r.returncode != 0 or not lines:
                res[name] = {"error": "rc %d: %s" % (r.returncode, (r.stderr or r.stdout).strip()[-300:])}
                continue
            d = json.loads(lines[-1])
            res[name] = {k: d[k] for k in EXTRA_KEYS if k in d}
        except Exception as e:   # noqa: BLE001 - recorded, the headline stands
            res[name] = {"error": repr(e)[:300]}
        res[name]["wall_s"] = time.perf_counter() - t0
    return res


def run_slabs(args, rank, world, local):
    """The planar workload split into ``world`` x slabs, one per GPU (strong
    scaling): every rank steps stage by stage on one CUDA stream and swaps its
    edge planes with its neighbours over NCCL after each stage
    (fdfault_b200.slabs).  value = the whole grid's node-stages / the slowest
    rank's device time."""
    import datetime

    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist.barrier()   # communicator set up before the first point-to-point exchange
    from fdfault_b200 import replicas, slabs
    from fdfault_b200 import solver as fs

    precision = fs.FP32 if args.precision == "fp32" else fs.FP64
    tmp = tempfile.mkdtemp(prefix="fdf_slab_%d_" % rank)
    ke = args.e2e_steps if args.e2e_steps > 0 else max(E2E_STEPS, 5 * args.steps)
    infile, _ = build_problem(tmp, args.warmup + args.steps + ke + 30,
                              **(WORKLOAD if args.size == "full" else PROFILE_WORKLOAD))
    p = fs.Problem(infile, precision=precision, device=local)
    vk = p.set_volume_kernel(args.volume_kernel)
    nodes, nstages, nblocks = p.nxyz, p.nstages, int(np.prod(p.nblocks))
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        run = slabs.SlabRun(p, rank, world, transport=slabs.DistTransport(rank, world) if world > 1 else None)
        owned = (run.x1 - run.x0) * (nodes // p.nx[0])
        run.step(args.warmup)
        torch.cuda.synchronize()
        clocks = ClockSampler(local)
        clocks.start()
        time.sleep(0.3)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run.step(args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        ms = e0.elapsed_time(e1)
        clk = clocks.stop()
        # per-kernel event times of this rank's volume stage
        p.profile(True)
        run.step(min(args.steps, 20))
        vol_ms, vol_n = p.profile_read(0)
        p.profile(False)
        p.synchronize()
        # end to end: state upload from pinned host memory, then steps with this
        # rank's on-fault arrays read back into pinned buffers after every step
        fields = [torch.empty(nodes, dtype=torch.float64, pin_memory=True) for _ in range(p.nfields)]
        for c in range(p.nfields):
            fields[c].numpy()[:] = p.field(c)
        outs = [torch.empty(p.fault_count(0, w), dtype=torch.float64, pin_memory=True)
                for w in (fs.V, fs.U, fs.S, fs.SN, fs.VX, fs.SX)]
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for c in range(p.nfields):
            p.set_field(c, fields[c].numpy())
        for _ in range(ke):
            run.step(1)
            for w, o in zip((fs.V, fs.U, fs.S, fs.SN, fs.VX, fs.SX), outs):
                p.fault_async(0, w, o.numpy())
        p.synchronize()
        te = time.perf_counter() - t0
    work, ms = replicas.reduce_totals(float(owned * nstages * args.steps), ms, device="cuda")
    e2e_work, te = replicas.reduce_totals(float(owned * nstages * ke), te, device="cuda")
    bps = p.bytes_per_node_stage()
    peak, peak_kind = measured_peak()
    vol_avg_ms = vol_ms / max(vol_n, 1)
    achieved = bps * owned / nblocks / (vol_avg_ms * 1e-3) / 1e9
    vol_per_stage = {0: 1, 1: 2 * nblocks, 2: nblocks, 3: 2 * nblocks + 1}[vk]
    launches = args.steps * nstages * (vol_per_stage + p.nifaces + 2 * len(run.sides))
    out = {"metric": METRIC, "value": work / (ms * 1e-3), "unit": "node-stage/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
           "scaling": "strong", "vs_baseline": None, "dtype": "f32" if precision == fs.FP32 else "f64",
           "data": "synthetic",
           "config": {"workload": PLANAR_WORKLOAD_NAME if args.size == "full" else "planar3d profile size",
                      "nodes": nodes, "stages_per_step": nstages, "parallelism": "x slabs %s" % run.slabs,
                      "ghost_bytes_per_stage_rank0": run.ghost_bytes_per_exchange,
                      "l2": "inputs larger than L2"},
           "clocks": clk,
           "e2e": {"value": e2e_work / te, "unit": "node-stage/s",
                   "h2d_bytes_per_step": 8 * nodes * p.nfields / ke,
                   "d2h_bytes_per_step": sum(o.numel() * 8 for o in outs), "steps": ke},
           "gpu_launches": launches,
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak, "peak_source": peak_kind, "kernel": KERNEL_NAMES[vk],
                        "algorithmic_bytes_per_node_stage": bps, "traffic": None}}
    run.release()
    p.close()
    if rank == 0:
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "b200" and args.config == "planar" and args.decomp == "slabs":
        run_slabs(args, rank, world, local)
        return
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return
    if args.config == "ensemble":
        run_ensemble(args, rank, world, local)
        return
    if args.config in ("stz", "mode2", "rough"):
        if rank == 0:
            {"stz": run_stz, "mode2": run_mode2, "rough": run_rough}[args.config](args, local)
        return
    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from fdfault_b200 import solver as fs

    precision = fs.FP32 if args.precision == "fp32" else fs.FP64
    tmp = tempfile.mkdtemp(prefix="fdf_bench_%d_" % rank)
    nsteps_total = args.warmup + args.steps + max(args.e2e_steps, E2E_STEPS, 5 * args.steps) + 30
    infile, prob = build_problem(tmp, nsteps_total, **(WORKLOAD if args.size == "full" else PROFILE_WORKLOAD))
    t_setup = time.perf_counter()
    p = fs.Problem(infile, precision=precision, device=local)
    t_setup = time.perf_counter() - t_setup
    vk = p.set_volume_kernel(args.volume_kernel)
    fast = vk != 0
    nodes = p.nxyz
    nstages = p.nstages
    nblocks = int(np.prod(p.nblocks))
    p.step(args.warmup)
    p.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ms = p.time_steps(args.steps)   # default path: each step replayed from a one-step CUDA graph
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    # per-kernel event times for the roofline: a separate pass, launched kernel by kernel
    p.profile(True)
    p.step(min(args.steps, 20))
    vol_ms, vol_n = p.profile_read(0)
    if_ms, if_n = p.profile_read(1)
    p.profile(False)
    p.synchronize()   # raises if any kernel reported a solver status
    from fdfault_b200 import replicas

    # replicas: every rank advances its own copy; work summed, time the slowest rank's
    node_stages, ms = replicas.reduce_totals(float(nodes * nstages * args.steps), ms, device="cuda")
    value = node_stages / (ms * 1e-3)

    # end to end through the C-ABI with host buffers: upload the state from
    # pinned host memory once, then run a stretch of the workload reading back
    # after every step, into preallocated pinned buffers, the on-fault output
    # arrays that the reference's output units write every step (V, U, S, Sn,
    # Vx, Sx); the upload is counted in the timed region and spread over the
    # steps in h2d_bytes_per_step
    ke = args.e2e_steps if args.e2e_steps > 0 else max(E2E_STEPS, 5 * args.steps)
    fields = [torch.empty(nodes, dtype=torch.float64, pin_memory=True) for _ in range(p.nfields)]
    for c in range(p.nfields):
        fields[c].numpy()[:] = p.field(c)
    outs = {w: torch.empty(p.fault_count(0, w), dtype=torch.float64, pin_memory=True)
            for w in (fs.V, fs.U, fs.S, fs.SN, fs.VX, fs.SX)}
    h2d = sum(f.numel() * 8 for f in fields)
    d2h = sum(o.numel() * 8 for o in outs.values())
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for c in range(p.nfields):
        p.set_field(c, fields[c].numpy())
    views = {w: o.numpy() for w, o in outs.items()}
    for _ in range(ke):
        p.step(1)
        for w, o in views.items():
            p.fault_async(0, w, o)
    p.synchronize()
    te = time.perf_counter() - t0
    e2e_work, te = replicas.reduce_totals(float(nodes * nstages * ke), te, device="cuda")
    e2e = e2e_work / te

    bps = p.bytes_per_node_stage()
    peak, peak_kind = measured_peak()
    vol_avg_ms = vol_ms / max(vol_n, 1)
    bytes_per_launch = bps * nodes / nblocks
    achieved = bytes_per_launch / (vol_avg_ms * 1e-3) / 1e9
    traffic_pn = profiled_traffic(vk)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": peak_kind, "kernel": KERNEL_NAMES[vk],
                "algorithmic_bytes_per_node_stage": bps,
                "traffic": (traffic_pn * nodes / nblocks) if traffic_pn else None}
    # per step: per stage the volume launches (tiled 3D: a marching and a face-node
    # kernel per block; register window: one pre-pass launch for all blocks (k-face
    # SAT increments, closure-plane x derivatives), then a marching and an x/y
    # face-node kernel per block; staged: one per block; reference order: one
    # for all blocks)
    # and one interface launch per interface, plus the graph's step-counter kernel;
    # one counter reset per call
    vol_per_stage = {0: 1, 1: 2 * nblocks, 2: nblocks, 3: 2 * nblocks + 1}[vk]
    launches = args.steps * (nstages * (vol_per_stage + p.nifaces) + 1) + 1
    out = {"metric": METRIC, "value": value, "unit": "node-stage/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32" if precision == fs.FP32 else "f64", "data": "synthetic",
           "config": {"workload": PLANAR_WORKLOAD_NAME if args.size == "full" else "planar3d profile size 2x201x201x201",
                      "nodes": nodes, "stages_per_step": nstages, "l2": "inputs larger than L2 (5.96 GB/stage)",
                      "parallelism": "replicas" if world > 1 else "single", "setup_s": t_setup},
           "clocks": clk,
           "e2e": {"value": e2e, "unit": "node-stage/s", "h2d_bytes_per_step": h2d / ke, "d2h_bytes_per_step": d2h,
                   "steps": ke, "note": "state uploaded once from pinned host memory (bytes spread over the "
                                        "steps); on-fault output arrays copied into pinned buffers after "
                                        "every step, queued behind the step (fdf_get_fault_async), all "
                                        "complete inside the timed region"},
           "gpu_launches": launches,
           "kernel_ms": {"volume_avg": vol_avg_ms, "volume_launches": vol_n,
                         "interface_avg_per_stage": if_ms / max(if_n, 1)},
           "roofline": roofline}
    p.close()
    if rank == 0 and world == 1 and args.size == "full" and not args.no_extras:
        out["extras"] = run_extras()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, kind, cores, secs = cpu_reference_sample(tempfile.mkdtemp(prefix="fdf_cpu_"), 16, cpu_workers())
        out["cpu_baseline"] = {"value": rate, "unit": "node-stage/s", "cores": cores, "kind": kind,
                               "sample": "%d concurrent single-process runs of the workload at 101x51x51 nodes per "
                                         "block, 16 RK3 steps each; time-stepping loop only (%.1f s)" % (cores, secs)}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
