#!/usr/bin/env python
"""Benchmark of the Dusty FARGO-ADSG gas time step (AlgoGas) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload NAME]

One "step" is one DT of AlgoGas (all of its CFL substeps) on one disc.  The
metric is gas cell-updates/s in FP64: (substeps x Nrad x Nsec) / time.

ours       value   : device time (CUDA events recorded by the library on its
                     own stream around every DT), state resident in HBM; L2 is
                     flushed (256 MB write) before each timed DT.
           e2e     : the same DTs through the public C ABI with the state in
                     pinned host memory: upload of the four fields, one DT,
                     download of the four fields, per step (host wall clock).
           roofline: the dominant kernel's algorithmic bytes / its CUDA-event
                     time (per-stage events, separate profiled pass).
           cpu_baseline: the reference's own sequential build (oracle/_ref)
                     timed on this host, one core, on a bounded sample.
reference  the reference's own build on every host core, one independent copy
           of the workload per core (the reference has no intra-disc threading
           without MPI); value = total cell-updates / wall.

Multi-GPU: discs are independent (no exchange), so N ranks run N replicas;
value is the sum over ranks divided by the slowest rank's time ("weak").
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

WORKLOADS = {
    # isothermal 128 x 384 disc, q=1e-3 planet on a fixed circular orbit
    "iso_128x384": dict(par="iso_128x384.par", noise=1e-4, seed=0),
    # isothermal disc on the largest grid of the batched sweep (HBM-resident)
    "iso_768x2304": dict(par="iso_768x2304.par", noise=1e-4, seed=0),
    # adiabatic + beta cooling + self-gravity 512 x 1536 disc, q=5e-4 planet
    "adiabatic_sg_512x1536": dict(par="adiabatic_sg_512x1536.par", noise=1e-4, seed=0),
    # gas of the 128x384 disc on 256 x 768 with 200,000 Lagrangian particles
    # (turbulent kicks), particles drawn from the drand48 stream seeded with 1
    "dust_256x768": dict(par="dust_256x768.par", noise=1e-4, seed=0, dust_seed=1),
}
BATCH_DISCS, BATCH_SEED = 64, 2  # the batched sweep: 64 discs drawn from seed 2
DEFAULT_WORKLOAD = "adiabatic_sg_512x1536"
CONFIG_DIR = os.path.join(REPO, "dustyfargoadsg_b200", "configs")
FALLBACK_HBM_GBS = 6650.0

# Algorithmic bytes per cell of each stage (distinct fields read + written,
# 8 B each), isothermal / with energy equation.
STAGE_BYTES = {
    "cfl_forces": (32, 40), "potential": (8, 8), "soundspeed": (0, 24),
    "substep1": (64, 64), "viscous_terms": (56, 56), "viscous_update": (64, 64),
    "substep2": (40, 56), "substep3": (0, 80),
    "transport_radial": (64, 80), "transport_azimuthal": (80, 96),
    "transport_vr_boundary": (40, 40), "transport_ring_means": (8, 8),
}


def par_grid(path):
    """(NRAD, NSEC) of a .par file, read with the reference's rules
    (case-insensitive keys, '#' comments; src/Interpret.c:82-130)."""
    grid = {"NRAD": 64, "NSEC": 64}  # the reference's defaults, src/var.c
    with open(path) as f:
        for line in f:
            tok = line.replace("\t", " ").split()
            if len(tok) >= 2 and not tok[0].startswith("#") and tok[0].upper() in grid:
                grid[tok[0].upper()] = int(float(tok[1]))
    return grid["NRAD"], grid["NSEC"]


def _env_int(name, dflt):
    try:
        return int(os.environ.get(name, dflt))
    except ValueError:
        return dflt


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.QUERY,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def traffic_per_launch(workload, stage):
    """DRAM bytes per launch of `stage` from the committed ncu summary."""
    path = os.path.join(REPO, "profiles", "dram_traffic.json")
    try:
        with open(path) as f:
            return json.load(f)[workload][stage]
    except (OSError, KeyError, ValueError):
        return None


def cpu_baseline_sample(par_path, noise, seed, budget_s, cells, cores=1):
    """Time the reference's own build (oracle/_ref) on a bounded sample.

    Returns (cell_updates_per_s, description) or (None, reason)."""
    from tests import _oracle  # test infrastructure: the CPU baseline only, never the product path
    if not _oracle.have_oracle():
        return None, "oracle binary not built"
    # a short probe run measures the substep rate, then one bounded sample
    probe_sub = 3
    d, t, _ = _oracle.run_oracle(par_path, steps=1, noise=noise, seed=seed, dump_every=10 ** 9,
                                 max_substeps=probe_sub, timeout=600)
    rate1 = t["wall_s"] / max(t["substeps"], 1)
    nsub = max(probe_sub, int(budget_s / max(rate1, 1e-6)))
    procs, tmpdirs = [], []
    t0 = time.perf_counter()
    for c in range(cores):
        wd = tempfile.mkdtemp(prefix="fb_cpu_")
        tmpdirs.append(wd)
        procs.append(threading.Thread(target=_run_one, args=(par_path, noise, seed, nsub, wd)))
    for p in procs:
        p.start()
    for p in procs:
        p.join()
    wall = time.perf_counter() - t0
    results = []
    for wd in tmpdirs:
        tf = os.path.join(wd, "timing.json")
        if os.path.exists(tf):
            results.append(json.load(open(tf)))
    if len(results) != cores:
        return None, "oracle sample failed"
    total = sum(r["substeps"] * cells for r in results)
    if cores == 1:
        rate = total / results[0]["wall_s"]
    else:
        rate = total / max(r["wall_s"] for r in results)
    desc = "%d CFL substeps of the workload per process (time inside AlgoGas, init excluded)" % nsub
    return rate, desc


def _run_one(par_path, noise, seed, nsub, wd):
    from tests import _oracle
    try:
        _oracle.run_oracle(par_path, steps=10 ** 6, noise=noise, seed=seed, dump_every=10 ** 9,
                           max_substeps=nsub, workdir=wd, keep=True, timeout=1800)
    except Exception as exc:  # recorded as a failed sample
        print("oracle sample failed: %s" % exc, file=sys.stderr)


def run_reference(args, par_path, wl, cells):
    rank = _env_int("RANK", 0)
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    budget = float(os.environ.get("FB_REF_BUDGET_S", "20"))
    budget = max(1.0, budget * max(args.steps, 1) / 10.0)
    rate, desc = cpu_baseline_sample(par_path, wl["noise"], wl["seed"], budget, cells, cores=cores)
    if rate is None:
        print(json.dumps({"impl": "reference", "unavailable": desc}))
        return
    unit = "cell-updates/s"
    line = {
        "metric": "gas cell-updates/s FP64", "value": rate, "unit": unit, "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": args.workload, "nrad": wl["nrad"], "nsec": wl["nsec"]},
        "cpu_baseline": {"value": rate, "unit": unit, "cores": cores, "kind": "reference",
                         "sample": desc + "; %d concurrent copies, one per core" % cores},
        "e2e": {"value": rate, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=None, choices=sorted(WORKLOADS))
    ap.add_argument("--mode", default=None, choices=["parity", "fast"],
                    help="library build: parity (exact divisions, unfused multiply-adds, the reference's "
                         "rounding) or fast (fused multiply-adds, approximate-reciprocal slopes); both "
                         "meet the same parity tests")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-sweep measurement")
    ap.add_argument("--no-dropin", action="store_true",
                    help="skip the measurement through the reference's own main (drop-in AlgoGas)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.workload is None:
        args.workload = DEFAULT_WORKLOAD
    wl = dict(WORKLOADS[args.workload])
    par_path = os.path.join(CONFIG_DIR, wl["par"])

    if args.impl == "reference":
        # the reference arm runs the reference's own build only: the package
        # (and its shared library) is not imported in this process
        grid = par_grid(par_path)
        wl["nrad"], wl["nsec"] = grid
        run_reference(args, par_path, wl, grid[0] * grid[1])
        return

    # the fast build is the benchmarked one: it meets the same parity tests
    # (one DT at 1e-11, 100 orbits at 1e-8, the full-size workloads)
    os.environ["FB_MODE"] = args.mode or os.environ.get("FB_MODE", "fast")
    import dustyfargoadsg_b200 as fb
    from dustyfargoadsg_b200 import _ffi
    args.mode = _ffi.default_mode()
    p = fb.read_par(par_path)
    wl["nrad"], wl["nsec"] = p.nrad, p.nsec
    cells = p.nrad * p.nsec

    import numpy as np
    import torch
    rank = _env_int("RANK", 0)
    world = _env_int("WORLD_SIZE", 1)
    local = _env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    fb.select_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from dustyfargoadsg_b200 import tune
    table = tune.load_table()
    disc = fb.Disc(p, noise=wl["noise"], seed=wl["seed"], dust_seed=wl.get("dust_seed"), tuning=table)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        disc.step()
    # --- timed region: K DTs, device time from CUDA events ---------------
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    launches0 = disc.kernel_launches()
    ms_total, substeps = 0.0, 0
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        rep = disc.step()
        ms_total += rep.gpu_ms
        substeps += rep.substeps
    barrier()
    clk = clocks.stop()
    launches = disc.kernel_launches() - launches0
    t_local = ms_total / 1e3
    if dist is not None:
        t = torch.tensor([t_local, float(substeps)], dtype=torch.float64, device="cuda")
        tmax = t.clone()
        dist.all_reduce(tmax[:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[1:], op=dist.ReduceOp.SUM)
        t_max, sub_all = float(tmax[0]), float(t[1])
    else:
        t_max, sub_all = t_local, float(substeps)
    value = sub_all * cells / t_max

    # --- e2e: host pinned state through the public API --------------------
    pinned = {k: torch.empty(disc.nf, dtype=torch.float64, pin_memory=True) for k in disc.fields}
    arrays = {k: v.numpy() for k, v in pinned.items()}
    disc.download()
    for k in arrays:
        arrays[k][:] = disc.fields[k]
    import ctypes as C
    for k, a in arrays.items():
        setattr(disc.st, k, a.ctypes.data_as(C.POINTER(C.c_double)))
    barrier()
    e2e_wall, e2e_sub = 0.0, 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        fb.check(disc.lib.fb_upload(disc.ctx, C.byref(disc.st), None), "fb_upload", disc.ctx)
        rep = disc.step()
        fb.check(disc.lib.fb_download(disc.ctx, C.byref(disc.st), C.c_uint(fb.FB_F_ALL)), "fb_download", disc.ctx)
        e2e_wall += time.perf_counter() - t0
        e2e_sub += rep.substeps
    if dist is not None:
        t = torch.tensor([e2e_wall, float(e2e_sub)], dtype=torch.float64, device="cuda")
        tm = t.clone()
        dist.all_reduce(tm[:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[1:], op=dist.ReduceOp.SUM)
        e2e_wall, e2e_sub = float(tm[0]), float(t[1])
    e2e_value = e2e_sub * cells / e2e_wall
    fbytes = disc.nf * 8 * len(arrays)
    d2h_extra = 0
    if disc.npart > 0:
        # the particles are outputs too: time their download once per step
        t0 = time.perf_counter()
        for _ in range(args.steps):
            disc.dust()
        e2e_wall_d = time.perf_counter() - t0
        e2e_value = e2e_sub * cells / (e2e_wall + e2e_wall_d)
        d2h_extra = disc.npart * 8 * len(disc.DUST_ARRAYS)

    # --- profiled pass: per-stage CUDA events -> roofline ------------------
    disc.profile(True)
    for _ in range(max(3, args.steps // 2)):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        disc.step()
    prof = disc.profile_read()
    disc.profile(False)
    energy = 1 if p.energy_equation else 0
    peak, peak_kind = measured_peak()
    best = None
    stages = {}
    # one radial pass per substep: the substeps of the profiled DTs (a stage
    # may launch several kernels per substep, so its time per pass is its
    # total over the substeps, not over its launches)
    nsub = prof.get("transport_radial", (0.0, 0))[1]
    for name, (ms, cnt) in prof.items():
        if cnt <= 0 or ms <= 0:
            continue
        per_launch_ms = ms / cnt
        stages[name] = {"ms_per_launch": per_launch_ms, "launches": cnt}
        if nsub > 0:
            stages[name]["ms_per_substep"] = ms / nsub
        if best is None or ms > prof[best][0]:
            best = name
    roofline = None
    if best is not None:
        bpc = STAGE_BYTES.get(best, (None, None))[energy]
        ms, cnt = prof[best]
        if nsub > 0:
            cnt = nsub  # the time of one pass of the stage
        units = cells
        if best == "dust_particles":
            # per particle and substep: read r, th, vr, vth, size, St, flag and
            # write r, th, vr, vth, St (96 B); the grid gathers are L2 hits
            bpc, units = 96, disc.npart
            if nsub <= 0:
                cnt = cnt / (8 if p.dust_feel_turb else 2)  # launches per substep
        achieved = (bpc * units / (ms / cnt * 1e-3) / 1e9) if bpc else None
        roofline = {"bound": "hbm", "kernel": best, "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": (achieved / peak) if achieved else None,
                    "traffic": traffic_per_launch(args.workload, best),
                    "algorithmic_bytes_per_launch": bpc * units if bpc else None,
                    "peak_kind": peak_kind + " HBM copy bandwidth",
                    "share_of_step": ms / sum(v[0] for v in prof.values())}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, desc = cpu_baseline_sample(par_path, wl["noise"], wl["seed"], 15.0, cells, cores=1)
        if rate is not None:
            cpu = {"value": rate, "unit": "cell-updates/s", "cores": 1, "kind": "reference", "sample": desc}
        else:
            cpu = {"value": None, "unit": "cell-updates/s", "cores": 1, "kind": "reference", "sample": desc}

    dropin = None
    if rank == 0 and world == 1 and not args.no_dropin:
        dropin = measure_dropin(par_path, wl, cells, steps=max(3, min(args.steps, 10)))

    batch = None
    if rank == 0 and world == 1 and not args.no_batch:
        batch = measure_batch(fb, table, flush, cpu_baseline=not args.no_cpu_baseline)

    if rank == 0:
        line = {
            "metric": "gas cell-updates/s FP64", "value": value, "unit": "cell-updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_max * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded white noise on the initial density)",
            "config": {"workload": args.workload, "nrad": p.nrad, "nsec": p.nsec,
                       "substeps_per_step": sub_all / world / args.steps,
                       "parallelism": "replicas%d" % world, "build": args.mode,
                       "l2": "flushed (256 MB write) before every timed step"},
            "e2e": {"value": e2e_value, "unit": "cell-updates/s", "h2d_bytes_per_step": fbytes,
                    "d2h_bytes_per_step": fbytes + d2h_extra},
            "gpu_launches": launches,
            "roofline": roofline,
            "stages": stages,
            "cpu_baseline": cpu,
            "clocks": clk,
        }
        if disc.npart > 0:
            line["config"]["particles"] = disc.npart
            line["particle_updates_per_s"] = disc.npart * sub_all / t_max
        if batch is not None:
            line["batched"] = batch
        if dropin is not None:
            line["dropin"] = dropin
        print(json.dumps(line))
    disc.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def measure_batch(fb, table, flush, warmup=2, steps=3, cpu_baseline=True):
    """The batched sweep: 64 discs of uneven grids and parameters (seed 2),
    one graph launch per DT for all of them; orbits/s summed over discs."""
    import torch
    from dustyfargoadsg_b200 import sweep
    wd = tempfile.mkdtemp(prefix="fb_batch_")
    discs = sweep.make_discs(sweep.draw_discs(BATCH_DISCS, BATCH_SEED), wd, tuning=table)
    try:
        with fb.Batch(discs) as batch:
            for _ in range(warmup):
                batch.step()
            ms, cell_updates, launches0 = 0.0, 0, sum(d.kernel_launches() for d in discs)
            for _ in range(steps):
                flush.fill_(1.0)
                torch.cuda.synchronize()
                reps = batch.step()
                ms += reps[0].gpu_ms
                cell_updates += sum(r.substeps * d.nr * d.ns for r, d in zip(reps, discs))
            launches = sum(d.kernel_launches() for d in discs) - launches0
            subs_per_dt = [r.substeps for r in reps]
        orbits = BATCH_DISCS * steps * sweep.orbits_per_dt(discs[0].p)
        out = {"metric": "batched orbits/s", "value": orbits / (ms / 1e3), "unit": "orbits/s",
               "discs": BATCH_DISCS, "seed": BATCH_SEED, "steps": steps, "warmup": warmup,
               "cell_updates_per_s": cell_updates / (ms / 1e3), "ms_per_step": ms / steps,
               "gpu_launches": launches, "graph_launches_per_step": 1,
               "grids": sorted({"%dx%d" % (d.nr, d.ns) for d in discs})}
        if cpu_baseline:
            cells = [d.nr * d.ns for d in discs]
            out["cpu_baseline"] = batch_cpu_baseline(wd, cells, subs_per_dt, sweep.orbits_per_dt(discs[0].p))
        return out
    finally:
        for d in discs:
            d.close()


def measure_dropin(par_path, wl, cells, steps, warmup=2):
    """The workload through the reference's own main() with AlgoGas answered
    by the library (oracle/_ref/fargo_dropin, built from
    dustyfargoadsg_b200/host/algogas_dropin.c): wall time of the reference's
    time loop per DT, its planet logs and every host-side step between the
    AlgoGas calls included, after `warmup` DTs (graph capture, first SG)."""
    from tests import _oracle  # test infrastructure: runs the drop-in binary
    if not os.path.exists(_oracle.DROPIN_BIN):
        return {"unavailable": "drop-in binary not built"}
    env = dict(os.environ, ORACLE_TIMING_SKIP=str(warmup))
    keep = dict(os.environ)
    os.environ.update(env)
    try:
        _, t, _ = _oracle.run_oracle(par_path, steps=warmup + steps, noise=wl["noise"], seed=wl["seed"],
                                     dump_every=10 ** 9, binary=_oracle.DROPIN_BIN, timeout=1800,
                                     extra_keys={"Ninterm": 10 ** 6})
    finally:
        os.environ.clear()
        os.environ.update(keep)
    wall, calls, sub = t["loop_wall_s"], t["loop_calls"], t["loop_substeps"]
    return {"metric": "gas cell-updates/s FP64 through the reference's main", "value": sub * cells / wall,
            "unit": "cell-updates/s", "ms_per_dt": wall * 1e3 / calls, "dts": calls, "warmup_dts": warmup,
            "substeps": sub,
            "how": "oracle/_ref/fargo_dropin: the reference's main(), per-DT planet logs (UpdateLog, and "
                   "UpdateLogSG after the loop's self-gravity call, both fed by the GPU) and the host fields "
                   "downloaded only where the loop reads them; wall clock of the loop"}


def batch_cpu_baseline(wd, cells, subs_per_dt, orbits_per_dt, budget_s=24.0):
    """The batched sweep on the host: one process of the reference's own
    build (oracle/_ref) per disc, as many at once as there are cores, each
    timed on a bounded sample of its own substeps (time inside AlgoGas).
    One DT of a disc costs its substeps per DT (as the GPU took them) at its
    measured substep rate; the cores share the discs, so one DT of every disc
    takes the sum of those costs over the cores.  Orbits/s counts the orbits
    of all discs, like the GPU figure."""
    import concurrent.futures as cf

    from tests import _oracle  # test infrastructure: the CPU baseline only
    if not _oracle.have_oracle():
        return {"value": None, "unit": "orbits/s", "kind": "reference", "sample": "oracle binary not built"}
    cores = os.cpu_count() or 1
    n = len(cells)
    per_disc = budget_s * min(cores, n) / n
    guess = 4.0e6  # cell-updates/s of one core, only to size the samples

    def one(d):
        nsub = max(2, int(per_disc * guess / cells[d]))
        w = tempfile.mkdtemp(prefix="fb_bcpu_")
        _, t, _ = _oracle.run_oracle(os.path.join(wd, "disc%03d.par" % d), steps=10 ** 6, noise=1e-4, seed=0,
                                     dump_every=10 ** 9, max_substeps=nsub, workdir=w, keep=True, timeout=1800)
        return t

    with cf.ThreadPoolExecutor(max_workers=cores) as ex:
        timings = list(ex.map(one, range(n)))
    # seconds one core needs for one DT of each disc; the cores share the
    # discs, so one DT of all of them takes their sum over the cores
    t_dt = [max(s, 1) * t["wall_s"] / t["substeps"] for t, s in zip(timings, subs_per_dt)]
    value = n * orbits_per_dt / (sum(t_dt) / min(cores, n))
    return {"value": value, "unit": "orbits/s", "cores": cores, "kind": "reference",
            "sample": "each of the %d discs run alone by the reference's build for about %.1f s of substeps "
                      "(%d at a time); a DT of a disc costs its substeps per DT (as the GPU took them) at its "
                      "measured substep rate, and the %d cores share the %d discs' DTs"
                      % (n, per_disc, min(cores, n), min(cores, n), n)}


if __name__ == "__main__":
    main()
