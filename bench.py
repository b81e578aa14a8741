"""Benchmark of the SwinMD B200 step: ns/day of one system on each GPU.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload lj4000] [--precision fp64|mixed]

One "step" is one MD time step of the workload (pair list check/rebuild,
forces, leap-frog Nose-Hoover update, observables) on the device.  Timing:
W untimed warm-up steps, then K steps in chunks of --chunk steps; between
chunks a buffer larger than L2 is written (the state of one small system
fits in L2, so each chunk starts cold), CUDA events on the library's stream
bracket every chunk, with a device synchronize on both sides.  Under torchrun
every rank advances its own independent replica (the path does not shard a
single system: "replicas only"), the timed region is bracketed by barriers,
and the slowest rank's time is used.

The reference arm (--impl reference) times the reference's own C++ build
(oracle/_ref/ref_dump, single-threaded, no MPI in this image) on a bounded
sample of the same workload on the host CPU.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

METRIC = "ns/day on 1 B200: learned-guess+mixed vs plain GPU path at matched force error"
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM = 6650.0


def workload(name):
    from swinmd_b200 import systems
    if name == "lj4000":
        s = systems.lj_fluid(ncell=10, seed=1)
        s.config.long_correct = True
        desc = {"workload": "lj4000: Lennard-Jones fluid, 4000 atoms (FCC 10x10x10), rho*=0.8442, "
                            "T*=0.722, rc=2.5 sigma (energy-shifted), skin 0.3 sigma, leap-frog "
                            "Nose-Hoover tau*=0.5, dt*=0.005 (10.78 fs), argon units",
                "atoms": s.n_atoms}
        return s, desc
    raise SystemExit(f"unknown workload {name}")


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def flush_l2(buf):
    buf.add_(1.0)


def cpu_reference(s, steps, timeout=600):
    """Times the reference build (oracle/_ref/ref_dump run) for `steps` steps."""
    import refdump
    from swinmd_b200 import systems
    if not os.path.exists(refdump.REF_DUMP):
        return None
    with tempfile.TemporaryDirectory() as d:
        systems.write_reference_case(s, d)
        t0 = time.perf_counter()
        r = refdump.run_ref(d, "run", steps, out="run.txt", timeout=timeout)
        wall = time.perf_counter() - t0
    loop = float(r["run_seconds"][0]) if "run_seconds" in r else wall
    return {"seconds": loop, "steps": steps, "wall": wall}


def ns_per_day(sec_per_step, dt_ps):
    return dt_ps * 1e-3 * 86400.0 / sec_per_step


def run_reference_arm(args, rank, world):
    s, desc = workload(args.workload)
    dt = s.config.timestep
    if rank != 0:
        return
    steps = max(1, args.cpu_sample_steps)
    res = []
    for _ in range(args.warmup and 1):
        cpu_reference(s, max(1, steps // 10))
    for _ in range(max(1, min(args.steps, 3))):
        r = cpu_reference(s, steps)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_dump not built"}))
            return
        res.append(r["seconds"] / steps)
    sps = statistics.median(res)
    v = ns_per_day(sps, dt)
    out = {"metric": METRIC, "value": v, "unit": "ns/day", "impl": "reference",
           "n_gpus": world, "steps": len(res) * steps, "warmup": args.warmup,
           "ms_per_step": sps * 1e3, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": desc,
           "cpu_baseline": {"value": v, "unit": "ns/day", "cores": 1, "kind": "reference",
                            "sample": f"{steps} steps of {desc['workload'].split(':')[0]} per timing, "
                                      "median of runs; SwinMD's own LFIntegrator::run, one process, "
                                      "one core (no MPI in this image)"},
           "e2e": {"value": v, "unit": "ns/day", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--warmup", type=int, default=200)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="lj4000")
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--chunk", type=int, default=1000)
    ap.add_argument("--e2e-every", type=int, default=10)
    ap.add_argument("--cpu-sample-steps", type=int, default=1500)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))

    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        if dist:
            dist.destroy_process_group()
        return

    import torch
    from swinmd_b200 import engine
    torch.cuda.set_device(local)
    s, desc = workload(args.workload)
    dt = s.config.timestep
    ens = engine.GpuEnsemble(s, precision=args.precision, device=local)
    lf = engine.LFIntegrator(ens)
    lf.start()
    lf.run(args.warmup)
    o = lf.observables()
    l2 = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{local}")  # 256 MB > L2

    # --- device-resident timing ------------------------------------------
    chunk = min(args.chunk, args.steps)
    nchunks = max(1, args.steps // chunk)
    steps = nchunks * chunk
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(local)
    clk.start()
    total_ms = 0.0
    for _ in range(nchunks):
        flush_l2(l2)
        torch.cuda.synchronize()
        total_ms += lf.run_timed(chunk)  # CUDA events on the library's stream
    torch.cuda.synchronize()
    clocks = clk.stop()
    # device time of the same work with CUDA events on the library stream:
    # smd_profile_stages times each stage; the per-step device time is
    # their sum (list rebuilds scaled by their observed frequency)
    o_end = lf.observables()
    prof = np.zeros(4)
    L = engine.L
    L.check(ens.ctx, ens.lib.smd_profile_stages(ens.ctx, 50, L.dptr(prof)))
    t = torch.tensor([total_ms], dtype=torch.float64)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.barrier()
    ms = float(t[0])
    ms_per_step = ms / steps
    value = ns_per_day(ms_per_step * 1e-3, dt) * world

    # --- end to end through the public API, host buffers ------------------
    n = s.n_atoms
    pos = torch.empty(3 * n, dtype=torch.float64).pin_memory().numpy()
    vel = torch.empty(3 * n, dtype=torch.float64).pin_memory().numpy()
    st = ens.state()
    pos[:] = st["pos"].reshape(-1)
    vel[:] = st["vel"].reshape(-1)
    every = args.e2e_every
    e2e_steps = max(every, (min(steps, 5000) // every) * every)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps // every):
        ens.upload_positions(pos)
        ens.upload_velocities(vel)
        lf.run(every)
        st = ens.state()
        pos[:] = st["pos"].reshape(-1)
        vel[:] = st["vel"].reshape(-1)
        obs = lf.observables()
    torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - t0) * 1e3
    te = torch.tensor([e2e_ms], dtype=torch.float64)
    if dist:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = ns_per_day(float(te[0]) / e2e_steps * 1e-3, dt) * world
    h2d = (2 * 3 * n * 8) / every
    d2h = (3 * 3 * n * 8 + 400) / every

    # --- roofline of the dominant kernel (pair kernel) ------------------
    kcount = ctypes_int(ens, "smd_step_kernel_count")
    pairs = int(o_end.pairs_in_cutoff)
    # algorithmic bytes per launch: every list entry (4 B index + 16 B
    # neighbour position) and per site 16 B position + 24 B force
    from swinmd_b200 import engine as E
    list_entries = 2 * pairs_in_list(ens)
    alg_bytes = list_entries * 20 + n * 40
    pair_ms = float(prof[0])
    achieved = alg_bytes / (pair_ms * 1e-3) / 1e9
    peak, peak_kind = FALLBACK_HBM, "fallback"
    if os.path.exists(PEAKS):
        peak = float(json.load(open(PEAKS)).get("hbm_gbs", FALLBACK_HBM))
        peak_kind = "measured"
    gpu_launches = kcount * steps

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = cpu_reference(s, args.cpu_sample_steps)
        if r:
            cpu = {"value": ns_per_day(r["seconds"] / r["steps"], dt), "unit": "ns/day", "cores": 1,
                   "kind": "reference",
                   "sample": f"{r['steps']} steps of lj4000 with SwinMD's own LFIntegrator::run "
                             "(oracle/_ref/ref_dump), one process, one core"}

    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": "ns/day", "n_gpus": world, "steps": steps,
               "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f32" if args.precision == "mixed" else "f64",
               "data": "synthetic", "precision_mode": args.precision,
               "config": dict(desc, precision=args.precision, l2="flushed between chunks of "
                              f"{chunk} steps (256 MB write)", replicas=world,
                              parallelism="replicas only"),
               "e2e": {"value": e2e_value, "unit": "ns/day", "h2d_bytes_per_step": h2d,
                       "d2h_bytes_per_step": d2h,
                       "how": f"upload positions+velocities from pinned host, smd_run({every}), "
                              "download state + observables, every chunk"},
               "gpu_launches": gpu_launches,
               "stage_ms": {"pair": prof[0], "recip": prof[1], "integrate": prof[2],
                            "list_rebuild": prof[3]},
               "list_updates": int(o_end.list_updates), "pairs_in_cutoff": pairs,
               "roofline": {"bound": "hbm", "kernel": "k_pair", "achieved": achieved, "peak": peak,
                            "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                            "peak_source": peak_kind,
                            "alg_bytes_per_launch": alg_bytes},
               "clocks": clocks, "cpu_baseline": cpu}
        print(json.dumps(out))
    ens.close()
    if dist:
        dist.destroy_process_group()


def ctypes_int(ens, fn):
    import ctypes
    v = ctypes.c_int()
    from swinmd_b200 import _lib as L
    L.check(ens.ctx, getattr(ens.lib, fn)(ens.ctx, ctypes.byref(v)))
    return v.value


def pairs_in_list(ens):
    return int(ens.pairs().shape[0])


if __name__ == "__main__":
    main()
