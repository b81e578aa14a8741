"""Benchmark of the SwinMD B200 step: ns/day of one system on each GPU.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload polwater4096|lj4000|replicas64|water_replicas64|
                                water_shear_replicas64]

Default workload: rigid polarisable multipole water, 4096 molecules (12,288
sites), the configuration the headline metric is quoted on.  The seeded
start (random orientations) is equilibrated on the GPU first.  Arms, timed
one after another on the same trajectory:
  plain                  FP64 throughout, the same algorithms as the fast arm
                         (column reciprocal passes with exact integer phases,
                         product-form buffered 14-7), dipole solve started
                         from the molecule-block solution M^-1 E0;
  plain_reference_forms  the same FP64 arm with the reference's own forms
                         (one FP64 sine/cosine per (site, k), pow() 14-7);
  fast_network_off       mixed precision, solve started from the second-order
                         extrapolation 2 p(t-1) - p(t-2) + M^-1 (E0(t) -
                         2 E0(t-1) + E0(t-2)): the learned guess's base with
                         the network switched off;
  fast                   mixed precision + the learned guess (that base plus
                         the per-site network's correction; the network is
                         trained beforehand, on the GPU's tensor cores, on
                         dipoles the solver itself converged): the headline
                         `value`.
Every arm solves the dipoles to the same tolerance (RMS change 1e-6 D).  The
line also carries the solver's iterations from each guess, each arm's force
error against FP64 with the dipoles solved to 1e-13 e nm, pair interactions
per second and both arms' energy drift in an NVE run from the same state
(10^4 steps), with the same drift of the rigid SPC/E water configuration in
both precisions.

One "step" is one MD time step: pair-list check/rebuild, all forces (vdW,
multipoles, dipole solve, induced terms), SHAKE + Nose-Hoover update and
observables, on the device.  Timing: W untimed warm-up steps, then K steps
in chunks; before every chunk a 256 MB buffer (> L2) is written, and CUDA
events on the library's stream bracket each chunk with a device synchronize
on both sides.  Under torchrun every rank advances its own independent
replica (one system does not shard: "replicas only"); the timed region is
bracketed by barriers and the slowest rank's time is used.

The reference arm (--impl reference) times the reference's own C++ build
(oracle/_ref/ref_dump: LFIntegrator::start, then LFIntegrator::run) on the
same workload, single-threaded (the build has no MPI), bounded to one MD
step because one step of this size takes more than a minute.
"""
import argparse
import ctypes
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
FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}
DIPOLE_TOL = 2.0819e-8   # 1e-6 D in e nm
SERIES_CAP = 10000       # per-step samples kept for the energy drift


def workload(name, nmol=None):
    from swinmd_b200 import systems
    if name == "polwater4096":
        n = nmol or 4096
        s = systems.polarizable_water(nmol=n, kmax=18 if n == 4096 else max(6, int(round(18 * (n / 4096) ** (1 / 3)))),
                                      seed=1)
        desc = {"workload": f"polwater{n}: rigid polarisable multipole water, {n} molecules "
                            f"({3 * n} sites), charge+dipole+quadrupole sites, Thole a=0.39, "
                            "buffered 14-7 (H sites pulled 0.91 to O), Ewald alpha=3.5/nm, rc=0.9 nm, "
                            "|n|<18 (k set), induced dipoles to 1e-6 D RMS, SHAKE, Nose-Hoover 298 K, "
                            "dt=1 fs, 0.997 g/cm3",
                "sites": 3 * n}
        return s, desc
    if name == "lj4000":
        s = systems.lj_fluid(ncell=10, seed=1)
        s.config.long_correct = True
        desc = {"workload": "lj4000: Lennard-Jones fluid, 4000 atoms (FCC 10x10x10), rho*=0.8442, "
                            "T*=0.722, rc=2.5 sigma (energy-shifted), skin 0.3 sigma, leap-frog "
                            "Nose-Hoover tau*=0.5, dt*=0.005 (10.78 fs), argon units",
                "sites": s.n_atoms}
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
            threading.Thread(target=self._read, daemon=True).start()
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


def ns_per_day(sec_per_step, dt_ps):
    return dt_ps * 1e-3 * 86400.0 / sec_per_step


def cpu_reference(s, steps, timeout=1800):
    """Times the reference build (oracle/_ref/ref_dump run) for `steps` steps;
    returns seconds of LFIntegrator::run per step, or None."""
    import refdump
    from swinmd_b200 import systems
    if not os.path.exists(refdump.REF_DUMP):
        return None
    with tempfile.TemporaryDirectory() as d:
        systems.write_reference_case(s, d)
        r = refdump.run_ref(d, "run", steps, out="run.txt", timeout=timeout)
    return float(r["run_seconds"][0]) / steps


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    if args.workload in REPLICA_WORKLOADS:
        return run_reference_replicas(args, world)
    s, desc = workload(args.workload)
    # the reference's dense dipole matrix makes one polwater4096 step take
    # minutes on one core: one step is the bounded sample
    steps = max(1, min(args.steps, 1 if args.workload == "polwater4096" else 2000))
    sps = cpu_reference(s, steps, timeout=3600)
    if sps is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_dump is not built"}))
        return
    v = ns_per_day(sps, s.config.timestep)
    print(json.dumps({
        "metric": METRIC, "value": v, "unit": "ns/day", "impl": "reference", "n_gpus": world,
        "steps": steps, "warmup": 0, "ms_per_step": sps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": desc,
        "cpu_baseline": {"value": v, "unit": "ns/day", "cores": 1, "kind": "reference",
                         "sample": f"{steps} MD step(s) of the full workload after "
                                   "LFIntegrator::start; SwinMD's own LFIntegrator::run, one "
                                   "process, one core (the image has no MPI)"},
        "e2e": {"value": v, "unit": "ns/day", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def run_reference_replicas(args, world):
    """The reference on the replica workload: one SwinMD process per host core
    (the reference is single-threaded and runs replicas as separate runs),
    each a bounded number of steps of one replica at zero shear (it has no
    SLLOD); the aggregate is the sum of the concurrent processes' ns/day."""
    import refdump
    from concurrent.futures import ThreadPoolExecutor
    from swinmd_b200 import systems
    if not os.path.exists(refdump.REF_DUMP):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_dump is not built"}))
        return
    water = args.workload != "replicas64"
    flexible = args.workload == "water_shear_replicas64"
    reps = (systems.water_replica_set(count=64, seed=1, flexible=flexible) if water
            else systems.replica_set(count=64, seed=1))
    cores = max(1, min(64, os.cpu_count() or 1))
    steps = max(1, min(args.steps, 5 if water else 50))

    def one(s):
        s.config.rate = 0.0
        s.config.test_mode = 0
        with tempfile.TemporaryDirectory() as d:
            systems.write_reference_case(s, d)
            r = refdump.run_ref(d, "run", steps, out="run.txt", timeout=1800)
        return float(r["run_seconds"][0]) / steps

    with ThreadPoolExecutor(cores) as ex:
        sps = list(ex.map(one, reps[:cores]))
    dt = reps[0].config.timestep
    v = sum(ns_per_day(x, dt) for x in sps)
    metric = REPLICA_METRICS[args.workload]
    print(json.dumps({
        "metric": metric,
        "value": v, "unit": "ns/day", "impl": "reference", "n_gpus": world, "steps": steps, "warmup": 0,
        "ms_per_step": float(np.mean(sps)) * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": {"workload": args.workload},
        "cpu_baseline": {"value": v, "unit": "ns/day", "cores": cores, "kind": "reference",
                         "sample": f"{cores} concurrent SwinMD processes (one per core), {steps} steps "
                                   "each of the first replicas at zero shear (the reference has no SLLOD), "
                                   "LFIntegrator::run"},
        "e2e": {"value": v, "unit": "ns/day", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


REPLICA_WORKLOADS = ("replicas64", "water_replicas64", "water_shear_replicas64")
REPLICA_METRICS = {
    "replicas64": "aggregate ns/day of 64 batched LJ replicas (uneven sizes, per-replica shear and Nose-Hoover "
                  "chain)",
    "water_replicas64": "aggregate ns/day of 64 batched LJ/Ewald water replicas (uneven sizes, per-replica seeds "
                        "and Nose-Hoover thermostats)",
    "water_shear_replicas64": "aggregate ns/day of 64 batched LJ/Ewald water replicas (uneven sizes, per-replica "
                              "strain rates and Nose-Hoover chains)",
}


def run_replicas(args, rank, world, local):
    """64 independent replicas in one graph per step; aggregate ns/day over
    all replicas and ranks.  replicas64: LJ fluids (sizes log-uniform
    500-8000 atoms, strain rates uniform 0-0.2 reduced, own Nose-Hoover
    chains); water_replicas64: rigid LJ + Ewald waters (500-8000 molecules,
    own seeds and Nose-Hoover thermostats, SHAKE, zero shear);
    water_shear_replicas64: flexible LJ + Ewald waters (500-8000 molecules,
    strain rates uniform 0-0.2 reduced under SLLOD with the sheared Ewald
    sum, own Nose-Hoover chains)."""
    import torch
    from swinmd_b200 import engine, systems
    torch.cuda.set_device(local)
    water = args.workload != "replicas64"
    flexible = args.workload == "water_shear_replicas64"
    reps = (systems.water_replica_set(count=64, seed=1 + rank, flexible=flexible) if water
            else systems.replica_set(count=64, seed=1 + rank))
    ens, integ = [], []
    for s in reps:
        e = engine.GpuEnsemble(s, precision="mixed", device=local)
        nh = engine.LFIntegrator(e) if water and not flexible else engine.NHIntegrator(e)
        nh.start()
        ens.append(e)
        integ.append(nh)
    batch = engine.ReplicaBatch(ens)
    tpp = batch.autotune(reps=10)
    batch.run(args.warmup)
    l2 = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{local}")
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    clk = ClockSampler(local)
    clk.start()
    total, done = 0.0, 0
    while done < args.steps:
        k = min(args.chunk, args.steps - done)
        l2.add_(1.0)
        torch.cuda.synchronize()
        total += batch.run(k)
        done += k
    clocks = clk.stop()
    t = torch.tensor([total], dtype=torch.float64)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t[0]) / args.steps
    dt = reps[0].config.timestep
    value = ns_per_day(ms * 1e-3, dt) * len(reps) * world
    # per-replica force error of the mixed path against FP64
    errs = []
    for e in ens:
        f32, _, _ = e.compute_forces()
        e.set_precision("fp64")
        f64, _, _ = e.compute_forces()
        e.set_precision("mixed")
        errs.append(float(np.sqrt(((f32 - f64) ** 2).sum() / (f64 ** 2).sum())))
    # end to end: host buffers in and out around every block of steps
    every = args.e2e_every
    hb = []
    for e in ens:
        st = e.state()
        p = torch.empty(st["pos"].size, dtype=torch.float64).pin_memory().numpy()
        v = torch.empty(st["vel"].size, dtype=torch.float64).pin_memory().numpy()
        p[:] = st["pos"].reshape(-1)
        v[:] = st["vel"].reshape(-1)
        hb.append((p, v))
    e2e_steps = max(every, (min(args.steps, 100) // every) * every)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps // every):
        for e, (p, v) in zip(ens, hb):
            e.upload_positions(p)
            e.upload_velocities(v)
        batch.run(every)
        for e, (p, v) in zip(ens, hb):
            st = e.state()
            p[:] = st["pos"].reshape(-1)
            v[:] = st["vel"].reshape(-1)
    torch.cuda.synchronize()
    te = torch.tensor([(time.perf_counter() - t0) * 1e3], dtype=torch.float64)
    if dist:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e = ns_per_day(float(te[0]) / e2e_steps * 1e-3, dt) * len(reps) * world
    import ctypes
    launches = 0
    for e in ens:
        kc = ctypes.c_int()
        L_ = __import__("swinmd_b200._lib", fromlist=["_lib"])
        L_.check(e.ctx, e.lib.smd_step_kernel_count(e.ctx, ctypes.byref(kc)))
        launches += kc.value
    natoms = sum(s.n_atoms for s in reps)
    pairs = sum(int(integ[r].observables().pairs_in_cutoff) for r in range(len(reps)))
    # FP32 rate of the whole step over the pair work (23 flop per LJ pair,
    # 40 with the Ewald real-space term, in each direction of the full list):
    # a lower bound for the pair kernel
    achieved = pairs * 2 * (40 if water else 23) / (ms * 1e-3) / 1e12
    peak = 148 * 128 * 2 * 1.965e9 / 1e12
    cpu = None
    if rank == 0 and not args.no_cpu_baseline and water:
        if flexible:
            sample = systems.spce_flexible(nmol=512, box=2.4953, cutoff=0.9, kmax=6, seed=11, n_steps=20)
        else:
            sample = systems.spce_water(nmol=512, box=2.4953, cutoff=0.9, kmax=6, seed=11, n_steps=20)
        sps = cpu_reference(sample, 20)
        if sps:
            kind = "flexible" if flexible else "rigid"
            cpu = {"value": ns_per_day(sps, sample.config.timestep), "unit": "ns/day", "cores": 1,
                   "kind": "reference",
                   "sample": f"20 steps of one 512-molecule {kind} water at zero shear (the reference has "
                             "no SLLOD) with SwinMD's own LFIntegrator::run, one process, one core; 64 such "
                             "processes on 64 cores would give 64x this"}
    elif rank == 0 and not args.no_cpu_baseline:
        sample = systems.lj_fluid(ncell=8, seed=5, n_steps=50)
        sample.config.long_correct = True
        sps = cpu_reference(sample, 50)
        if sps:
            cpu = {"value": ns_per_day(sps, dt), "unit": "ns/day", "cores": 1, "kind": "reference",
                   "sample": "50 steps of one 2048-atom replica at zero shear with SwinMD's own "
                             "LFIntegrator::run (the reference has no SLLOD), one process, one core; "
                             "64 such processes on 64 cores would give 64x this"}
    if rank == 0 and flexible:
        nmol = sum(s.n_mols for s in reps)
        rates = [s.config.rate for s in reps]
        print(json.dumps({
            "metric": REPLICA_METRICS[args.workload],
            "value": value, "unit": "ns/day", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 pair and reciprocal math on exact fractions, f64 bonded terms and integrator",
            "data": "synthetic (seeded lattices, random orientations, Maxwell-Boltzmann velocities)",
            "config": {"workload": f"water_shear_replicas64: 64 flexible SPC/E-like waters, {nmol} molecules "
                                   "in total, sizes log-uniform 500-8000 molecules at 0.997 g/cm3, harmonic "
                                   "O-H bonds and H-O-H angle, LJ on O + Ewald (alpha 3.1/nm, rc 1.0 nm, kmax "
                                   "scaled with the box from 9 at 4.03 nm; the sheared cell's k list rebuilt "
                                   "every step), SLLOD with Lees-Edwards images at strain rates uniform 0-0.2 "
                                   "reduced (sigma_O sqrt(m/eps_O) = 1.666 ps), NH chain 298 K tau 0.1 ps, "
                                   "dt 0.5 fs; one CUDA graph per step over all replicas",
                       "replicas": len(reps) * world, "l2": "256 MB buffer written before every chunk",
                       "parallelism": "replicas only",
                       "strain_rate_per_ps": {"min": min(rates), "max": max(rates)}},
            "autotuned_threads_per_site": [int(x) for x in tpp],
            "force_rms_rel_err_vs_fp64": {"max": max(errs), "median": float(np.median(errs))},
            "e2e": {"value": e2e, "unit": "ns/day", "h2d_bytes_per_step": natoms * 6 * 8 / every,
                    "d2h_bytes_per_step": natoms * 9 * 8 / every},
            "gpu_launches": launches * args.steps,
            "roofline": {"bound": "fp32", "kernel": "k_pair (LJ + Ewald real) over the whole step",
                         "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                         "traffic": None, "peak_source": "nominal FP32 SIMT rate at the measured max SM clock"},
            "clocks": clocks, "cpu_baseline": cpu}))
    elif rank == 0 and water:
        nmol = sum(s.n_mols for s in reps)
        print(json.dumps({
            "metric": REPLICA_METRICS[args.workload],
            "value": value, "unit": "ns/day", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 pair and reciprocal math on exact fractions, f64 SHAKE and integrator",
            "data": "synthetic (seeded lattices, random orientations, Maxwell-Boltzmann velocities)",
            "config": {"workload": f"water_replicas64: 64 rigid SPC/E-like waters, {nmol} molecules in total, "
                                   "sizes log-uniform 500-8000 molecules at 0.997 g/cm3, LJ on O + Ewald "
                                   "(alpha 3.1/nm, rc 1.0 nm, kmax scaled with the box from 9 at 4.03 nm), "
                                   "SHAKE 1e-8, Nose-Hoover 298 K, dt 2 fs, zero shear (Ewald under shear "
                                   "is not built); one CUDA graph per step over all replicas",
                       "replicas": len(reps) * world, "l2": "256 MB buffer written before every chunk",
                       "parallelism": "replicas only"},
            "autotuned_threads_per_site": [int(x) for x in tpp],
            "force_rms_rel_err_vs_fp64": {"max": max(errs), "median": float(np.median(errs))},
            "e2e": {"value": e2e, "unit": "ns/day", "h2d_bytes_per_step": natoms * 6 * 8 / every,
                    "d2h_bytes_per_step": natoms * 9 * 8 / every},
            "gpu_launches": launches * args.steps,
            "roofline": {"bound": "fp32", "kernel": "k_pair (LJ + Ewald real) over the whole step",
                         "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                         "traffic": None, "peak_source": "nominal FP32 SIMT rate at the measured max SM clock"},
            "clocks": clocks, "cpu_baseline": cpu}))
    elif rank == 0:
        print(json.dumps({
            "metric": REPLICA_METRICS[args.workload],
            "value": value, "unit": "ns/day", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 pair math on exact fractions, f64 integrator",
            "data": "synthetic (seeded FCC lattices, Maxwell-Boltzmann velocities)",
            "config": {"workload": f"replicas64: 64 LJ fluids, {natoms} atoms in total, sizes log-uniform "
                                   "500-8000 atoms (FCC 4 ncell^3), rho*=0.8442, T*=0.722, rc=2.5 sigma, "
                                   "strain rates uniform 0-0.2 (SLLOD, Lees-Edwards), NH chain tau*=0.5, "
                                   "dt*=0.005; one CUDA graph per step over all replicas",
                       "replicas": len(reps) * world, "l2": "256 MB buffer written before every chunk",
                       "parallelism": "replicas only"},
            "autotuned_threads_per_site": [int(x) for x in tpp],
            "force_rms_rel_err_vs_fp64": {"max": max(errs), "median": float(np.median(errs))},
            "e2e": {"value": e2e, "unit": "ns/day", "h2d_bytes_per_step": natoms * 6 * 8 / every,
                    "d2h_bytes_per_step": natoms * 9 * 8 / every},
            "gpu_launches": launches * args.steps,
            "roofline": {"bound": "fp32", "kernel": "k_pair (LJ) over the whole step", "achieved": achieved,
                         "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak, "traffic": None,
                         "peak_source": "nominal FP32 SIMT rate at the measured max SM clock"},
            "clocks": clocks, "cpu_baseline": cpu}))
    batch.close()


def spce_drift(steps, equilibrate=2000):
    """NVE energy drift of rigid SPC/E water (2160 molecules in a 4.03 nm
    box, LJ on O, Ewald alpha 3.1/nm with |n| < 9, SHAKE tolerance 1e-8,
    dt 2 fs) in FP64 and in the mixed path from the same state, equilibrated
    with the Nose-Hoover thermostat first; and the mixed path's RMS relative
    force error against FP64 at that state."""
    from swinmd_b200 import engine, systems
    from swinmd_b200 import _lib as L
    s = systems.spce_water(nmol=2160, box=4.03, cutoff=1.0, kmax=9, seed=1)
    ens = engine.GpuEnsemble(s, precision="mixed")
    lf = engine.LFIntegrator(ens, series_capacity=SERIES_CAP)
    lf.start()
    lf.run(equilibrate)
    st0 = ens.state()
    ens.set_precision("fp64")
    f64, _, _ = ens.compute_forces()
    ens.set_precision("mixed")
    f32, _, _ = ens.compute_forces()
    err = float(np.sqrt(((f32 - f64) ** 2).sum() / (f64 ** 2).sum()))
    nve = lf.params
    nve.thermostat = L.THERMO_NONE
    L.check(ens.ctx, ens.lib.smd_set_integrator(ens.ctx, ctypes.byref(nve)))
    dt = s.config.timestep
    steps = min(steps, SERIES_CAP)
    out = {"workload": "spce2160: rigid SPC/E water, 2160 molecules, 4.03 nm box, LJ (O) + Ewald "
                       "alpha=3.1/nm |n|<9, rc=1.0 nm, SHAKE tol 1e-8, dt=2 fs, NVE after "
                       f"{equilibrate} Nose-Hoover steps at 298 K",
           "force_rms_rel_err_vs_fp64": err}
    for name, prec in (("plain", "fp64"), ("fast", "mixed")):
        ens.set_precision(prec)
        ens.upload_positions(st0["pos"])
        ens.upload_velocities(st0["vel"], st0["vtminus"])
        lf.run(steps)
        ser = lf.series()[-steps:]
        h = ser[:, 0] + ser[:, 1]
        tt = np.arange(steps) * dt * 1e-3   # ns
        fit = np.polyfit(tt, h, 1)
        out[name] = {"kj_mol_per_ns": float(fit[0]), "kj_mol_per_ns_per_molecule": float(fit[0]) / s.n_mols,
                     "rms_fluctuation_kj_mol": float(np.std(h - np.polyval(fit, tt))), "steps": steps}
    ens.close()
    return out


def timed_steps(lf, l2, steps, chunk):
    import torch
    total = 0.0
    done = 0
    while done < steps:
        k = min(chunk, steps - done)
        l2.add_(1.0)
        torch.cuda.synchronize()
        total += lf.run_timed(k)
        done += k
    return total


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="polwater4096")
    ap.add_argument("--chunk", type=int, default=100)
    ap.add_argument("--train-frames", type=int, default=2000)
    ap.add_argument("--train-every", type=int, default=1)
    ap.add_argument("--train-epochs", type=int, default=8)
    ap.add_argument("--e2e-every", type=int, default=10)
    ap.add_argument("--cpu-sample-mols", type=int, default=1024)
    ap.add_argument("--equilibrate", type=int, default=10000)
    ap.add_argument("--iter-steps", type=int, default=20)
    ap.add_argument("--drift-steps", type=int, default=10000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mlp-tensor-path", type=int, default=1, choices=[0, 1],
                    help="network inference on tcgen05 128-row tiles (1) or warp-level mma.sync tiles (0)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))

    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        if dist:
            dist.destroy_process_group()
        return
    if args.workload in REPLICA_WORKLOADS:
        run_replicas(args, rank, world, local)
        if dist:
            dist.destroy_process_group()
        return

    import torch
    from swinmd_b200 import engine
    from swinmd_b200 import _lib as L
    torch.cuda.set_device(local)
    s, desc = workload(args.workload)
    dt = s.config.timestep
    polar = args.workload == "polwater4096"
    t_setup = time.perf_counter()
    ens = engine.GpuEnsemble(s, precision="mixed", device=local)
    if polar:
        ens.set_solver(tol=DIPOLE_TOL, max_iter=500, guess=L.GUESS_FIRST_ORDER)
    lf = engine.LFIntegrator(ens, series_capacity=SERIES_CAP)
    lf.start()
    # equilibration from the seeded start (random orientations release a lot
    # of energy): mixed path, cheap
    lf.run(args.equilibrate)
    l2 = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{local}")  # 256 MB > L2

    train = {}
    if polar:
        # training rows: the solver's own converged dipoles along the trajectory
        ens.mlp_init(capacity_frames=args.train_frames, seed=1)
        ens.mlp_set_tensor_path(args.mlp_tensor_path)
        t0 = time.perf_counter()
        for _ in range(args.train_frames):
            lf.run(args.train_every)
            ens.compute_forces(L.TERM_IND_SHORT)
            ens.mlp_collect()
        t1 = time.perf_counter()
        loss = ens.mlp_train(epochs=args.train_epochs, batch=16384, lr=2e-3)
        train = {"frames": args.train_frames, "rows": args.train_frames * s.n_atoms,
                 "epochs": args.train_epochs, "final_mse": loss,
                 "inference": "tcgen05" if args.mlp_tensor_path else "mma.sync",
                 "collect_s": t1 - t0, "train_s": time.perf_counter() - t1}

    clk_all = ClockSampler(local)
    clk_all.start()

    def arm(precision, guess, reference_forms=False, steps=None):
        steps = steps or args.steps
        ens.set_precision(precision)
        ens.set_reference_forms(reference_forms)
        if polar:
            ens.set_solver(tol=DIPOLE_TOL, max_iter=500, guess=guess)
        lf.run(args.warmup)
        if dist:
            dist.barrier()
        o0 = lf.observables()
        clk = ClockSampler(local)
        clk.start()
        ms = timed_steps(lf, l2, steps, args.chunk)
        clocks = clk.stop()
        o1 = lf.observables()
        t = torch.tensor([ms], dtype=torch.float64)
        if dist:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        it = ens.solver_stats() if polar else (0, 0.0)
        ms_step = float(t[0]) / steps
        return {"value": ns_per_day(ms_step * 1e-3, dt) * world, "ms_per_step": ms_step,
                "solver_iterations": it[0], "dipole_rms_change_at_exit": it[1],
                "list_rebuilds_per_step": (o1.list_updates - o0.list_updates) / steps,
                "pairs_in_cutoff": int(o1.pairs_in_cutoff), "clocks": clocks}

    # plain: FP64 throughout, the same algorithms as the fast arm (column
    # reciprocal passes with exact integer phases, product-form 14-7), the
    # solve started from the molecule-block solution M^-1 E0
    plain = arm("fp64", L.GUESS_DIRECT)
    prof_plain = np.zeros(12)
    L.check(ens.ctx, ens.lib.smd_profile_stages(ens.ctx, 5, L.dptr(prof_plain)))
    # the same FP64 arm with the reference's own forms (pow() 14-7, one FP64
    # sine and cosine per (site, k)): what a direct GPU port of the reference
    # arithmetic runs at
    plain_ref = arm("fp64", L.GUESS_DIRECT, reference_forms=True, steps=max(10, args.steps // 4))
    ens.set_reference_forms(False)
    # fast without the network: mixed path, first-order guess
    network_off = arm("mixed", L.GUESS_EXTRAP2) if polar else None
    # fast: mixed path + learned guess (the headline)
    fast = arm("mixed", L.GUESS_LEARNED if polar else L.GUESS_DIRECT)
    clocks_all = clk_all.stop()
    prof = np.zeros(12)
    L.check(ens.ctx, ens.lib.smd_profile_stages(ens.ctx, 5, L.dptr(prof)))
    value = fast["value"]

    # iterations of the working-tolerance solve from each guess, step by step
    iters = {}
    if polar:
        for name, g in (("direct", L.GUESS_DIRECT), ("previous", L.GUESS_PREVIOUS),
                        ("first_order", L.GUESS_FIRST_ORDER), ("extrap2", L.GUESS_EXTRAP2),
                        ("extrap3", L.GUESS_EXTRAP3), ("learned", L.GUESS_LEARNED)):
            ens.set_solver(tol=DIPOLE_TOL, max_iter=500, guess=g)
            lf.run(3)
            its, first = [], []
            for _ in range(args.iter_steps):
                lf.run(1)
                its.append(ens.solver_stats()[0])
                first.append(ens.solver_trace()[0])
            iters[name] = {"mean": float(np.mean(its)), "min": int(min(its)), "max": int(max(its)),
                           "first_update_rms": float(np.exp(np.mean(np.log(first))))}

    # force error at matched dipole tolerance: each arm's evaluation of the
    # current configuration against FP64 with the dipoles solved to 1e-13 e nm
    force_err = {}
    n = s.n_atoms
    if polar:
        pos_now = ens.state()["pos"].copy()
        ens.set_precision("fp64")
        ens.set_solver(tol=1e-13, max_iter=3000, guess=L.GUESS_DIRECT)
        f_tight, _, _ = ens.compute_forces()
        for name, prec, g in (("plain", "fp64", L.GUESS_DIRECT), ("fast", "mixed", L.GUESS_LEARNED)):
            ens.set_precision(prec)
            ens.set_solver(tol=DIPOLE_TOL, max_iter=500, guess=g)
            ens.upload_positions(pos_now)
            f, _, _ = ens.compute_forces()
            force_err[name] = float(np.sqrt(((f - f_tight) ** 2).sum() / (f_tight ** 2).sum()))
        ens.set_solver(tol=DIPOLE_TOL, max_iter=500, guess=L.GUESS_LEARNED)
    else:
        ens.set_precision("fp64")
        f64, _, _ = ens.compute_forces()
        ens.set_precision("mixed")
        f32, _, _ = ens.compute_forces()
        force_err["fast"] = float(np.sqrt(((f32 - f64) ** 2).sum() / (f64 ** 2).sum()))
    ens.set_precision("mixed")

    # energy conservation: the same state advanced without thermostat (NVE)
    # by each arm; drift = slope of U + K over the run
    def drift(precision, guess, steps, st0):
        ens.set_precision(precision)
        if polar:
            ens.set_solver(tol=DIPOLE_TOL, max_iter=500, guess=guess)
        ens.upload_positions(st0["pos"])
        ens.upload_velocities(st0["vel"], st0["vtminus"])
        lf.run(steps)
        ser = lf.series()[-steps:]
        h = ser[:, 0] + ser[:, 1]
        tt = np.arange(steps) * dt * 1e-3   # ns
        slope = float(np.polyfit(tt, h, 1)[0])
        return {"kj_mol_per_ns": slope, "kj_mol_per_ns_per_molecule": slope / s.n_mols,
                "rms_fluctuation_kj_mol": float(np.std(h - np.polyval(np.polyfit(tt, h, 1), tt))),
                "steps": steps}
    drift_steps = min(args.drift_steps, SERIES_CAP)
    st0 = ens.state()
    nve = lf.params
    nve_thermo = nve.thermostat
    nve.thermostat = L.THERMO_NONE
    L.check(ens.ctx, ens.lib.smd_set_integrator(ens.ctx, ctypes.byref(nve)))
    energy_drift = {"plain": drift("fp64", L.GUESS_DIRECT, drift_steps, st0),
                    "fast": drift("mixed", L.GUESS_LEARNED if polar else L.GUESS_DIRECT, drift_steps, st0),
                    "how": "NVE from the same state (thermostat off), slope of U + K"}
    nve.thermostat = nve_thermo
    L.check(ens.ctx, ens.lib.smd_set_integrator(ens.ctx, ctypes.byref(nve)))
    ens.upload_positions(st0["pos"])
    ens.upload_velocities(st0["vel"], st0["vtminus"])
    ens.set_precision("mixed")
    if polar:
        ens.set_solver(tol=DIPOLE_TOL, max_iter=500, guess=L.GUESS_LEARNED)

    # energy drift of the rigid water of the SPC/E configuration (2160
    # molecules, LJ + Ewald |n| < 9, SHAKE): both precisions from the same
    # equilibrated state, NVE, and the mixed path's force error against FP64
    drift_c3 = spce_drift(args.drift_steps) if polar and world == 1 else None

    # --- end to end through the public API, host buffers ------------------
    pos = torch.empty(3 * n, dtype=torch.float64).pin_memory().numpy()
    vel = torch.empty(3 * n, dtype=torch.float64).pin_memory().numpy()
    st = ens.state()
    pos[:] = st["pos"].reshape(-1)
    vel[:] = st["vel"].reshape(-1)
    every = args.e2e_every
    e2e_steps = max(every, (min(args.steps, 200) // every) * every)
    lf.run(args.warmup)
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
        lf.observables()
    torch.cuda.synchronize()
    te = torch.tensor([(time.perf_counter() - t0) * 1e3], dtype=torch.float64)
    if dist:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = ns_per_day(float(te[0]) / e2e_steps * 1e-3, dt) * world

    # --- roofline of the reciprocal passes ---------------------------------
    kc = ctypes.c_int()
    L.check(ens.ctx, ens.lib.smd_step_kernel_count(ens.ctx, ctypes.byref(kc)))
    names = ["pair", "recip", "integrate", "list_rebuild", "frames", "mp_real", "mp_recip",
             "dipole_solve", "ind_real", "polar_recip", "field_rows", "pcg"]
    stage_ms = {k: float(v) for k, v in zip(names, prof)}
    stage_plain = {k: float(v) for k, v in zip(names, prof_plain)}
    peaks = dict(FALLBACK)
    peak_src = "fallback"
    if os.path.exists(PEAKS):
        peaks.update(json.load(open(PEAKS)))
        peak_src = "measured"
    # a forced rebuild is timed, but the list is rebuilt only when a site has
    # moved half the skin: weigh it by the rebuilds seen in the timed steps
    amortised = dict(stage_ms, list_rebuild=stage_ms["list_rebuild"] * fast["list_rebuilds_per_step"])
    amortised.pop("dipole_solve")   # field_rows + pcg
    dom = max(amortised, key=amortised.get)
    sm_mhz = peaks.get("sm_max_mhz", 1965.0)
    fp32_peak = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12
    hbm_peak = peaks["hbm_gbs"]
    rooflines = {}
    nk = ens.ewald_nk() if polar else 0
    if polar:
        # (1) reciprocal sums and forces of the permanent + induced multipoles:
        # FP32 operations of the column formulation (an FMA is 2): 33 per
        # (site, k) in the sums pass (27 per k plus the run's shared 22 over
        # 3.7 k) and 26 in the force pass (24 per k plus the column fold, 42
        # over 24 k); bound by the FP32 SIMT rate
        flops = float(nk) * n * (33 + 26)
        t = stage_ms["polar_recip"] * 1e-3
        rooflines["polar_recip"] = {
            "bound": "fp32", "kernel": "k_rsk_seg<float,2,4> + k_rforce_grp<float,1>",
            "achieved": flops / t / 1e12, "peak": fp32_peak, "unit": "TFLOP/s",
            "frac": flops / t / 1e12 / fp32_peak, "alg_flops_per_launch": flops, "k_vectors": nk,
            # DRAM bytes of one launch of each pass, from one ncu capture
            # (dram__bytes_read.sum + dram__bytes_write.sum: 6.45 + 0 MB and 3.17 + 0 MB)
            "traffic": 6.45e6 + 3.17e6, "ms": stage_ms["polar_recip"]}
        # (2) fused multipole + induced real space over the solve's tensor rows:
        # about 550 operations per directed pair (FP32 multipole algebra, FP64
        # radial factors and force assembly), rows = both directions of every
        # pair inside the cutoff plus the molecule's own sites
        entries = 2.0 * fast["pairs_in_cutoff"] + 2.0 * n
        flops = 550.0 * entries
        t = stage_ms["ind_real"] * 1e-3
        rooflines["fused_real"] = {
            "bound": "fp32+fp64 issue", "kernel": "k_polar_real_f<1> (+ k_polar_mol)",
            "achieved": flops / t / 1e12, "peak": fp32_peak, "unit": "TFLOP/s",
            "frac": flops / t / 1e12 / fp32_peak, "alg_flops_per_launch": flops, "row_entries": entries,
            "traffic": 17.7e6, "ms": stage_ms["ind_real"],
            "note": "half of the work is FP64 (nominal FP64 rate 37.2 TFLOP/s); ncu: FP64 pipe 33%, FMA 28%"}
        # (3) the PCG kernel: every product streams the FP32 tensor rows
        # (4 B partner + 16 B coefficients per entry) and gathers the packed
        # vector (16 B per entry); iterations + 1 products per solve
        products = fast["solver_iterations"] + 1
        nbytes = products * entries * (4 + 16 + 16)
        t = stage_ms["pcg"] * 1e-3
        rooflines["pcg"] = {
            "bound": "hbm", "kernel": "k_ind_pcg_pipe (pipelined PCG, molecule blocks)",
            "achieved": nbytes / t / 1e9, "peak": hbm_peak,
            "unit": "GB/s", "frac": nbytes / t / 1e9 / hbm_peak, "alg_bytes_per_launch": nbytes,
            "products": products, "traffic": 154e6, "ms": stage_ms["pcg"],
            "note": "rows and gathers are served mostly from L2 (126 MB); DRAM bytes from the ncu capture"}
        # the dominant kernel: the largest device time of one kernel (the
        # reciprocal figure covers two kernels)
        rooflines["polar_recip"]["kernels"] = 2
        main_kernel = max(rooflines, key=lambda k: rooflines[k]["ms"] / rooflines[k].get("kernels", 1))
        roofline = dict(rooflines[main_kernel], which=main_kernel)
    else:
        pairs = fast["pairs_in_cutoff"]
        flops = pairs * 2 * 23
        t = stage_ms["pair"] * 1e-3
        roofline = {"bound": "fp32", "kernel": "k_pair (LJ)", "achieved": flops / t / 1e12, "peak": fp32_peak,
                    "unit": "TFLOP/s", "frac": flops / t / 1e12 / fp32_peak, "traffic": None, "which": "pair"}
    roofline.update(peak_source=f"HBM: hbm_gbs of MEASURED_PEAKS.json ({peak_src}); FP32: nominal SIMT rate "
                                "148 SMs x 128 lanes x 2 at sm_max_mhz (the file has no FP32 figure)",
                    dominant_stage=dom,
                    traffic_source="ncu --set full captures of the polwater4096 step (profiles/)")

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and polar:
        sample, _ = workload("polwater4096", nmol=args.cpu_sample_mols)
        sps = cpu_reference(sample, 1)
        if sps:
            cpu = {"value": ns_per_day(sps, dt), "unit": "ns/day", "cores": 1, "kind": "reference",
                   "sample": f"1 MD step of polwater{args.cpu_sample_mols} (the same model at "
                             f"{args.cpu_sample_mols} molecules; the reference's dense dipole "
                             "matrix makes its step cost grow as N^2) with SwinMD's own "
                             "LFIntegrator::run, one process, one core"}

    if rank == 0:
        pairs = fast["pairs_in_cutoff"]
        out = {"metric": METRIC, "value": value, "unit": "ns/day", "n_gpus": world,
               "steps": args.steps, "warmup": args.warmup, "ms_per_step": fast["ms_per_step"],
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
               "dtype": "f32 pair/reciprocal/field math, f64 solver and integrator",
               "data": "synthetic (seeded lattice, random orientations, equilibrated on the GPU)",
               "config": dict(desc, l2="256 MB buffer written before every chunk of "
                              f"{args.chunk} steps", replicas=world, parallelism="replicas only",
                              equilibration_steps=args.equilibrate),
               "plain": dict(plain, dtype="f64", guess="M^-1 E0 (molecule blocks)",
                             algorithms="the fast arm's: column reciprocal passes, product-form 14-7"),
               "plain_reference_forms": dict(plain_ref, dtype="f64", guess="M^-1 E0 (molecule blocks)",
                                             algorithms="the reference's: one FP64 sine/cosine per (site, k), "
                                                        "pow() 14-7"),
               "fast_network_off": network_off and dict(
                   network_off, guess="2 p(t-1) - p(t-2) + M^-1 (E0 - 2 E0(t-1) + E0(t-2)) (network off)"),
               "fast": dict(fast, guess="learned" if polar else "n/a",
                            force_rms_rel_err_vs_fp64_tight=force_err.get("fast")),
               "plain_force_rms_rel_err_vs_fp64_tight": force_err.get("plain"),
               "speedup_fast_vs_plain": plain["ms_per_step"] / fast["ms_per_step"],
               "speedup_fast_vs_plain_reference_forms": plain_ref["ms_per_step"] / fast["ms_per_step"],
               "speedup_learned_vs_network_off": (network_off["ms_per_step"] / fast["ms_per_step"]
                                                  if network_off else None),
               "solver_iterations_by_guess": iters,
               "pair_interactions_per_s": pairs / (fast["ms_per_step"] * 1e-3),
               "pair_interactions_note": "unordered site pairs inside the short-range cutoff per step "
                                         "(the fast arm's) / s per step",
               "energy_drift": energy_drift,
               "energy_drift_spce2160": drift_c3,
               "training": train,
               "e2e": {"value": e2e_value, "unit": "ns/day", "h2d_bytes_per_step": 2 * 3 * n * 8 / every,
                       "d2h_bytes_per_step": (2 * 3 * n * 8 + 512) / every,
                       "how": f"upload positions+velocities from pinned host, smd_run({every}), "
                              "download positions+velocities+observables"},
               "gpu_launches": kc.value * args.steps,
               "kernels_per_step": kc.value,
               "stage_ms_fast": stage_ms, "stage_ms_plain": stage_plain,
               "stage_notes": "stage_ms_* time each stage alone (list_rebuild: one forced rebuild); in the fast "
                              "arm the multipole and induced real space are one fused pass, reported under "
                              "ind_real (mp_real 0)",
               "roofline": roofline,
               "rooflines": rooflines,
               "clocks": clocks_all, "cpu_baseline": cpu,
               "setup_s": time.perf_counter() - t_setup}
        print(json.dumps(out))
    ens.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
