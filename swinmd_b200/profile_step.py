"""Runs a few MD steps of a workload between cudaProfilerStart/Stop, for a
profiler started with `--profile-from-start off` (ncu) to see exactly those
steps and nothing of the set-up or training.

    python -m swinmd_b200.profile_step --workload polwater4096 --precision mixed --guess learned --steps 3
"""
import argparse

import torch

from . import engine, systems
from . import _lib as L


def build(workload: str):
    if workload == "polwater4096":
        return systems.polarizable_water(nmol=4096, kmax=18, seed=1)
    if workload == "lj4000":
        s = systems.lj_fluid(ncell=10, seed=1)
        s.config.long_correct = True
        return s
    raise SystemExit(f"unknown workload {workload}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="polwater4096")
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--guess", default="learned", choices=["direct", "learned"])
    ap.add_argument("--train-frames", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--steps", type=int, default=3)
    args = ap.parse_args()
    s = build(args.workload)
    ens = engine.GpuEnsemble(s, precision="fp64")
    polar = args.workload == "polwater4096"
    if polar:
        ens.set_solver(tol=2.0819e-8, guess=L.GUESS_DIRECT)
    lf = engine.LFIntegrator(ens)
    lf.start()
    lf.run(args.warmup)
    if polar and args.guess == "learned":
        ens.mlp_init(capacity_frames=args.train_frames, seed=1)
        for _ in range(args.train_frames):
            lf.run(1)
            ens.compute_forces(L.TERM_IND_SHORT)
            ens.mlp_collect()
        ens.mlp_train(epochs=8, batch=16384, lr=2e-3)
    ens.set_precision(args.precision)
    if polar:
        ens.set_solver(tol=2.0819e-8, guess=L.GUESS_LEARNED if args.guess == "learned" else L.GUESS_DIRECT)
    lf.run(args.warmup)
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    lf.run(args.steps)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    it = ens.solver_stats()[0] if polar else 0
    print(f"profiled {args.steps} steps of {args.workload} ({args.precision}, guess {args.guess}); "
          f"solver iterations {it}")
    ens.close()


if __name__ == "__main__":
    main()
