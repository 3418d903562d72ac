"""Runs a fixed number of evaluations of one workload, for profilers.

    python -m agbnp3_b200.profile_run --natoms 25000 --evals 3 --mode mixed [--autotune]
    python -m agbnp3_b200.profile_run --batch 64 --evals 2

The first evaluation sizes the buffers and captures the CUDA graph; the
rest replay it with the coordinates resident on the device.
"""
import argparse
import time

import numpy as np

import agbnp3_b200 as A


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--natoms", type=int, default=25000)
    p.add_argument("--seed", type=int, default=1)
    p.add_argument("--evals", type=int, default=3)
    p.add_argument("--mode", default="mixed", choices=["mixed", "fp64"])
    p.add_argument("--batch", type=int, default=0, help="instances of log-uniform size in [300, 5000]")
    p.add_argument("--timing", action="store_true", help="print per-stage device times")
    p.add_argument("--autotune", action="store_true", help="tune the pair-stage decomposition first")
    a = p.parse_args()
    prec = A.PREC_MIXED if a.mode == "mixed" else A.PREC_FP64
    A.initialize()
    if a.batch:
        rng = np.random.default_rng(a.seed)
        sizes = np.exp(rng.uniform(np.log(300), np.log(5000), a.batch)).astype(int)
        systems = [A.make_globule(int(n), a.seed * 100003 + k, noise=0.2) for k, n in enumerate(sizes)]
        obj = A.Batch([A.Instance(s, precision=prec) for s in systems])
        obj.set_mode(prec, True)
        obj.set_coords(np.concatenate([s.coords() for s in systems]))
        natoms = obj.natoms
    else:
        s = A.make_globule(a.natoms, a.seed)
        obj = A.Instance(s, precision=prec)
        obj.set_coords(s.coords())
        natoms = s.natoms
    if a.autotune:
        print("autotune:", obj.autotune())
    obj.stage_timing(a.timing)
    t = time.perf_counter()
    for _ in range(a.evals):
        obj.ener_resident()
    dt = time.perf_counter() - t
    print(f"{a.evals} evaluations of {natoms} atoms ({a.mode}): {1e3 * dt / a.evals:.3f} ms/eval wall")
    if a.timing:
        print(obj.stage_times())
    A.terminate()


if __name__ == "__main__":
    main()
