#!/usr/bin/env python
"""AGBNP3 energy+gradient throughput on B200.

Default workload: one 25,000-atom synthetic globule (seeded generator,
0.05 heavy atoms/A^3), evaluated in the engine's chosen mode (FP32 pair,
overlap and descreening math with FP64 accumulation).  A step is one full
energy+gradient evaluation (agbnp3_ener).  The plain FP64 path is timed in
the same run for the speed-up and accuracy columns.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

With N > 1 (torchrun, one process per GPU) every rank evaluates its own
conformation (a different seed); no collective touches the data path
(weak scaling).  --impl reference times the reference's own CPU library
(oracle/_ref, built from the reference sources) through its public API on
the same workload with all host cores.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
def metric_name(natoms):
    k = f"{natoms // 1000}k" if natoms % 1000 == 0 else str(natoms)
    return f"energy+grad evals/s @{k} atoms (chosen mode: FP32 math + FP64 accumulation)"

UNIT = "evals/s"


def workload_name(natoms, nheavy, seed):
    """config.workload of both arms for the single-globule workloads"""
    return f"globule {natoms} atoms ({nheavy} heavy), 0.05 heavy/A^3, seed {seed}"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="engine", choices=["engine", "reference"])
    p.add_argument("--natoms", type=int, default=25000)
    p.add_argument("--seed", type=int, default=1)
    p.add_argument("--fp64-steps", type=int, default=20)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-single-core", action="store_true", help="skip the 1-thread reference timing")
    p.add_argument("--cpu-best-of", type=int, default=3, help="reference evaluations per CPU baseline timing")
    p.add_argument("--no-batch", action="store_true", help="skip the 512-instance batch sub-measurement")
    p.add_argument("--no-large", action="store_true",
                   help="skip the 100,000-atom sub-measurement (chosen mode, plain FP64, per-term error)")
    p.add_argument("--no-surrogate", action="store_true",
                   help="skip the learned surrogate's sub-measurement (training on a reduced set, then its "
                        "inference time, fallback and errors at 25,000 and 50,000 atoms)")
    p.add_argument("--batch-steps", type=int, default=20, help="timed steps of the batch sub-measurement")
    p.add_argument("--chosen-batch", type=int, default=4,
                   help="conformations of the globule evaluated together for the batched chosen-mode figure (<2: off)")
    p.add_argument("--config", default="globule25k", choices=["globule25k", "globule100k", "batch512"],
                   help="globule25k: one 25,000-atom globule (headline); globule100k: one 100,000-atom globule "
                        "(per-term error of the chosen mode against the FP64 path); batch512: 512 instances of "
                        "300-5,000 atoms (log-uniform) with 0.2 A coordinate noise, one batched evaluation per step")
    p.add_argument("--ninst", type=int, default=512)
    p.add_argument("--shard", action="store_true",
                   help="strong scaling: ONE globule of --natoms atoms row-sharded over all ranks (NCCL all-reduce "
                        "of the pair passes' partial sums inside each evaluation) instead of one conformation per rank")
    a = p.parse_args()
    if a.config == "globule100k":
        a.natoms = 100000
        a.no_single_core = True
    return a


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during the timed
    region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu, self.rows, self.proc = gpu, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if len(r) > 5 + k and r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ----------------------------------------------------------------------------
# reference arm and CPU baseline: the reference library built from its sources
# ----------------------------------------------------------------------------
def _ref_child(natoms, seed, steps, warmup, threads, out_path):
    os.environ["OMP_NUM_THREADS"] = str(threads)
    # the reference library prints its own notices on stdout, which carries
    # only the bench's JSON line
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from agbnp3_b200.system import make_globule
    s = make_globule(natoms, seed)
    ref = O.RefLib(harness=False)
    tag = ref.new(s)
    times = []
    for k in range(warmup + steps):
        t0 = time.perf_counter()
        r = ref.ener(tag, s)
        dt = time.perf_counter() - t0
        if k >= warmup:
            times.append(dt)
    json.dump({"times": times, "egb": r["egb"], "rc": r["rc"]}, open(out_path, "w"))


def run_reference(natoms, seed, steps, warmup, threads):
    """Times agbnp3_ener of the reference library in a fresh process (the
    reference supports one instance per process)."""
    import multiprocessing as mp
    import tempfile
    out = tempfile.NamedTemporaryFile(suffix=".json", delete=False).name
    ctx = mp.get_context("spawn")
    p = ctx.Process(target=_ref_child, args=(natoms, seed, steps, warmup, threads, out))
    p.start()
    p.join(timeout=3600)
    if p.exitcode != 0:
        raise RuntimeError(f"reference run failed (exit {p.exitcode})")
    d = json.load(open(out))
    os.unlink(out)
    return d


def reference_arm(args):
    rank, world, local = dist_env()
    if rank != 0:
        return
    ref_lib = os.path.join(ROOT, "oracle", "_ref", "libagbnp3_ref.so")
    from agbnp3_b200.system import make_globule
    nheavy = make_globule(args.natoms, args.seed).nheavy
    cfg = {"workload": workload_name(args.natoms, nheavy, args.seed), "natoms": args.natoms}
    if not os.path.exists(ref_lib):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libagbnp3_ref.so not built "
                          "(needs the reference sources at build time)"}))
        return
    threads = os.cpu_count() or 1
    d = run_reference(args.natoms, args.seed, args.steps, args.warmup, threads)
    tot = sum(d["times"])
    v = len(d["times"]) / tot
    print(json.dumps({
        "impl": "reference", "metric": metric_name(args.natoms), "value": v, "unit": UNIT, "n_gpus": world,
        "devices": f"host CPU ({threads} threads); the reference has no GPU path", "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(d["times"]), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": cfg,
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"{args.steps} full evaluations of the {args.natoms}-atom globule"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


# Operations per pair of each pair stage, counted from the stage's formulas
# (an FMA counts as two flops; add, multiply and compare-free selects one):
#   descreening (invb), atom i by heavy atom j: distance 8, sqrt (SFU),
#     a/h 1, interval offset 1, cubic 6, weighted sum 2            = 18 + 1 SFU
#   GB pair energy (agb), unordered pair: distance 8, BiBj 1, exponent 2,
#     exp2 (SFU), d^2 + BiBj e 2, rsqrt (SFU), qiqj 1, q f^3 3, energy 2,
#     force weight 3, force 3 + 6 sums, A_i term 4 + 2 sums       = 37 + 2 SFU
#   Born-radius chain rule (gbders), per direction with a heavy descreener:
#     a/h 1, offset 1, cubic 6, derivative 6, Q 1, dQ 3, U, V 4, force
#     weights 6 = 28; per pair: distance 8, rsqrt (SFU), d 1, scaling 2,
#     force components 6, 12 sums = 29 + 1 SFU; heavy-heavy pairs have two
#     directions, heavy-hydrogen pairs one
PAIR_OPS = {"invb": (18, 1), "agb": (37, 2), "gbders_hh": (29 + 2 * 28, 1), "gbders_hx": (29 + 28, 1)}


# DRAM traffic per launch of each kernel, read from an ncu capture of the
# 25,000-atom workload (`python -m agbnp3_b200.ncu_summary --traffic-json`);
# ncu counters cannot be read inside the timed run, so the traffic is
# reported for that workload only
TRAFFIC_JSON = os.path.join(ROOT, "profiles", "dram_traffic_globule25k_mixed.json")


def load_traffic(natoms):
    if natoms != 25000 or not os.path.exists(TRAFFIC_JSON):
        return None
    with open(TRAFFIC_JSON) as f:
        return json.load(f)


# kernels of each O(N) stage (name prefixes)
STAGE_KERNELS = {"nblist": ("k_cell_", "k_nl_", "k_skin_", "k_cand_"),
                 "volumes": ("k_l2_", "k_lm_", "agb_scan", "k_scan"),
                 "ws": ("k_ws_",), "treeders": ("k_tree_ders",)}


def tree_roofline(natoms, nheavy, counts, stage_ms, hbm_gbs, rbytes, traffic):
    """The O(N) stages against the HBM roofline.  Algorithmic bytes per
    evaluation = what the stage must read and write at least once:
      nblist:   heavy-atom positions and radii (16 B each) in; near-list
                entries (index + float d^2, 8 B) and per-atom count/offset
                (8 B) out;
      volumes:  near-list entries (4 B) and per-atom Gaussian operands
                (x, y, z, exponent, 1/R: 5 R) in; per kept overlap one
                8-slot record (8 R) and its parents (4 B each) out, plus
                the per-atom volume and area (16 B);
      ws:       positions of all atoms (3 R) and heavy-atom scaling
                factors (8 B) in; per water site its position (3 R), its
                3x3 Jacobians to up to four parents (36 R), its scaling
                factor and HB energy (16 B) out;
      treeders: every kept record and its parents in, per heavy atom the
                four chain-rule factors (32 B) in, per atom four gradient
                rows (96 B) out.
    R is the working precision's size (4 mixed, 8 FP64)."""
    R = rbytes
    P = counts["near_pairs"]
    K = counts["kept"]
    nws = counts["water_sites"]
    rec = sum(k * (8 * R + 4 * m) for m, k in zip(range(2, 6), K))
    alg = {"nblist": 16 * nheavy + 8 * P + 8 * nheavy,
           "volumes": 4 * P + 5 * R * natoms + rec + 16 * nheavy,
           "ws": 3 * R * natoms + 8 * nheavy + nws * (39 * R + 16),
           "treeders": rec + 32 * nheavy + 96 * natoms}
    out = {}
    for k, b in alg.items():
        t = stage_ms.get(k)
        if not t:
            continue
        gbs = b / (t * 1e-3) / 1e9
        e = {"alg_bytes": b, "ms": t, "achieved_gbs": gbs, "frac_of_hbm": gbs / hbm_gbs}
        if traffic:
            dram = sum(v["dram_bytes_per_eval"] for n, v in traffic["kernels"].items()
                       if n.startswith(STAGE_KERNELS[k]))
            e["dram_bytes_ncu"] = dram
            e["dram_over_alg"] = dram / b
        out[k] = e
    return out


def pair_roofline(natoms, nheavy, stage_ms, peaks):
    nx = natoms - nheavy
    work = {  # (flops, SFU ops) per launch
        "invb": [(natoms * nheavy - nheavy) * w for w in PAIR_OPS["invb"]],
        "agb": [natoms * (natoms - 1) // 2 * w for w in PAIR_OPS["agb"]],
        "gbders": [nheavy * (nheavy - 1) // 2 * a + nheavy * nx * b
                   for a, b in zip(PAIR_OPS["gbders_hh"], PAIR_OPS["gbders_hx"])],
    }
    stages = {}
    for k, (fl, sf) in work.items():
        t = stage_ms[k] * 1e-3
        stages[k] = {"gflop_per_launch": fl / 1e9, "ms": stage_ms[k], "tflops": fl / t / 1e12,
                     "fp32_frac": fl / t / 1e12 / peaks["fp32_tflops"],
                     "sfu_frac": sf / t / 1e12 / peaks["ex2_tops"]}
    tot_fl = sum(w[0] for w in work.values())
    tot_ms = sum(stage_ms[k] for k in work)
    stages["all_pair_stages"] = {"gflop_per_launch": tot_fl / 1e9, "ms": tot_ms,
                                 "tflops": tot_fl / (tot_ms * 1e-3) / 1e12,
                                 "fp32_frac": tot_fl / (tot_ms * 1e-3) / 1e12 / peaks["fp32_tflops"]}
    dom = max(work, key=lambda k: stages[k]["ms"])
    d = stages[dom]
    kern = {"gbders": "k_gbders_x2", "agb": "k_agb_x2", "invb": "k_descreen_s"}[dom]  # FP32 (chosen mode) kernels
    tr = load_traffic(natoms)
    hits = [v for n, v in tr["kernels"].items() if n == kern or n.startswith(kern + "<")] if tr else []
    traffic = hits[0]["dram_bytes_per_launch"] if len(hits) == 1 else None
    return {"kernel": kern,
            "stage": dom, "bound": "fp32", "achieved": d["tflops"], "peak": peaks["fp32_tflops"],
            "unit": "TFLOP/s", "frac": d["fp32_frac"], "traffic": traffic,
            "traffic_note": f"DRAM bytes per launch, ncu capture of this workload ({tr['command']})" if traffic else None,
            "peak_source": "measured in this run: FP32 FMA chains on every SM (agbnp3_measure_peaks)",
            "sfu_frac": d["sfu_frac"], "peaks": peaks, "stages": stages}


def measured_hbm_gbs():
    """HBM copy bandwidth of this pool's B200s (MEASURED_PEAKS.json, written
    by the pool's own measurement), else the pool's earlier fallback figure"""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return {"gbs": float(json.load(f)["hbm_gbs"]), "source": "measured (MEASURED_PEAKS.json hbm_gbs)"}
    except (OSError, KeyError, ValueError):
        return {"gbs": 6650.0, "source": "fallback 6.65 TB/s"}


def batch_systems(A, ninst, seed, rank=0):
    from agbnp3_b200.shard import rank_seed
    rs = rank_seed(seed, 1000 * rank)
    rng = np.random.default_rng(rs)
    sizes = np.exp(rng.uniform(np.log(300), np.log(5000), ninst)).astype(int)
    return [A.make_globule(int(n), rs * 100003 + k, noise=0.2) for k, n in enumerate(sizes)]


def time_batches(A, torch, subs, steps, warmup, local, flush):
    """Device time (ms) of `steps` evaluations of the batches `subs` issued
    together (agbnp3_batches_ener_resident): the L2 flush and the start
    event on the first batch's stream, which every other batch's stream
    waits for; the end event after all batches are done."""
    dev = torch.device("cuda", local)
    streams = [torch.cuda.ExternalStream(b.stream, device=dev) for b in subs]
    for _ in range(warmup):
        A.ener_resident_many(subs)
    times = []
    for _ in range(steps):
        with torch.cuda.stream(streams[0]):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(streams[0])
        for st in streams[1:]:
            st.wait_event(e0)
        A.ener_resident_many(subs)
        with torch.cuda.stream(streams[0]):
            e1.record(streams[0])
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    return times


def split_batches(A, insts, systems, nsplit):
    """nsplit batches over the instances, member k in batch k % nsplit (the
    members' sizes are random, so the batches are of similar size), each
    set up, evaluated once and tuned on its own"""
    subs, tunes = [], []
    for q in range(nsplit):
        B = A.Batch(insts[q::nsplit])
        B.set_mode(A.PREC_MIXED, True)
        B.set_coords(np.concatenate([x.coords() for x in systems[q::nsplit]]))
        B.ener_resident()
        tunes.append(B.autotune())
        subs.append(B)
    return subs, tunes


def measure_batch(A, torch, ninst, steps, warmup, seed, rank, world, local, clocks=True, splits=(1, 2, 4)):
    """Builds the batched configuration (ninst instances, log-uniform
    300-5,000 atoms, 0.2 A noise) and times `steps` evaluations of all of
    them (L2 flushed between steps) for each way of splitting them into
    batches that run side by side on their own streams (`splits`); the
    fastest split is the reported value.  Returns the measurements."""
    from agbnp3_b200.shard import max_over_ranks, throughput
    systems = batch_systems(A, ninst, seed, rank)
    insts = [A.Instance(x, precision=A.PREC_MIXED) for x in systems]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    per_split = {}
    best = None
    clk = Clocks(local) if clocks else None
    if clk:
        clk.__enter__()
    for nsplit in splits:
        subs, tunes = split_batches(A, insts, systems, nsplit)
        times = time_batches(A, torch, subs, steps, warmup, local, flush)
        tot = max_over_ranks(sum(times), world, f"cuda:{local}")
        per_split[nsplit] = {"value": throughput(ninst * steps, tot / 1e3, world), "ms_per_step": tot / steps,
                             "autotune": tunes,
                             "launches_per_step": int(sum(b.stats()["launches"] for b in subs))}
        if best is None or per_split[nsplit]["value"] > per_split[best[0]]["value"]:
            if best:
                for b in best[1]:
                    b.close()
            best = (nsplit, subs)
        else:
            for b in subs:
                b.close()
    if clk:
        clk.__exit__()
    nsplit, subs = best
    # per-stage device times of the unsplit batch
    B = A.Batch(insts)
    B.set_mode(A.PREC_MIXED, True)
    xyz = np.concatenate([x.coords() for x in systems])
    B.set_coords(xyz)
    B.ener_resident()
    B.stage_timing(True)
    B.ener_resident()
    stage_ms = B.stage_times()
    B.stage_timing(False)
    # e2e with the fastest split: host coordinates in, all outputs out, every step
    xyzs = [np.concatenate([x.coords() for x in systems[q::nsplit]]) for q in range(nsplit)]
    e2e = []
    for _ in range(steps):
        t0 = time.perf_counter()
        for b, c in zip(subs, xyzs):
            b.set_coords(c)
        A.ener_resident_many(subs)
        for b in subs:
            b.results()
        e2e.append(time.perf_counter() - t0)
    # the split batches give the unsplit batch's energies
    R = B.results()
    split_dev = 0.0
    for q, b in enumerate(subs):
        Rq = b.results()
        for key in ("egb", "evdw", "ecav", "ehb"):
            ref = R[key][q::nsplit]
            split_dev = max(split_dev, float(np.max(np.abs(Rq[key] - ref) / np.maximum(np.abs(ref), 1e-12))))
    # accuracy of the batched mixed path against the FP64 path on 8 members
    acc = []
    for k in range(0, ninst, max(1, ninst // 8)):
        a = A.Instance(systems[k], precision=A.PREC_FP64)
        F = a.ener()
        e_m = sum(R[q][k] for q in ("egb", "evdw", "ecav", "ehb"))
        e_f = sum(F[q] for q in ("egb", "evdw", "ecav", "ehb"))
        acc.append(abs(e_m - e_f) / abs(e_f))
        a.close()
    natoms = int(sum(x.natoms for x in systems))
    B.close()
    for b in subs:
        b.close()
    for i in insts:
        i.close()
    m = per_split[nsplit]
    return {"value": m["value"], "unit": "evals/s", "ms_per_step": m["ms_per_step"], "steps": steps, "warmup": warmup,
            "workload": f"batch of {ninst} globules, {natoms} atoms total, 0.2 A noise", "natoms": natoms,
            "streams": nsplit, "autotune": m["autotune"], "stage_ms": stage_ms,
            "by_streams": {str(k): {"value": v["value"], "ms_per_step": v["ms_per_step"]} for k, v in per_split.items()},
            "split_vs_unsplit_max_rel_diff": split_dev,
            "e2e": {"value": world * ninst * steps / sum(e2e), "unit": "evals/s",
                    "h2d_bytes_per_step": 3 * 8 * natoms, "d2h_bytes_per_step": 15 * 8 * natoms + 56 * ninst},
            "accuracy_vs_fp64": {"max_energy_rel_err": max(acc)}, "launches_per_step": m["launches_per_step"],
            "clocks": clk.summary() if clk else None}


def measure_conformations(A, torch, s, k, steps, warmup, local, world, full, tot, frc, splits=(1, 2, 4)):
    """The chosen mode on k conformations of system s (the first s itself,
    the others with N(0, 0.1 A) coordinate noise), evaluated together: as
    one batch, or split into batches that run side by side on their own
    streams (`splits`, the fastest reported); one step = one evaluation of
    all k; value = conformation evaluations per second; accuracy of the
    first against the FP64 results `full` of s."""
    from agbnp3_b200.shard import max_over_ranks, throughput
    rng = np.random.default_rng(12345)
    confs = [s] + [s.with_coords(s.coords() + rng.normal(0.0, 0.1, (s.natoms, 3))) for _ in range(k - 1)]
    insts = [A.Instance(c, precision=A.PREC_MIXED, compat=True) for c in confs]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    per_split, best = {}, None
    for nsplit in [q for q in splits if k % q == 0]:
        subs, tunes = split_batches(A, insts, confs, nsplit)
        times = time_batches(A, torch, subs, steps, warmup, local, flush)
        t = max_over_ranks(sum(times), world, f"cuda:{local}")
        per_split[nsplit] = {"value": throughput(k * steps, t / 1e3, world), "ms_per_step": t / steps,
                             "autotune": tunes, "launches_per_step": int(sum(b.stats()["launches"] for b in subs))}
        if best is None or per_split[nsplit]["value"] > per_split[best[0]]["value"]:
            if best:
                for b in best[1]:
                    b.close()
            best = (nsplit, subs)
        else:
            for b in subs:
                b.close()
    nsplit, subs = best
    R = subs[0].results()  # the first conformation is member 0 of batch 0
    n = s.natoms
    first = {q: R[q][0] for q in ("egb", "evdw", "ecav", "ehb")}
    g = sum(R[q][:n] for q in ("dgbdr", "dvwdr", "decav", "dehb"))
    m = per_split[nsplit]
    out = {"value": m["value"], "unit": UNIT, "conformations": k, "streams": nsplit,
           "ms_per_batched_step": m["ms_per_step"], "steps": steps, "autotune": m["autotune"],
           "launches_per_step": m["launches_per_step"],
           "by_streams": {str(q): {"value": v["value"], "ms_per_step": v["ms_per_step"]} for q, v in per_split.items()},
           "accuracy_vs_fp64": {"energy_rel_err": abs(sum(first.values()) - tot(full)) / abs(tot(full)),
                                "force_rms_rel_err": float(np.sqrt(((g - frc(full)) ** 2).sum() / (frc(full) ** 2).sum()))},
           "workload": f"{k} conformations of the globule (N(0, 0.1 A) noise on all but the first), "
                       f"as {nsplit} batch(es) on their own streams"}
    for b in subs:
        b.close()
    for i in insts:
        i.close()
    return out


def measure_large(A, torch, natoms, seed, steps, steps64, local, world):
    """One large globule (configs' mixed-precision case): the chosen mode and
    the plain FP64 path, each autotuned, device-timed over `steps` / `steps64`
    evaluations (L2 flushed between them), and the chosen mode's per-term
    error against the FP64 path."""
    from agbnp3_b200.shard import max_over_ranks, throughput
    s = A.make_globule(natoms, seed)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    res = {}
    for prec, k, n in ((A.PREC_MIXED, "mixed", steps), (A.PREC_FP64, "fp64", steps64)):
        inst = A.Instance(s, precision=prec, compat=True)
        inst.ener()
        inst.set_coords(s.coords())
        tune = inst.autotune()
        stream = torch.cuda.ExternalStream(inst.stream, device=torch.device("cuda", local))
        inst.ener_resident()
        times = []
        for _ in range(n):
            with torch.cuda.stream(stream):
                flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            inst.ener_resident()
            with torch.cuda.stream(stream):
                e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        t = max_over_ranks(sum(times), world, f"cuda:{local}")
        res[k] = {"value": throughput(n, t / 1e3, world), "ms_per_step": t / n, "steps": n, "autotune": tune,
                  "out": inst.results()}
        inst.close()
    M, F = res["mixed"].pop("out"), res["fp64"].pop("out")
    tot = lambda R: sum(R[q] for q in ("egb", "evdw", "ecav", "ehb"))  # noqa: E731
    frc = lambda R: R["dgbdr"] + R["dvwdr"] + R["decav"] + R["dehb"]  # noqa: E731
    return {"workload": workload_name(natoms, s.nheavy, seed), "unit": UNIT, "mixed": res["mixed"],
            "fp64_plain": res["fp64"], "speedup_of_chosen": res["mixed"]["value"] / res["fp64"]["value"],
            "accuracy_vs_fp64": {"energy_rel_err": abs(tot(M) - tot(F)) / abs(tot(F)),
                                 "force_rms_rel_err": float(np.sqrt(((frc(M) - frc(F)) ** 2).sum() / (frc(F) ** 2).sum())),
                                 "per_term_rel_err": {q: abs(M[q] - F[q]) / max(abs(F[q]), 1e-12)
                                                      for q in ("egb", "evdw", "ecav", "ehb", "mol_volume")}}}


def batch_main(args, A, torch, rank, world, local):
    """512 independent instances (log-uniform 300-5,000 atoms, 0.2 A noise)
    evaluated together: one step = one batched evaluation of all instances;
    the metric is instance evaluations per second."""
    m = measure_batch(A, torch, args.ninst, args.steps, args.warmup, args.seed, rank, world, local)
    if rank == 0:
        print(json.dumps({
            "metric": "instance energy+grad evals/s, 512-instance batch (300-5,000 atoms)", "value": m["value"],
            "unit": "evals/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": m["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 math / f64 accumulation", "data": "synthetic",
            "config": {"workload": m["workload"], "l2": "256 MB flush between timed steps", "autotune": m["autotune"],
                       "streams": m["streams"]},
            "by_streams": m["by_streams"],
            "stage_ms": m["stage_ms"], "e2e": m["e2e"], "accuracy_vs_fp64": m["accuracy_vs_fp64"],
            "gpu_launches": m["launches_per_step"] * args.steps, "clocks": m["clocks"]}))


def shard_main(args, A, torch, rank, world, local):
    """One instance row-sharded over all ranks (strong scaling): every rank
    holds the same globule and evaluates its share of the pair passes; one
    step = one whole evaluation, timed on every rank, max over ranks."""
    from agbnp3_b200.shard import max_over_ranks, shard_instance
    s = A.make_globule(args.natoms, args.seed)
    inst = A.Instance(s, precision=A.PREC_MIXED, compat=True)
    inst.ener()  # sizes the buffers and orders the pair slots
    if world > 1:
        shard_instance(inst)
    else:
        inst.shard(0, 1, A.shard_unique_id())
    stream = torch.cuda.ExternalStream(inst.stream, device=torch.device("cuda", local))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    inst.set_coords(s.coords())
    for _ in range(args.warmup):
        inst.ener_resident()
    times = []
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            inst.ener_resident()
            with torch.cuda.stream(stream):
                e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
    tot = max_over_ranks(sum(times), world, f"cuda:{local}")
    R = inst.results()
    # e2e: host coordinates in, all outputs out, every step, on every rank
    e2e = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        inst.ener()
        e2e.append(time.perf_counter() - t0)
    e2e_tot = max_over_ranks(sum(e2e), world, f"cuda:{local}")
    st = inst.stats()
    if rank == 0:
        print(json.dumps({
            "metric": metric_name(args.natoms) + ", one instance row-sharded", "value": args.steps / (tot / 1e3),
            "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": tot / args.steps, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f32 math / f64 accumulation", "data": "synthetic",
            "config": {"workload": f"globule {args.natoms} atoms, seed {args.seed}, row-sharded over {world} ranks",
                       "l2": "256 MB flush between timed steps"},
            "e2e": {"value": args.steps / e2e_tot, "unit": UNIT, "h2d_bytes_per_step": 3 * 8 * args.natoms,
                    "d2h_bytes_per_step": 15 * 8 * args.natoms + 56},
            "gpu_launches": int(st["launches"]) * args.steps,
            "energies": {k: R[k] for k in ("egb", "evdw", "ecav", "ehb")},
            "clocks": clk.summary()}))
    inst.close()


# ----------------------------------------------------------------------------
# engine arm
# ----------------------------------------------------------------------------
def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    rank, world, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    import agbnp3_b200 as A
    A.lib().agbnp3_set_device(local)
    A.initialize()
    if args.config == "batch512" or args.shard:
        (shard_main if args.shard else batch_main)(args, A, torch, rank, world, local)
        A.terminate()
        if world > 1:
            torch.distributed.destroy_process_group()
        return

    from agbnp3_b200.shard import max_over_ranks, rank_seed, throughput
    natoms = args.natoms
    s = A.make_globule(natoms, rank_seed(args.seed, rank))
    inst = A.Instance(s, precision=A.PREC_MIXED, compat=True)
    ref_out = inst.ener()  # sizes the buffers
    inst.set_coords(s.coords())
    tune = inst.autotune()  # pair-stage decomposition for this system
    stream = torch.cuda.ExternalStream(inst.stream, device=torch.device("cuda", local))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")

    def timed_resident(obj, steps, warmup):
        obj.set_coords(s.coords())
        for _ in range(warmup):
            obj.ener_resident()
        times = []
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.zero_()  # evicts the 126 MB L2 between steps
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            obj.ener_resident()
            with torch.cuda.stream(stream):
                e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        return times

    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        times = timed_resident(inst, args.steps, args.warmup)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    tot_ms = max_over_ranks(sum(times), world, f"cuda:{local}")
    value = throughput(args.steps, tot_ms / 1e3, world)
    mixed = inst.results()
    st = inst.stats()

    # per-stage device times (CUDA events between stages, direct launches)
    inst.stage_timing(True)
    stage = {}
    for _ in range(3):
        inst.ener_resident()
        for k, v in inst.stage_times().items():
            stage.setdefault(k, []).append(v)
    inst.stage_timing(False)
    stage_ms = {k: statistics.median(v) for k, v in stage.items()}

    # plain FP64 path: speed and the accuracy of the chosen mode against it
    inst64 = A.Instance(s, precision=A.PREC_FP64, compat=True)
    inst64.ener()
    inst64.set_coords(s.coords())
    tune64 = inst64.autotune()  # the plain path at its own best decomposition
    t64 = timed_resident(inst64, args.fp64_steps, 1)
    fp64_value = throughput(len(t64), max_over_ranks(sum(t64), world, f"cuda:{local}") / 1e3, world)
    full = inst64.results()
    inst64.close()
    tot = lambda R: sum(R[k] for k in ("egb", "evdw", "ecav", "ehb"))  # noqa: E731
    frc = lambda R: R["dgbdr"] + R["dvwdr"] + R["decav"] + R["dehb"]  # noqa: E731
    acc = {"energy_rel_err": abs(tot(mixed) - tot(full)) / abs(tot(full)),
           "force_rms_rel_err": float(np.sqrt(((frc(mixed) - frc(full)) ** 2).sum() / (frc(full) ** 2).sum())),
           "per_term_rel_err": {k: abs(mixed[k] - full[k]) / max(abs(full[k]), 1e-12)
                                for k in ("egb", "evdw", "ecav", "ehb", "mol_volume")}}

    # e2e: through agbnp3_ener with host buffers (pinned), copies included
    L = A.lib()
    pin = lambda n: torch.empty(n, dtype=torch.float64, pin_memory=True)  # noqa: E731
    hx, hy, hz = pin(natoms), pin(natoms), pin(natoms)
    hx.numpy()[:], hy.numpy()[:], hz.numpy()[:] = s.x, s.y, s.z
    outs = [pin(natoms) for _ in range(3)] + [pin(3 * natoms) for _ in range(4)]
    import ctypes
    dptr = lambda t: ctypes.cast(t.data_ptr(), ctypes.POINTER(ctypes.c_double))  # noqa: E731
    es = [ctypes.c_double() for _ in range(7)]

    def call():
        rc = L.agbnp3_ener(inst.tag, 0, dptr(hx), dptr(hy), dptr(hz), dptr(outs[0]), dptr(outs[1]),
                           ctypes.byref(es[6]), dptr(outs[2]), ctypes.byref(es[0]), dptr(outs[3]),
                           ctypes.byref(es[1]), ctypes.byref(es[2]), dptr(outs[4]), ctypes.byref(es[3]),
                           ctypes.byref(es[4]), dptr(outs[5]), ctypes.byref(es[5]), dptr(outs[6]))
        if rc != A.AGBNP_OK:
            raise RuntimeError(A.last_error())

    for _ in range(args.warmup):
        call()
    e2e_t = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        call()
        e2e_t.append(time.perf_counter() - t0)
    e2e_tot = max_over_ranks(sum(e2e_t), world, f"cuda:{local}")
    e2e_value = throughput(args.steps, e2e_tot, world)

    # the same call with pageable host arrays (plain numpy), as a C caller
    # passing its own malloc'd arrays would
    pg = [np.ascontiguousarray(a, dtype=np.float64) for a in (s.x, s.y, s.z)]
    pouts = [np.zeros(natoms) for _ in range(3)] + [np.zeros((natoms, 3)) for _ in range(4)]
    pptr = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731

    def call_pageable():
        rc = L.agbnp3_ener(inst.tag, 0, pptr(pg[0]), pptr(pg[1]), pptr(pg[2]), pptr(pouts[0]), pptr(pouts[1]),
                           ctypes.byref(es[6]), pptr(pouts[2]), ctypes.byref(es[0]), pptr(pouts[3]),
                           ctypes.byref(es[1]), ctypes.byref(es[2]), pptr(pouts[4]), ctypes.byref(es[3]),
                           ctypes.byref(es[4]), pptr(pouts[5]), ctypes.byref(es[5]), pptr(pouts[6]))
        if rc != A.AGBNP_OK:
            raise RuntimeError(A.last_error())

    for _ in range(args.warmup):
        call_pageable()
    e2e_p = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        call_pageable()
        e2e_p.append(time.perf_counter() - t0)
    e2e_pageable = throughput(args.steps, max_over_ranks(sum(e2e_p), world, f"cuda:{local}"), world)

    # roofline of the pair stages: algorithmic FP32 work per launch (pair
    # counts x frozen per-pair operation counts) over the stage's device
    # time, against FP32 / special-function peaks measured in this run
    peaks = A.measure_peaks(local)
    roof = pair_roofline(natoms, s.nheavy, stage_ms, peaks)
    hbm = measured_hbm_gbs()
    roof["hbm_stages"] = tree_roofline(natoms, s.nheavy, st, stage_ms, hbm["gbs"], 4, load_traffic(natoms))
    roof["hbm_stages_peak"] = hbm

    # the chosen mode batched: K conformations of the same globule (0.1 A
    # coordinate noise each, the first unperturbed) in one batched evaluation
    chosen_batch = None
    if args.chosen_batch > 1:
        chosen_batch = measure_conformations(A, torch, s, args.chosen_batch, max(4, args.steps // args.chosen_batch), 3,
                                             local, world, full, tot, frc)
        chosen_batch["speedup_over_fp64_plain"] = chosen_batch["value"] / fp64_value

    # the batched configuration (512 instances), measured in the same run
    batch = None
    if not args.no_batch:
        batch = measure_batch(A, torch, args.ninst, args.batch_steps, 3, args.seed, rank, world, local,
                              clocks=False)

    # the 100,000-atom globule (mixed-precision configuration), same run
    large = None
    if not args.no_large and natoms != 100000:
        large = measure_large(A, torch, 100000, args.seed, 10, 3, local, world)

    # the learned surrogate, measured (not part of the chosen mode: the
    # figures show why)
    sur = None
    if rank == 0 and not args.no_surrogate:
        try:
            from agbnp3_b200 import surrogate as SG
            sur = SG.bench_report()
        except Exception as e:  # noqa: BLE001
            sur = {"failed": str(e)}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline and os.path.exists(os.path.join(ROOT, "oracle", "_ref",
                                                                             "libagbnp3_ref.so")):
        try:
            threads = os.cpu_count() or 1
            k = args.cpu_best_of
            d = run_reference(natoms, args.seed, k, 1, threads)
            cpu = {"value": 1.0 / min(d["times"]), "unit": UNIT, "cores": threads, "kind": "reference",
                   "sample": f"best of {k} evaluations (after 1 untimed) of the {natoms}-atom globule, reference "
                             f"library, {threads} OpenMP threads",
                   "times_s": d["times"]}
            if not args.no_single_core and threads > 1:
                d1 = run_reference(natoms, args.seed, k, 0, 1)
                cpu["single_core"] = {"value": 1.0 / min(d1["times"]), "unit": UNIT, "cores": 1,
                                      "sample": f"best of {k} evaluations of the {natoms}-atom globule, 1 thread",
                                      "times_s": d1["times"]}
        except Exception as e:  # noqa: BLE001
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"failed: {e}"}

    if rank == 0:
        line = {
            "metric": metric_name(natoms), "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tot_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 math / f64 accumulation", "data": "synthetic",
            "config": {"workload": workload_name(natoms, s.nheavy, args.seed),
                       "mode": "mixed", "compat": True, "l2": "256 MB flush between timed steps", "autotune": tune,
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "fp64_plain": {"value": fp64_value, "unit": UNIT, "ms_per_step": sum(t64) / len(t64), "autotune": tune64,
                           "speedup_of_chosen": value / fp64_value},
            "accuracy_vs_fp64": acc,
            "chosen_batched": chosen_batch,
            "stage_ms": stage_ms,
            "counts": st,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 3 * 8 * natoms,
                    "d2h_bytes_per_step": (3 + 12) * 8 * natoms + 7 * 8, "host_buffers": "pinned",
                    "pageable": {"value": e2e_pageable, "unit": UNIT,
                                 "host_buffers": "pageable (numpy arrays, as a C caller's malloc'd arrays)"}},
            "gpu_launches": int(st["launches"]) * args.steps,
            "roofline": roof,
            "batch512": batch,
            "globule100k": large,
            "surrogate": sur,
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
        }
        print(json.dumps(line))
    inst.close()
    A.terminate()
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
