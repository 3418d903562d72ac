"""Summarises an ncu launch list (``--metrics gpu__time_duration.sum --csv``)
per kernel: launches, total device time and share of the total.

    python -m agbnp3_b200.ncu_summary launches.csv [--evals N]
    python -m agbnp3_b200.ncu_summary capture.csv --evals N --traffic-json out.json \
        --command "<the ncu command>" --workload "<what it ran>"

With --traffic-json the capture must also hold dram__bytes_read.sum and
dram__bytes_write.sum; the file lists per kernel its launches and DRAM
bytes per launch and per evaluation (bench.py reads it for the roofline's
traffic figures).

Kernel names are grouped without their template arguments' values kept
apart (``k_tree_ders<float, 3>`` and ``<float, 5>`` stay separate, the
argument list is dropped).  ``--evals`` divides launches and time by the
number of evaluations the profiled command ran, giving per-evaluation
figures.  ncu serialises launches and runs them with cold caches, so the
shares are the figures to compare with in-process timings, not the
absolute times.
"""
import argparse
import collections
import csv
import json
import re


def kernel_key(name: str) -> str:
    name = re.sub(r"\(View.*$|\(const .*$|\(int.*$|\(double.*$|\(float.*$", "", name)
    name = re.sub(r"^void ", "", name)
    return name.strip()


TIME_SCALE = {"ns": 1.0, "nsecond": 1.0, "us": 1e3, "usecond": 1e3, "ms": 1e6, "msecond": 1e6}
BYTE_SCALE = {"byte": 1.0, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9, "KB": 1e3, "MB": 1e6, "GB": 1e9}


def _rows(path: str):
    with open(path) as f:
        lines = [ln for ln in f if ln.startswith('"')]
    return list(csv.DictReader(lines))


def summarise(path: str):
    """total device time (ns) and launch count per kernel"""
    tot = collections.defaultdict(float)
    cnt = collections.Counter()
    for r in _rows(path):
        if r.get("Metric Name") != "gpu__time_duration.sum":
            continue
        v = float(r["Metric Value"].replace(",", ""))
        k = kernel_key(r["Kernel Name"])
        tot[k] += v * TIME_SCALE.get(r["Metric Unit"], 1.0)
        cnt[k] += 1
    return tot, cnt


def traffic(path: str, evals: int):
    """per kernel: launches, DRAM bytes (dram__bytes_read.sum +
    dram__bytes_write.sum) per launch and per evaluation, device time per
    launch, from a capture with those metrics"""
    tot, cnt = summarise(path)
    dram = collections.defaultdict(float)
    for r in _rows(path):
        if r.get("Metric Name") not in ("dram__bytes_read.sum", "dram__bytes_write.sum"):
            continue
        v = float(r["Metric Value"].replace(",", ""))
        dram[kernel_key(r["Kernel Name"])] += v * BYTE_SCALE.get(r["Metric Unit"], 1.0)
    out = {}
    for k in cnt:
        out[k] = {"launches_per_eval": cnt[k] / evals, "dram_bytes_per_launch": dram[k] / cnt[k],
                  "dram_bytes_per_eval": dram[k] / evals, "us_per_launch": tot[k] / cnt[k] / 1e3}
    return out


def main():
    p = argparse.ArgumentParser()
    p.add_argument("csv")
    p.add_argument("--evals", type=int, default=1)
    p.add_argument("--traffic-json", help="write per-kernel DRAM traffic (needs the dram__bytes metrics) here")
    p.add_argument("--command", default="", help="the profiled command, recorded in the traffic file")
    p.add_argument("--workload", default="", help="the profiled workload, recorded in the traffic file")
    a = p.parse_args()
    if a.traffic_json:
        with open(a.traffic_json, "w") as f:
            json.dump({"command": a.command, "workload": a.workload, "evals": a.evals,
                       "kernels": traffic(a.csv, a.evals)}, f, indent=1, sort_keys=True)
    tot, cnt = summarise(a.csv)
    all_ns = sum(tot.values())
    print(f"{'kernel':44s} {'launches':>9s} {'total us':>10s} {'share':>7s}")
    for k in sorted(tot, key=lambda k: -tot[k]):
        print(f"{k:44s} {cnt[k] / a.evals:9.1f} {tot[k] / a.evals / 1e3:10.1f} {100 * tot[k] / all_ns:6.1f}%")
    print(f"{'total':44s} {sum(cnt.values()) / a.evals:9.1f} {all_ns / a.evals / 1e3:10.1f}")


if __name__ == "__main__":
    main()
