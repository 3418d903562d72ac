"""Summarises an ncu launch list (``--metrics gpu__time_duration.sum --csv``)
per kernel: launches, total device time and share of the total.

    python -m agbnp3_b200.ncu_summary launches.csv [--evals N]

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
import re


def kernel_key(name: str) -> str:
    name = re.sub(r"\(View.*$|\(const .*$|\(int.*$|\(double.*$|\(float.*$", "", name)
    name = re.sub(r"^void ", "", name)
    return name.strip()


def summarise(path: str):
    tot = collections.defaultdict(float)
    cnt = collections.Counter()
    with open(path) as f:
        lines = [ln for ln in f if ln.startswith('"')]
    for r in csv.DictReader(lines):
        if r.get("Metric Name") != "gpu__time_duration.sum":
            continue
        v = float(r["Metric Value"].replace(",", ""))
        scale = {"ns": 1.0, "us": 1e3, "usecond": 1e3, "ms": 1e6, "msecond": 1e6}.get(r["Metric Unit"], 1.0)
        k = kernel_key(r["Kernel Name"])
        tot[k] += v * scale
        cnt[k] += 1
    return tot, cnt


def main():
    p = argparse.ArgumentParser()
    p.add_argument("csv")
    p.add_argument("--evals", type=int, default=1)
    a = p.parse_args()
    tot, cnt = summarise(a.csv)
    all_ns = sum(tot.values())
    print(f"{'kernel':44s} {'launches':>9s} {'total us':>10s} {'share':>7s}")
    for k in sorted(tot, key=lambda k: -tot[k]):
        print(f"{k:44s} {cnt[k] / a.evals:9.1f} {tot[k] / a.evals / 1e3:10.1f} {100 * tot[k] / all_ns:6.1f}%")
    print(f"{'total':44s} {sum(cnt.values()) / a.evals:9.1f} {all_ns / a.evals / 1e3:10.1f}")


if __name__ == "__main__":
    main()
