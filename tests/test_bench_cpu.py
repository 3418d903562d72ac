"""The benchmark's roofline arithmetic (no GPU): pair counts per launch,
flop weights, fractions of the measured peak, and the captured DRAM traffic
reported only for the workload it was captured on."""
import importlib.util
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


PEAKS = {"fp32_tflops": 72.0, "fp64_tflops": 36.0, "ex2_tops": 4.6, "nominal_sm_mhz": 1965.0}


def test_pair_roofline_25k(bench):
    n, nh = 25000, 12500
    stage = {"invb": 0.32, "agb": 0.44, "gbders": 0.74}
    r = bench.pair_roofline(n, nh, stage, PEAKS)
    # unordered pairs, directed pairs with a heavy descreener, pairs with a heavy atom
    agb_flops = n * (n - 1) // 2 * bench.PAIR_OPS["agb"][0]
    invb_flops = (n * nh - nh) * bench.PAIR_OPS["invb"][0]
    gbd_flops = nh * (nh - 1) // 2 * bench.PAIR_OPS["gbders_hh"][0] + nh * (n - nh) * bench.PAIR_OPS["gbders_hx"][0]
    st = r["stages"]
    assert st["agb"]["gflop_per_launch"] == pytest.approx(agb_flops / 1e9)
    assert st["invb"]["gflop_per_launch"] == pytest.approx(invb_flops / 1e9)
    assert st["gbders"]["gflop_per_launch"] == pytest.approx(gbd_flops / 1e9)
    for k, ms in stage.items():
        assert st[k]["fp32_frac"] == pytest.approx(st[k]["gflop_per_launch"] / (ms * 1e-3) / 1e3 / PEAKS["fp32_tflops"])
    # the dominant (slowest) pair kernel carries the headline fraction and its captured traffic
    assert r["kernel"] == "k_gbders_sym" and r["frac"] == st["gbders"]["fp32_frac"]
    assert r["achieved"] == pytest.approx(r["frac"] * r["peak"])
    assert r["traffic"] == bench.NCU_TRAFFIC_25K["k_gbders_sym"]
    tot = sum(st[k]["gflop_per_launch"] for k in stage)
    assert st["all_pair_stages"]["tflops"] == pytest.approx(tot / (sum(stage.values()) * 1e-3) / 1e3)


def test_pair_roofline_other_size_has_no_traffic(bench):
    r = bench.pair_roofline(100000, 50000, {"invb": 4.0, "agb": 6.7, "gbders": 7.6}, PEAKS)
    assert r["kernel"] == "k_gbders_sym" and r["traffic"] is None
    assert 0.0 < r["frac"] < 1.5


def test_metric_name(bench):
    assert bench.metric_name(25000).startswith("energy+grad evals/s @25k atoms")
    assert "@2500 atoms" in bench.metric_name(2500)


def test_reference_arm_line():
    """`bench.py --impl reference` on a small globule: one JSON line with the
    benchmark contract's keys, timing the reference library on host cores."""
    import json
    import subprocess
    import sys
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libagbnp3_ref.so")):
        pytest.skip("reference library not built")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--natoms", "2000",
                          "--steps", "2", "--warmup", "1"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["steps"] == 2
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]


def test_ncu_launch_summary(tmp_path):
    """The launch-list summariser groups kernels by name (template arguments
    kept apart), converts units and skips ncu's banner lines."""
    from agbnp3_b200.ncu_summary import kernel_key, summarise
    hdr = ('"ID","Process ID","Process Name","Host Name","Kernel Name","Context","Stream","Block Size","Grid Size",'
           '"Device","CC","Section Name","Metric Name","Metric Unit","Metric Value"\n')
    rows = [("k_prep(View)", "ns", "6,000"), ("void k_tree_ders<float, 3>(View)", "us", "40.5"),
            ("void k_tree_ders<float, 3>(View)", "us", "39.5"), ("void k_tree_ders<float, 4>(View)", "ns", "1000")]
    text = "==PROF== Connected\n" + hdr + "".join(
        f'"{i}","1","py","h","{k}","1","13","(128, 1, 1)","(1, 1, 1)","0","10.0","s","gpu__time_duration.sum","{u}","{v}"\n'
        for i, (k, u, v) in enumerate(rows))
    p = tmp_path / "launches.csv"
    p.write_text(text)
    tot, cnt = summarise(str(p))
    assert kernel_key("void k_tree_ders<float, 3>(View)") == "k_tree_ders<float, 3>"
    assert cnt["k_tree_ders<float, 3>"] == 2 and tot["k_tree_ders<float, 3>"] == pytest.approx(80000.0)
    assert tot["k_prep"] == pytest.approx(6000.0) and tot["k_tree_ders<float, 4>"] == pytest.approx(1000.0)
