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


def test_pair_roofline_25k(bench, tmp_path, monkeypatch):
    import json
    tr = tmp_path / "traffic.json"
    tr.write_text(json.dumps({"command": "ncu ...", "workload": "w", "evals": 2,
                              "kernels": {"k_gbders_x2<1>": {"dram_bytes_per_launch": 2.5e6, "dram_bytes_per_eval": 2.5e6,
                                                           "launches_per_eval": 1, "us_per_launch": 700.0}}}))
    monkeypatch.setattr(bench, "TRAFFIC_JSON", str(tr))
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
    assert r["kernel"] == "k_gbders_x2" and r["frac"] == st["gbders"]["fp32_frac"]
    assert r["achieved"] == pytest.approx(r["frac"] * r["peak"])
    assert r["traffic"] == 2.5e6 and "ncu ..." in r["traffic_note"]
    tot = sum(st[k]["gflop_per_launch"] for k in stage)
    assert st["all_pair_stages"]["tflops"] == pytest.approx(tot / (sum(stage.values()) * 1e-3) / 1e3)


def test_pair_roofline_other_size_has_no_traffic(bench):
    r = bench.pair_roofline(100000, 50000, {"invb": 4.0, "agb": 6.7, "gbders": 7.6}, PEAKS)
    assert r["kernel"] == "k_gbders_x2" and r["traffic"] is None
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


def test_tree_roofline(bench):
    """HBM roofline of the O(N) stages: algorithmic bytes from the counts,
    fraction of the HBM peak, and the captured DRAM bytes of the stage's
    kernels when a traffic record is given."""
    counts = {"near_pairs": 300000, "kept": [160000, 350000, 240000, 60000], "water_sites": 6000}
    stage = {"nblist": 0.1, "volumes": 0.16, "ws": 0.1, "treeders": 0.12}
    tr = {"kernels": {"k_nl_slab": {"dram_bytes_per_eval": 1e6}, "k_cell_fill": {"dram_bytes_per_eval": 2e5},
                      "k_tree_ders<float, 2>": {"dram_bytes_per_eval": 3e6}}}
    r = bench.tree_roofline(25000, 12500, counts, stage, 6500.0, 4, tr)
    assert r["nblist"]["alg_bytes"] == 16 * 12500 + 8 * 300000 + 8 * 12500
    rec = sum(k * (32 + 4 * m) for m, k in zip(range(2, 6), counts["kept"]))
    assert r["treeders"]["alg_bytes"] == rec + 32 * 12500 + 96 * 25000
    for k, e in r.items():
        assert e["achieved_gbs"] == pytest.approx(e["alg_bytes"] / (stage[k] * 1e-3) / 1e9)
        assert e["frac_of_hbm"] == pytest.approx(e["achieved_gbs"] / 6500.0)
    assert r["nblist"]["dram_bytes_ncu"] == pytest.approx(1.2e6)
    assert r["treeders"]["dram_bytes_ncu"] == pytest.approx(3e6)
    assert r["ws"]["dram_bytes_ncu"] == 0


def test_ncu_traffic_summary(tmp_path):
    """DRAM bytes per launch and per evaluation from a capture with the
    dram__bytes metrics (units converted)."""
    from agbnp3_b200.ncu_summary import traffic
    hdr = ('"ID","Process ID","Process Name","Host Name","Kernel Name","Context","Stream","Block Size","Grid Size",'
           '"Device","CC","Section Name","Metric Name","Metric Unit","Metric Value"\n')
    rows = []
    for i in range(2):
        rows += [(i, "k_agb_sym(View)", "gpu__time_duration.sum", "us", "450"),
                 (i, "k_agb_sym(View)", "dram__bytes_read.sum", "Mbyte", "1.5"),
                 (i, "k_agb_sym(View)", "dram__bytes_write.sum", "Kbyte", "500")]
    text = hdr + "".join(f'"{i}","1","py","h","{k}","1","13","(128, 1, 1)","(1, 1, 1)","0","10.0","s","{m}","{u}","{v}"\n'
                         for i, k, m, u, v in rows)
    p = tmp_path / "cap.csv"
    p.write_text(text)
    t = traffic(str(p), evals=2)
    assert t["k_agb_sym"]["dram_bytes_per_launch"] == pytest.approx(2.0e6)
    assert t["k_agb_sym"]["dram_bytes_per_eval"] == pytest.approx(2.0e6)
    assert t["k_agb_sym"]["us_per_launch"] == pytest.approx(450.0)
