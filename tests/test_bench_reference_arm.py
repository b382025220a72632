"""bench.py's reference arm runs on the host cores only (no GPU): its JSON
line must carry the contract's keys."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--workload", "random_extra", "--steps", "1", "--warmup", "0"],
                         capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads([x for x in out.stdout.splitlines() if x.startswith("{")][-1])
    assert line["impl"] == "reference"
    assert line["metric"] == "fill_path_gteps" and line["unit"] == "GTEPS"
    assert line["value"] > 0 and line["higher_is_better"] is True
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["e2e"]["value"] == line["value"]


def test_reference_arm_without_a_counterpart_is_unavailable():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--workload", "order"], capture_output=True, text=True, timeout=120,
                         cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads([x for x in out.stdout.splitlines() if x.startswith("{")][-1])
    assert line["impl"] == "reference" and "unavailable" in line


def test_roofline_entry():
    """The roofline object is the hardware one: measured DRAM bytes per
    launch over the kernel time, as a fraction of the measured peak; the
    algorithmic (work-equivalent) rate is reported beside it, not as frac."""
    sys.path.insert(0, ROOT)
    import bench
    # config 2's numbers: E_alg, V_alg, edges inspected, n, kernel ms, peak, ncu bytes per launch
    r = bench.roofline_entry(1316542257033, 148212479438, 63747717944, 659033, 871.76, 6456.2,
                             "measured", 548526653696.0)
    assert r["bound"] == "hbm" and r["unit"] == "GB/s"
    assert abs(r["achieved"] - 548526653696.0 / 0.87176 / 1e9) < 1e-6
    assert abs(r["frac"] - r["achieved"] / 6456.2) < 1e-12
    assert 0.09 < r["frac"] < 0.11
    we = r["work_equivalent"]
    assert we["bytes_alg"] == 8 * 1316542257033 + 16 * 148212479438 + 4 * 11 * 659033
    assert we["gbs"] > r["peak"]  # closure reuse: not a bandwidth fraction
    assert abs(r["inspected_edges_per_s"] - 63747717944 / 0.87176) < 1.0
    r0 = bench.roofline_entry(10, 1, 4, 5, 1.0, 100.0, "fallback", None)
    assert r0["traffic"] is None and r0["achieved"] is None and r0["frac"] is None


def test_roofline_traffic_matches_its_profile():
    """The traffic the bench line reports is the committed ncu summary's
    read + write bytes of one full-size traversal launch."""
    import glob
    import importlib.util
    import re
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    seen = 0
    for path in glob.glob(os.path.join(ROOT, "profiles", "traverse_*.md")):
        text = open(path).read()
        if "dram_bytes_per_launch:" not in text:
            continue
        workload = os.path.basename(path)[len("traverse_"):-len(".md")]
        rd = re.search(r"\| dram__bytes_read\.sum \| ([0-9,]+) B \|", text)
        wr = re.search(r"\| dram__bytes_write\.sum \| ([0-9,]+) B \|", text)
        assert rd and wr, path
        total = int(rd.group(1).replace(",", "")) + int(wr.group(1).replace(",", ""))
        assert bench.read_traffic(workload) == total, (path, total)
        seen += 1
    assert seen >= 1
    roof = bench.roofline_entry(1e12, 1e9, 1e10, 1000, 500.0, 6450.9, "measured", 3.2e11)
    assert abs(roof["achieved"] - 640.0) < 1e-6 and abs(roof["frac"] - 640.0 / 6450.9) < 1e-12
