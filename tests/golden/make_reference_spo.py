"""Records the reference's own answers: runs the unmodified SPO build
(oracle/_ref/spo_symbfact, `make -C oracle ref` in a checkout with the
reference tree) on a GPU machine over the matrices of
tests/reference_inputs.py, after oracle/ref_spo.check has cleared each input
and pool size, and writes the fill counts it prints, with the time its own
timer reports for the fill detection, to tests/golden/reference_spo.json.
tests/test_reference_spo.py then checks the oracle against them on the CPU;
bench.py --workload reference_build times this library on the same inputs.

Usage (GPU machine): python tests/golden/make_reference_spo.py [label ...]
"""
import json
import os
import re
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref_spo  # noqa: E402
from tests import reference_inputs as RI  # noqa: E402


def main():
    labels = sys.argv[1:] or list(RI.INPUTS)
    out_path = os.path.join(HERE, "reference_spo.json")
    recs = json.load(open(out_path))["records"] if os.path.exists(out_path) else {}
    for label in labels:
        spec = RI.INPUTS[label]
        beg, end, col = RI.build(label)
        v = spec.get("virtual_gpus", 1)
        gb = spec.get("memory_gb") or ref_spo.min_memory_gb(beg, end, col)
        why = ref_spo.check(beg, end, col, v, gb)
        if why:
            print(label, "refused:", why, flush=True)
            continue
        t0 = time.time()
        fills, out = ref_spo.run(beg, end, col, v, gb, timeout=spec.get("timeout", 600))
        dt = time.time() - t0
        tail = [ln.strip() for ln in out.splitlines()
                if ln.strip().startswith(("vertex count", "Total Number", "GPU:"))]
        # the reference's own timer around its fill detection (symbfact.cuh:2004, :2420),
        # printed per virtual GPU (:2530); with one virtual GPU, the whole run
        m = re.search(r"Slowest virtual GPU takes: ([0-9.eE+-]+) ms", out)
        recs[label] = {"n": len(beg), "nnz": len(col), "virtual_gpus": v, "memory_gb": gb,
                       "fills_reference": fills, "seconds": round(dt, 2), "printed": tail,
                       "ms_reference": float(m.group(1)) if m else None}
        print(label, len(beg), fills, "%.1f s" % dt, flush=True)
        with open(out_path, "w") as f:
            json.dump({"generator": "tests/golden/make_reference_spo.py",
                       "binary": "SpaceOptimization/main.cu + symbfact.cuh, unmodified, sm_100a",
                       "records": recs}, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
