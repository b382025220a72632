"""Generates the full-size parity fixtures tests/golden/fullsize_<config>.json
with the CPU oracle over EVERY row (and, for unsymmetric patterns, every
row of A^T) of the five benchmark workloads:

  c1  n=20,000 random: diagonal + tridiagonal + 3 uniform columns/row, mss 128
  c2  circuit-like n=659,033 (~5.84M nnz), mss 128
  c3  64^3 7-point grid in nested-dissection order, mss 256
  c4  the 512-matrix batch mix (2D 5-point ND grids and random-banded), mss 128
  c5  the 48-request serving stream (gen.SERVE_STREAM), mss 128

Each fixture holds, per matrix, the totals and per-row array hashes of
tests/fullsize.py.  Seeded generators rebuild the matrices, so no matrix is
stored.  The whole set takes a few CPU-hours (c2 and c4 dominate).

Usage: python tests/golden/make_fullsize.py [--threads T] c1 c3 c2 c4 c5
"""
import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from gsofatpds_b200 import gen  # noqa: E402
from tests import fullsize as F  # noqa: E402


def workloads(name):
    """[(label, (n, rowptr, col), mss)] of one benchmark workload."""
    if name == "c1":
        return [("random_extra_20000", gen.random_extra(20000, 3, seed=1), 128)]
    if name == "c2":
        return [("circuit_like_659033", gen.circuit_like(), 128)]
    if name == "c3":
        return [("grid3d_64_7pt", gen.grid_nd((64, 64, 64), "7"), 256)]
    if name == "c4":
        return [("batch_%03d" % k, m, 128) for k, m in enumerate(gen.batch_mix(512))]
    if name == "c5":
        out = []
        for k, (_, kind, spec) in enumerate(gen.request_stream(**gen.SERVE_STREAM)):
            out.append(("request_%02d_%s_%d" % (k, kind, spec["n"]), gen.make_request(kind, spec),
                        128))
        return out
    raise SystemExit("unknown workload " + name)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("configs", nargs="+")
    a = ap.parse_args()
    for name in a.configs:
        t0 = time.time()
        recs = []
        for label, (n, rp, col), mss in workloads(name):
            beg, end = gen.csr_to_beg_end(rp)
            rec = F.oracle_record(beg, end, col, mss, nthreads=a.threads)
            rec["label"] = label
            recs.append(rec)
            print("%s %s n=%d fills=%d %.0f s" % (name, label, n, rec["totals"]["fill_count"],
                                                  time.time() - t0), flush=True)
        out = {"workload": name, "generator": "tests/golden/make_fullsize.py",
               "oracle": "oracle/gsofa_oracle.c (or_rows over every row of A and A^T)",
               "records": recs}
        with open(os.path.join(HERE, "fullsize_%s.json" % name), "w") as f:
            json.dump(out, f, indent=0, sort_keys=True)
        print("%s done in %.0f s" % (name, time.time() - t0), flush=True)


if __name__ == "__main__":
    main()
