"""Records the reference's own supernode kernel's answers: for each matrix of
tests/reference_inputs.py (and each max_supernode_size listed below) the
oracle's nz_row_U counters and L rows are fed to the unmodified SOA kernel
through oracle/_ref/soa_supernodes (see oracle/ref_soa.py) on a GPU machine;
its detected count and starts per chunk are written, with a hash of the
inputs, to tests/golden/reference_soa.json.  tests/test_reference_spo.py
checks the oracle's rule against them on the CPU.

Usage (GPU machine): python tests/golden/make_reference_soa.py
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from oracle import ref_soa  # noqa: E402
from tests import reference_inputs as RI  # noqa: E402

# (input, max_supernode_size): the reference's 128, the 64^3 grid's 256, and
# chunk sizes that are not multiples of the kernel's 128 threads
CASES = [("bc", 128), ("bc", 64), ("bc", 200), ("random_extra", 128), ("grid3d_64", 256),
         ("circuit_20k", 128), ("banded_3000", 128), ("grid2d_45", 8)] + \
        [("rand_%d" % k, [4, 8, 128, 200, 256, 16, 32, 100][k]) for k in range(8)]


def inputs_hash(nz, lptr, lcols):
    h = hashlib.sha256()
    for a in (np.ascontiguousarray(nz, np.int32), np.ascontiguousarray(lptr, np.int64),
              np.ascontiguousarray(lcols, np.int32)):
        h.update(a.tobytes())
    return h.hexdigest()[:16]


def main():
    recs = {}
    for label, mss in CASES:
        beg, end, col = RI.build(label)
        r = O.rows(beg, end, col, pattern=True)
        t0 = time.time()
        nsup, starts = ref_soa.run(r["nzU_ref"], r["Lptr"], r["Lcols"], mss)
        key = "%s_mss%d" % (label, mss)
        recs[key] = {"label": label, "mss": mss, "n": len(beg),
                     "inputs_sha16": inputs_hash(r["nzU_ref"], r["Lptr"], r["Lcols"]),
                     "detected_reference": nsup, "printed_reference": nsup + 1,
                     "starts_per_chunk_sha16": hashlib.sha256(
                         np.asarray(starts, np.int32).tobytes()).hexdigest()[:16],
                     "seconds": round(time.time() - t0, 2)}
        print(key, nsup + 1, flush=True)
    with open(os.path.join(HERE, "reference_soa.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_reference_soa.py",
                   "kernel": "warpcentric_local_detection_test, unmodified SOA header, sm_100a",
                   "records": recs}, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
