"""The oracle's supernode rule against the reference's own supernode kernel.
The unmodified SOA kernel warpcentric_local_detection_test
(gSoFa_SOAComparison/symbfact_warp_centric_new_scheduling.cuh:1790-2123)
was run on a B200 through oracle/_ref/soa_supernodes (oracle/ref_soa.py) on
the oracle's nz_row_U counters and L rows of the matrices of
tests/reference_inputs.py, at the reference's 128 and at chunk sizes that
are not multiples of its 128 threads; its counts and starts per chunk are
committed in tests/golden/reference_soa.json (tests/golden/
make_reference_soa.py).  or_supernodes must give the same on every one --
for BC at 128 rows, the reference's 6,800."""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests import reference_inputs as RI
from tests.golden.make_reference_soa import CASES, inputs_hash

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
REF = json.load(open(os.path.join(GOLD, "reference_soa.json")))["records"]


def test_every_case_was_run():
    assert set(REF) == {"%s_mss%d" % c for c in CASES}
    assert REF["bc_mss128"]["printed_reference"] == 6800


@pytest.mark.parametrize("label,mss", [c for c in CASES if c[0] != "grid3d_64"])
def test_oracle_rule_equals_reference_kernel(label, mss):
    rec = REF["%s_mss%d" % (label, mss)]
    beg, end, col = RI.build(label)
    r = O.rows(beg, end, col, pattern=True)
    assert inputs_hash(r["nzU_ref"], r["Lptr"], r["Lcols"]) == rec["inputs_sha16"]
    # a supernode never spans a forced start (offsets 0, 128, ... of a chunk),
    # so the 128-bit L masks suffice for any chunk size
    detected, flags = O.supernodes(r["nzU_ref"], r["lback"], mss)
    assert detected == rec["detected_reference"]
    n = len(beg)
    starts = [int(np.sum(flags[c * mss:min(n, (c + 1) * mss)] == 1))
              for c in range((n + mss - 1) // mss)]
    assert hashlib.sha256(np.asarray(starts, np.int32).tobytes()).hexdigest()[:16] == \
        rec["starts_per_chunk_sha16"]


def test_oracle_rule_equals_reference_kernel_on_the_grid():
    """64^3 grid at mss 256: the committed full-size record (every row)."""
    fx = json.load(open(os.path.join(GOLD, "fullsize_c3.json")))["records"][0]
    rec = REF["grid3d_64_mss256"]
    assert fx["mss"] == 256 and fx["totals"]["n_supernodes"] == rec["printed_reference"]
