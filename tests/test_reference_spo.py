"""The oracle against the reference's own CUDA build.  The unmodified SPO
binary (SpaceOptimization/main.cu + symbfact.cuh, compiled for sm_100a by
oracle/Makefile's `ref` target) was run on a B200 over the matrices of
tests/reference_inputs.py -- after oracle/ref_spo.check had shown that it
bounds every device write for each input -- and its printed fill counts are
committed in tests/golden/reference_spo.json (tests/golden/
make_reference_spo.py).  The oracle must give the same count on every one:
the reference's BC matrix, the n=20,000 random and 64^3 grid benchmark
matrices, a circuit-like, a banded and a grid matrix, and small patterns in
the reference's raw layout (rows out of order, columns unsorted,
duplicates)."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests import reference_inputs as RI

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
REF = json.load(open(os.path.join(GOLD, "reference_spo.json")))["records"]


def test_every_input_was_run():
    assert set(REF) == set(RI.INPUTS)
    assert REF["bc_264"]["fills_reference"] == 980136  # the reference's own log
    assert REF["bc_264"]["virtual_gpus"] == 264 and REF["bc_264"]["memory_gb"] == 5.0


@pytest.mark.parametrize("label", sorted(k for k in RI.INPUTS if k != "grid3d_64"))
def test_oracle_equals_reference_build(label):
    beg, end, col = RI.build(label)
    rec = REF[label]
    assert rec["n"] == len(beg) and rec["nnz"] == len(col)
    r = O.rows(beg, end, col)
    assert int(r["fills"].sum()) == rec["fills_reference"]


def test_oracle_equals_reference_build_on_the_grid():
    """64^3 grid: the oracle's full-size record (tests/golden/fullsize_c3.json,
    every row) against the reference build's count."""
    fx = json.load(open(os.path.join(GOLD, "fullsize_c3.json")))["records"][0]
    assert fx["n"] == REF["grid3d_64"]["n"] and fx["nnz"] == REF["grid3d_64"]["nnz"]
    assert fx["totals"]["fill_count"] == REF["grid3d_64"]["fills_reference"]


def test_reference_sizing_check_refuses_unbounded_inputs():
    """The host-side restatement of the reference's sizing refuses what the
    binary would not bound: short row files, label offsets that wrap, and
    pools too small for the seeding queue."""
    from oracle import ref_spo
    n = 50
    beg = np.arange(n, dtype=np.int32)
    end = beg + 1
    col = np.arange(n, dtype=np.int32)
    assert ref_spo.check(beg, end, col, 1, 1.0) is None
    assert "fewer entries" in ref_spo.check(beg[:n], end[:n] * 0 + beg[:n], col[:10], 1, 1.0)
    # a pool of a few hundred words leaves no room for labels, markers and queues
    assert ref_spo.check(beg, end, col, 1, 1e-6) is not None
    # a row list whose entries fall outside the entry array
    assert "outside" in ref_spo.check(beg, end + 100, col, 1, 1.0)
    assert ref_spo.compute_src_group_original(11948) == 4096
    assert ref_spo.compute_src_group_original(262144) == 2048
