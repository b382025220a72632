"""Full-size parity: every row and column of the five benchmark workloads on
the device against the oracle's committed answers (tests/golden/
fullsize_<config>.json, made by tests/golden/make_fullsize.py from or_rows
over every row of A and A^T).  Nothing is sampled: each per-row array
(U-row / L-column / L-row counts, nz_row_U, the three digests, the 128-bit
L-column masks and the supernode flags) must hash to the oracle's value and
every total must be equal.

  c1  n=20,000 random, plain call
  c2  circuit-like n=659,033 (the benchmark matrix), plain call
  c3  64^3 7-point ND grid, mss 256, plain call
  c4  the 512-matrix mix: the graph-captured batch, and every matrix alone
  c5  the 48-request serving stream, all requests served in one request loop
"""
import json
import os

import pytest

from tests import fullsize as F

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def fixture(name):
    p = os.path.join(GOLD, "fullsize_%s.json" % name)
    with open(p) as f:
        return json.load(f)["records"]


@pytest.fixture(scope="module")
def ctx():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gsofatpds_b200 import Context
    c = Context(0)
    yield c
    c.close()


def _plain(ctx, n_rp_col, mss):
    n, rp, col = n_rp_col
    m = ctx.load_rowptr(rp, col)
    res = ctx.factor(m, max_supernode_size=mss, l_row_stats=True)
    rec = F.device_record(res, l_rows=True)
    res.close()
    m.close()
    return rec


def test_c1_random_extra_every_row(ctx):
    from gsofatpds_b200 import gen
    ref, = fixture("c1")
    F.compare(_plain(ctx, gen.random_extra(20000, 3, seed=1), 128), ref, "c1")


def test_c3_grid3d_64_every_row(ctx):
    from gsofatpds_b200 import gen
    ref, = fixture("c3")
    F.compare(_plain(ctx, gen.grid_nd((64, 64, 64), "7"), 256), ref, "c3")


def test_c2_circuit_like_every_row(ctx):
    """The benchmark matrix: all 659,033 U rows, L columns and L rows, and
    the full supernode partition."""
    from gsofatpds_b200 import gen
    ref, = fixture("c2")
    F.compare(_plain(ctx, gen.circuit_like(), 128), ref, "c2")


def test_c4_batch_and_alone_every_matrix(ctx):
    from gsofatpds_b200 import gen
    refs = fixture("c4")
    mats_np = gen.batch_mix(512)
    assert len(refs) == len(mats_np)
    mats = [ctx.load_rowptr(rp, col) for (_, rp, col) in mats_np]
    b = ctx.batch(mats, max_supernode_size=128, l_row_stats=True)
    b.run()
    for i, ref in enumerate(refs):
        F.compare(F.device_record(b.result(i), l_rows=True), ref, "c4 batch %d" % i)
    b.close()
    for i, (m, ref) in enumerate(zip(mats, refs)):
        res = ctx.factor(m, max_supernode_size=128, l_row_stats=True)
        F.compare(F.device_record(res, l_rows=True), ref, "c4 alone %d" % i)
        res.close()
    for m in mats:
        m.close()


def test_c5_served_stream_every_request(ctx):
    """All 48 requests of the serving stream (largest: the 100^3 27-point
    grid, n = 1,000,000) submitted to one request loop at once, so that
    they overlap on the device; each served result against the oracle."""
    from gsofatpds_b200 import gen
    refs = fixture("c5")
    stream = gen.request_stream(**gen.SERVE_STREAM)
    assert len(refs) == len(stream)
    reqs = [gen.make_request(kind, spec) for (_, kind, spec) in stream]
    max_n = max(n for (n, _, _) in reqs)
    with ctx.server(max_n, max_supernode_size=128, l_row_stats=True) as srv:
        tickets = [srv.submit_rowptr(rp, col) for (_, rp, col) in reqs]
        for k, (t, ref) in enumerate(zip(tickets, refs)):
            res = srv.wait(t, timeout_ms=600000)
            assert res is not None, "request %d timed out" % k
            F.compare(F.device_record(res, l_rows=True), ref, "c5 request %d" % k)
            res.close()
