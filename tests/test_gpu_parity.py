"""GPU parity: the CUDA path (through the C-ABI) against the CPU oracle.

Every comparison is bit-exact (integer counts, 64-bit digests, patterns,
supernode flags).  Full-size workloads are checked on sampled rows and
chunks plus size-independent identities."""
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import load_bc, random_pattern, scrambled_csr

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gsofatpds_b200 import Context
    c = Context(0)
    yield c
    c.close()


def colmask_from_lback(lback):
    """Column-side 128-bit masks (bit j: L(f+1+j, f)) from the oracle's
    row-side masks (bit j: L(r, r-1-j)); both index the same j."""
    n = lback.shape[0]
    cm = np.zeros((n, 4), np.uint32)
    for j in range(128):
        if j + 1 >= n:
            break
        w, b = j >> 5, np.uint32(j & 31)
        bits = (lback[j + 1:, w] >> b) & np.uint32(1)
        cm[:n - j - 1, w] |= bits << b
    return cm


def oracle_full(beg, end, col, pattern=False):
    r = O.rows(beg, end, col, pattern=pattern)
    tb, te, tc = O.transpose(beg, end, col)
    rt = O.rows(tb, te, tc, pattern=pattern)
    return r, rt


def check_full(res, r, rt, mss=128, l_rows=True, supernodes=True):
    rc = res.row_counts(l_rows=l_rows)
    np.testing.assert_array_equal(rc["nnz_u_row"], r["nnzU"])
    np.testing.assert_array_equal(rc["nz_row_u"], r["nzU_ref"])
    np.testing.assert_array_equal(rc["nnz_l_col"], rt["nnzU"])
    if l_rows:
        np.testing.assert_array_equal(rc["nnz_l_row"], r["nnzL"])
    dg = res.digests(l_rows=l_rows)
    np.testing.assert_array_equal(dg["dig_u_row"], r["digU"])
    np.testing.assert_array_equal(dg["dig_l_col"], rt["digU"])
    if l_rows:
        np.testing.assert_array_equal(dg["dig_l_row"], r["digL"])
    np.testing.assert_array_equal(res.lmask(), colmask_from_lback(r["lback"]))
    c = res.counts
    assert c["fill_count"] == int(r["fills"].sum())
    assert c["nnz_u"] == int(r["nnzU"].sum()) and c["nnz_l"] == int(r["nnzL"].sum())
    assert c["edges_alg"] == int(r["e_alg"].sum())
    assert c["vertices_alg"] == int(r["v_alg"].sum())
    if supernodes:
        nsup, flags = O.supernodes(r["nzU_ref"], r["lback"], mss)
        gflags, _ = res.supernodes()
        np.testing.assert_array_equal(gflags, flags)
        assert c["n_supernodes"] == nsup + 1


# traversal modes: defaults; bottom-up as early as possible with warp-walked
# rows from 4 entries, 7-source chunks and 2 cached closures; top-down only
# without closure reuse; bottom-up without switching back, 1000-source chunks
# and 32 cached closures
MODES = [dict(), dict(bu_alpha=1000, bu_min_source=1, heavy_row=4, chunk_sources=7,
                     cached_closures=2),
         dict(bu_alpha=-1, heavy_row=8, merge=False),
         dict(bu_alpha=2, bu_beta=1, bu_min_source=1, chunk_sources=1000, cached_closures=32)]


@pytest.fixture(scope="module")
def bc_oracle():
    z = load_bc()
    return z, oracle_full(z["beg"], z["end"], z["col"], pattern=True)


@pytest.mark.parametrize("mode", range(4))
def test_bc_matches_reference_and_oracle(ctx, bc_oracle, mode):
    z, (r, rt) = bc_oracle
    m = ctx.load_csr(z["beg"], z["end"], z["col"])  # non-contiguous, unsorted rows
    res = ctx.factor(m, l_row_stats=True, pattern=True, **MODES[mode])
    c = res.counts
    assert c["fill_count"] == 980136  # reference log, with_supernodes/...warp_centric.dat:2
    assert c["n_supernodes"] == 6800
    check_full(res, r, rt)
    up, uc = res.pattern_u()
    np.testing.assert_array_equal(up, r["Uptr"])
    np.testing.assert_array_equal(uc, r["Ucols"])
    lp, lr = res.pattern_l()
    np.testing.assert_array_equal(lp, rt["Uptr"])
    np.testing.assert_array_equal(lr, rt["Ucols"])
    res.close()
    m.close()


@pytest.mark.parametrize("seed", range(12))
def test_random_small_patterns(ctx, seed):
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(1, 300))
    pat = random_pattern(rng, n, float(rng.uniform(0.002, 0.05)), diag=bool(seed % 3))
    if seed % 5 == 1 and n > 3:
        pat[1] = set()  # an empty row
    beg, end, col = scrambled_csr(rng, pat, dup_prob=0.3 if seed % 4 == 0 else 0.0)
    m = ctx.load_csr(beg, end, col)
    mss = [4, 8, 128, 200, 256][seed % 5]
    res = ctx.factor(m, max_supernode_size=mss, l_row_stats=True, pattern=True,
                     threads_per_source=[128, 256, 512, 1024][seed % 4], **MODES[(seed // 3) % 4])
    r, rt = oracle_full(beg, end, col, pattern=True)
    check_full(res, r, rt, mss=mss)
    up, uc = res.pattern_u()
    np.testing.assert_array_equal(uc, r["Ucols"])
    lp, lr = res.pattern_l()
    np.testing.assert_array_equal(lr, rt["Ucols"])
    res.close()
    m.close()


def test_launch_shapes_agree(ctx):
    from gsofatpds_b200 import gen
    n, rp, col = gen.random_banded(3000, bw=6, extra=2, seed=11)
    m = ctx.load_rowptr(rp, col)
    base = None
    for k, (tps, inflight) in enumerate([(128, 0), (256, 3), (512, 1), (1024, 0), (512, 0),
                                         (256, 0), (512, 2), (1024, 5)]):
        res = ctx.factor(m, threads_per_source=tps, sources_in_flight=inflight, l_row_stats=True,
                         **MODES[k % 4])
        got = (res.row_counts(l_rows=True), res.digests(l_rows=True), res.supernodes()[0],
               res.counts["fill_count"])
        if base is None:
            base = got
        else:
            for a, b in zip(base[0].values(), got[0].values()):
                np.testing.assert_array_equal(a, b)
            for a, b in zip(base[1].values(), got[1].values()):
                np.testing.assert_array_equal(a, b)
            np.testing.assert_array_equal(base[2], got[2])
            assert base[3] == got[3]
        res.close()
    m.close()


def test_random_extra_20000_full(ctx):
    """Plain factorization, n=20,000 with 3 uniform extra columns per row:
    pattern, per-row counts and supernodes against the full oracle."""
    from gsofatpds_b200 import gen
    n, rp, col = gen.random_extra(20000, 3, seed=1)
    beg, end = gen.csr_to_beg_end(rp)
    m = ctx.load_rowptr(rp, col)
    res = ctx.factor(m, l_row_stats=True, pattern=True)
    r, rt = oracle_full(beg, end, col)
    check_full(res, r, rt)
    up, uc = res.pattern_u()
    np.testing.assert_array_equal(np.diff(up), r["nnzU"])
    rows = np.array([0, 1, 777, 10000, 19998, 19999], np.int32)
    rs = O.rows(beg, end, col, rows=rows, pattern=True)
    for i, s in enumerate(rows):
        np.testing.assert_array_equal(uc[up[s]:up[s + 1]], rs["Ucols"][rs["Uptr"][i]:rs["Uptr"][i + 1]])
    # every row strictly increasing and inside (s, n)
    rowid = np.repeat(np.arange(n), np.diff(up))
    assert np.all(uc > rowid) and np.all(uc < n)
    same = rowid[1:] == rowid[:-1]
    assert np.all(np.diff(uc.astype(np.int64))[same] > 0)
    res.close()
    m.close()


def _chunk_supernode_flags(beg, end, col, n, mss, chunks):
    """Oracle supernode flags for whole chunks only (rows of other chunks are
    never read by the rule)."""
    out = {}
    for c in chunks:
        lo, hi = c * mss, min(n, (c + 1) * mss)
        rows = np.arange(lo, hi, dtype=np.int32)
        rr = O.rows(beg, end, col, rows=rows)
        fl = np.zeros(hi - lo, np.int8)
        nz = np.zeros(hi - lo, np.int32)
        nz[:] = rr["nzU_ref"]
        # the rule inside one chunk, on a matrix re-based at the chunk start
        k, fl = O.supernodes(nz, rr["lback"], mss)
        out[c] = fl
    return out


def test_grid3d_64_sampled(ctx):
    """64^3 7-point grid in nested-dissection order, supernodes with
    max supernode width 256: sampled rows and whole sampled chunks."""
    from gsofatpds_b200 import gen
    n, rp, col = gen.grid_nd((64, 64, 64), "7")
    beg, end = gen.csr_to_beg_end(rp)
    m = ctx.load_rowptr(rp, col)
    res = ctx.factor(m, max_supernode_size=256)
    rc = res.row_counts()
    dg = res.digests()
    rng = np.random.default_rng(3)
    rows = np.sort(rng.choice(n, 200, replace=False)).astype(np.int32)
    rows = np.unique(np.concatenate([rows, [0, n - 1, n - 2]]).astype(np.int32))
    rr = O.rows(beg, end, col, rows=rows)
    np.testing.assert_array_equal(rc["nnz_u_row"][rows], rr["nnzU"])
    np.testing.assert_array_equal(rc["nz_row_u"][rows], rr["nzU_ref"])
    np.testing.assert_array_equal(dg["dig_u_row"][rows], rr["digU"])
    # symmetric pattern: L column m has the same ids as U row m
    bad = np.nonzero(rc["nnz_l_col"] != rc["nnz_u_row"])[0].astype(np.int32)
    if bad.size:
        rb = O.rows(beg, end, col, rows=bad[:8])
        pytest.fail("L column / U row counts differ at %s: L col %s, U row %s, oracle %s" % (
            bad[:8].tolist(), rc["nnz_l_col"][bad[:8]].tolist(), rc["nnz_u_row"][bad[:8]].tolist(),
            rb["nnzU"].tolist()))
    flags, _ = res.supernodes()
    chunks = [0, 1, 500, (n - 1) // 256]
    ref = _chunk_supernode_flags(beg, end, col, n, 256, chunks)
    for c, fl in ref.items():
        np.testing.assert_array_equal(flags[c * 256:c * 256 + fl.shape[0]], fl)
    c = res.counts
    assert c["nnz_u"] == int(rc["nnz_u_row"].sum())
    assert c["fill_count"] == c["nnz_u"] + c["nnz_l"] - (int(rp[-1]) - n)
    res.close()
    m.close()


def test_circuit_like_sampled(ctx):
    """Circuit-like n=659,033 (~5.83M nnz): sampled U rows and L columns
    against the oracle, plus identities over all rows."""
    from gsofatpds_b200 import gen
    n, rp, col = gen.circuit_like()
    beg, end = gen.csr_to_beg_end(rp)
    m = ctx.load_rowptr(rp, col)
    res = ctx.factor(m, max_supernode_size=128)
    rc = res.row_counts()
    dg = res.digests()
    rng = np.random.default_rng(5)
    rows = np.unique(np.concatenate([rng.choice(n, 24, replace=False),
                                     [0, n - 1]])).astype(np.int32)
    rr = O.rows(beg, end, col, rows=rows)
    np.testing.assert_array_equal(rc["nnz_u_row"][rows], rr["nnzU"])
    np.testing.assert_array_equal(rc["nz_row_u"][rows], rr["nzU_ref"])
    np.testing.assert_array_equal(dg["dig_u_row"][rows], rr["digU"])
    tb, te, tc = O.transpose(beg, end, col)
    rt = O.rows(tb, te, tc, rows=rows)
    np.testing.assert_array_equal(rc["nnz_l_col"][rows], rt["nnzU"])
    np.testing.assert_array_equal(dg["dig_l_col"][rows], rt["digU"])
    c = res.counts
    assert c["nnz_u"] == int(rc["nnz_u_row"].sum())
    assert c["nnz_l"] == int(rc["nnz_l_col"].sum())
    assert c["fill_count"] == c["nnz_u"] + c["nnz_l"] - (int(rp[-1]) - n)
    res.close()
    m.close()


@pytest.fixture(scope="module")
def circuit_40k():
    from gsofatpds_b200 import gen
    n, rp, col = gen.circuit_like(n=40000, target_nnz=int(5830000 * 40000 / 659033), seed=9)
    beg, end = gen.csr_to_beg_end(rp)
    r = O.rows(beg, end, col)
    tb, te, tc = O.transpose(beg, end, col)
    rt = O.rows(tb, te, tc)
    return rp, col, r, rt


@pytest.mark.parametrize("tps,ring", [(128, 16), (256, 16), (512, 16), (1024, 32), (512, 4)])
def test_closure_reuse_repeatable(ctx, circuit_40k, tps, ring):
    """Every U row and L column of a 40k circuit-like matrix, several runs:
    the closure ring and its merges must never depend on thread timing."""
    rp, col, r, rt = circuit_40k
    m = ctx.load_rowptr(rp, col)
    for _ in range(3):
        res = ctx.factor(m, threads_per_source=tps, cached_closures=ring, chunk_sources=64)
        rc = res.row_counts()
        np.testing.assert_array_equal(rc["nnz_u_row"], r["nnzU"])
        np.testing.assert_array_equal(rc["nnz_l_col"], rt["nnzU"])
        np.testing.assert_array_equal(res.digests()["dig_u_row"], r["digU"])
        res.close()
    m.close()


def test_autotune_picks_valid_shapes_with_same_results(ctx):
    from gsofatpds_b200 import gen
    n, rp, col = gen.random_banded(6000, bw=5, extra=2, seed=5)
    m = ctx.load_rowptr(rp, col)
    tuned = ctx.autotune(m)
    assert tuned["threads_per_source"] in (128, 256, 512, 1024)
    assert tuned["chunk_sources"] > 0 and tuned["cached_closures"] in (1, 2, 4, 8, 16, 32, 64)
    assert ctx.autotune(m) == tuned  # cached for the size class
    a = ctx.factor(m, l_row_stats=True)
    b = ctx.factor(m, l_row_stats=True, **tuned)
    for x, y in zip(a.row_counts(True).values(), b.row_counts(True).values()):
        np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(a.supernodes()[0], b.supernodes()[0])
    assert a.counts["fill_count"] == b.counts["fill_count"]
    a.close()
    b.close()
    m.close()


def test_autotune_batch_shapes_give_the_same_results(ctx):
    from gsofatpds_b200 import gen
    mats_np = gen.batch_mix(12, nmin=1000, nmax=8000, seed=11)
    mats = [ctx.load_rowptr(rp, col) for (_, rp, col) in mats_np]
    tuned = ctx.autotune_batch(mats)
    assert tuned["threads_per_source"] in (128, 256, 512, 1024)
    assert tuned["cached_closures"] in (1, 2, 4, 8, 16, 32, 64)
    alone = [ctx.factor(m) for m in mats]
    batch = ctx.factor_batch(mats, **tuned)
    for a, b in zip(alone, batch):
        for x, y in zip(a.row_counts().values(), b.row_counts().values()):
            np.testing.assert_array_equal(x, y)
        np.testing.assert_array_equal(a.supernodes()[0], b.supernodes()[0])
        assert a.counts["fill_count"] == b.counts["fill_count"]
        a.close()
        b.close()
    for m in mats:
        m.close()


def test_batch_of_symmetric_matrices_repeated(ctx):
    """Every direction-1 item of a symmetric matrix is empty (the direction-0
    item fills both halves), so a batch of grids hands each CTA many items
    with no source loop in a row.  Each CTA must finish reading an item's
    descriptor before it takes the next one: repeated launches must all
    succeed with the alone results."""
    from gsofatpds_b200 import gen
    mats_np = [gen.grid_nd((s, s + 3), "5" if s % 2 else "9") for s in range(20, 60, 4)]
    mats_np += [gen.random_banded(3000, bw=6, extra=2, seed=5)]
    mats = [ctx.load_rowptr(rp, col) for (_, rp, col) in mats_np]
    ref = []
    for m in mats:
        r = ctx.factor(m)
        ref.append((r.counts["fill_count"], r.row_counts()["nnz_u_row"]))
        r.close()
    for rep in range(25):
        tps = (256, 512, 1024)[rep % 3]
        rs = ctx.factor_batch(mats, chunk_sources=16, threads_per_source=tps)
        for (fill, urow), r in zip(ref, rs):
            assert r.counts["fill_count"] == fill, rep
            np.testing.assert_array_equal(r.row_counts()["nnz_u_row"], urow)
            r.close()
    for m in mats:
        m.close()


def test_batch_equals_alone(ctx):
    from gsofatpds_b200 import gen
    mats_np = [gen.grid_nd((40, 37), "5"), gen.random_banded(2500, bw=5, extra=1, seed=2),
               gen.random_extra(900, 2, seed=4), gen.grid_nd((9, 8, 7), "27"),
               gen.random_banded(64, bw=4, extra=3, seed=9)]
    mats = [ctx.load_rowptr(rp, col) for (_, rp, col) in mats_np]
    batch = ctx.factor_batch(mats, l_row_stats=True)
    for m, rb in zip(mats, batch):
        ra = ctx.factor(m, l_row_stats=True)
        for a, b in zip(ra.row_counts(True).values(), rb.row_counts(True).values()):
            np.testing.assert_array_equal(a, b)
        for a, b in zip(ra.digests(True).values(), rb.digests(True).values()):
            np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(ra.supernodes()[0], rb.supernodes()[0])
        for k in ("fill_count", "nnz_l", "nnz_u", "edges_alg", "vertices_alg", "n_supernodes"):
            assert ra.counts[k] == rb.counts[k], k
        ra.close()
        rb.close()
    for m in mats:
        m.close()


@pytest.mark.parametrize("mode", [0, 1, 3])
def test_graph_batch_equals_alone_twice(ctx, mode):
    """The graph-captured batch (one persistent launch for all matrices,
    batched supernode kernel) replayed twice gives each matrix's own result."""
    from gsofatpds_b200 import gen
    mats_np = [gen.grid_nd((31, 29), "5"), gen.random_banded(3000, bw=6, extra=2, seed=12),
               gen.random_extra(1500, 2, seed=8), gen.grid_nd((7, 6, 5), "7"),
               gen.random_banded(200, bw=4, extra=1, seed=3), gen.random_extra(1, 0, seed=1)]
    mats = [ctx.load_rowptr(rp, col) for (_, rp, col) in mats_np]
    kw = dict(l_row_stats=True, max_supernode_size=[128, 8, 256, 64][mode], **MODES[mode])
    alone = [ctx.factor(m, **kw) for m in mats]
    b = ctx.batch(mats, **kw)
    for _ in range(2):
        b.run()
        for i, ra in enumerate(alone):
            rb = b.result(i)
            for x, y in zip(ra.row_counts(True).values(), rb.row_counts(True).values()):
                np.testing.assert_array_equal(x, y)
            for x, y in zip(ra.digests(True).values(), rb.digests(True).values()):
                np.testing.assert_array_equal(x, y)
            np.testing.assert_array_equal(ra.supernodes()[0], rb.supernodes()[0])
            np.testing.assert_array_equal(ra.lmask(), rb.lmask())
            for k in ("fill_count", "nnz_l", "nnz_u", "edges_alg", "vertices_alg", "n_supernodes"):
                assert ra.counts[k] == rb.counts[k], k
    b.close()
    for r in alone:
        r.close()
    for m in mats:
        m.close()


def test_global_bitmap_variant_matches(ctx):
    """Orders whose bitmap exceeds shared memory keep it in global memory;
    force that variant on a small case and compare."""
    from gsofatpds_b200 import gen
    from gsofatpds_b200 import _lib as C
    import ctypes
    n, rp, col = gen.random_banded(5000, bw=8, extra=2, seed=21)
    m = ctx.load_rowptr(rp, col)
    a = ctx.factor(m, l_row_stats=True)
    o = ctx.opts(l_row_stats=True)
    o.flags |= C.FORCE_GLOBAL_BITMAP
    h = ctypes.c_void_p()
    ctx._check(ctx._L.gsofa_factor_symbolic(ctx.handle, m.handle, ctypes.byref(o), ctypes.byref(h)),
               "factor")
    from gsofatpds_b200.api import Result
    b = Result(ctx, h)
    for x, y in zip(a.row_counts(True).values(), b.row_counts(True).values()):
        np.testing.assert_array_equal(x, y)
    for x, y in zip(a.digests(True).values(), b.digests(True).values()):
        np.testing.assert_array_equal(x, y)
    assert a.counts["fill_count"] == b.counts["fill_count"]
    a.close()
    b.close()
    m.close()


def test_errors_are_status_codes(ctx):
    from gsofatpds_b200 import Context, GsofaError
    from gsofatpds_b200 import _lib as C
    with pytest.raises(GsofaError) as e:
        ctx.load_csr(np.array([0, 1], np.int32), np.array([1, 2], np.int32),
                     np.array([0, 7], np.int32))  # column 7 outside [0, 2)
    assert e.value.status == C.ERR_ARG
    with pytest.raises(GsofaError) as e:
        ctx.load_csr(np.array([0, 1], np.int32), np.array([1, 9], np.int32),
                     np.array([0, 1], np.int32))  # row end past nnz
    assert e.value.status == C.ERR_ARG
    m = ctx.load_csr(np.array([0, 1], np.int32), np.array([1, 2], np.int32),
                     np.array([0, 1], np.int32))
    with pytest.raises(GsofaError) as e:
        ctx.factor(m, max_supernode_size=0)
    assert e.value.status == C.ERR_ARG
    with pytest.raises(GsofaError) as e:
        ctx.factor(m, threads_per_source=100)
    assert e.value.status == C.ERR_ARG
    m.close()
    small = Context(0, budget_bytes=1 << 16)
    with pytest.raises(GsofaError) as e:
        small.load_rowptr(*__import__("gsofatpds_b200").gen.random_extra(20000)[1:])
    assert e.value.status == C.ERR_OOM_BUDGET
    small.close()
    # the context stays usable after errors
    m = ctx.load_csr(np.array([0], np.int32), np.array([1], np.int32), np.array([0], np.int32))
    r = ctx.factor(m)
    assert r.counts["fill_count"] == 0
    r.close()
    m.close()


def test_reference_entry_point_and_cli(ctx, tmp_path):
    from gsofatpds_b200 import _lib as C
    from gsofatpds_b200 import gen, symbfact_min_id
    z = load_bc()
    n = z["beg"].shape[0]
    pb, pe, pc = (str(tmp_path / ("%s_%d.dat" % (k, n))) for k in ("colbeg", "colend", "csr"))
    with open(pc, "w") as f:
        f.write("%d\n%d\n%s\n" % (z["col"].shape[0], n, " ".join(map(str, z["col"].tolist()))))
    with open(pb, "w") as f:
        f.write(" ".join(map(str, z["beg"].tolist())))
    with open(pe, "w") as f:
        f.write(" ".join(map(str, z["end"].tolist())))
    # SOA layout (gSoFa_SOAComparison/Makefile:37)
    fills, ms, nsup, edges = symbfact_min_id(["exe", pb, pe, pc, "1", "128", "0", "0", "1", "4", "4096"])
    assert fills == 980136 and nsup == 6800 and ms > 0 and edges > 0
    # SPO layout (SpaceOptimization/Makefile:33)
    fills, ms, nsup, edges = symbfact_min_id(["exe", pb, pe, pc, "264", "5"])
    assert fills == 980136
    out = subprocess.run([C.CLI_PATH, pb, pe, pc, "1", "128", "0", "0", "1", "4", "4096"],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert "Final Number of fill-ins detected: 980136" in out.stdout
    assert "Final Number of Supernodes detected: 6800" in out.stdout
    # the generator's ASCII writer round-trips through the library's reader
    n2, rp, col = gen.random_extra(500, 2, seed=3)
    paths = gen.write_dat(str(tmp_path / "x_"), n2, rp, col)
    m = ctx.load_files(*paths)
    r = ctx.factor(m)
    b, e = gen.csr_to_beg_end(rp)
    assert r.counts["fill_count"] == int(O.rows(b, e, col)["fills"].sum())
    r.close()
    m.close()


def test_symmetric_pattern_shortcut(ctx):
    """A symmetric pattern runs only the U-row searches (the L columns repeat
    them); one extra unmatched entry turns the shortcut off.  Both must equal
    the oracle, and the symmetric run inspects about half the entries."""
    from gsofatpds_b200 import gen
    _, rp, col = gen.grid_nd((14, 14, 14), "7")
    n = rp.shape[0] - 1
    beg, end = rp[:-1].copy(), rp[1:].copy()
    # asymmetric twin: one more entry (v, w) without (w, v)
    v, w = 5, n - 3
    col2 = np.concatenate([col[:end[v]], [w], col[end[v]:]]).astype(np.int32)
    beg2, end2 = beg.copy(), end.copy()
    end2[v] += 1
    beg2[v + 1:] += 1
    end2[v + 1:] += 1
    out = []
    for b, e, c in [(beg, end, col), (beg2, end2, col2)]:
        r, rt = oracle_full(b, e, c)
        m = ctx.load_csr(b, e, c)
        res = ctx.factor(m, l_row_stats=True)
        check_full(res, r, rt)
        out.append(res.counts["edges_traversed"])
        res.close()
        m.close()
    assert out[0] * 1.5 < out[1], out
    # duplicated entries and unsorted rows keep a symmetric pattern symmetric
    rng = np.random.default_rng(7)
    pat = random_pattern(rng, 60, 0.08, diag=True)
    pat = [set(p) | {j for j in range(60) if i in pat[j]} for i, p in enumerate(pat)]
    b, e, c = scrambled_csr(rng, pat, dup_prob=0.3)
    r, rt = oracle_full(b, e, c)
    m = ctx.load_csr(b, e, c)
    res = ctx.factor(m, l_row_stats=True)
    check_full(res, r, rt)
    res.close()
    m.close()


def _supernodal_reference(n, r, flags):
    """The supernodal block form from the oracle's own patterns: L rows
    (transposed to columns) and U rows, blocks from the oracle's flags."""
    starts = [int(x) for x in np.nonzero(flags)[0]] + [n]
    lcols = [[] for _ in range(n)]
    for s in range(n):
        for c in r["Lcols"][r["Lptr"][s]:r["Lptr"][s + 1]]:
            lcols[int(c)].append(s)
    out = dict(block_start=np.array(starts, np.int32), lptr=[0], lrows=[], uptr=[0], ucols=[])
    for k in range(len(starts) - 1):
        f, l = starts[k], starts[k + 1]
        rows, cols = set(), set()
        for c in range(f, l):
            rows.update(x for x in lcols[c] if x >= l)
            cols.update(int(x) for x in r["Ucols"][r["Uptr"][c]:r["Uptr"][c + 1]] if x >= l)
        out["lrows"] += sorted(rows)
        out["ucols"] += sorted(cols)
        out["lptr"].append(len(out["lrows"]))
        out["uptr"].append(len(out["ucols"]))
    return out


@pytest.mark.parametrize("which", ["bc", "grid", "random"])
def test_supernodal_handoff_matches_oracle(ctx, which):
    """gsofa_result_supernodal against a restatement from the oracle's
    patterns and supernode partition."""
    from gsofatpds_b200 import gen
    if which == "bc":
        z = load_bc()
        beg, end, col = z["beg"], z["end"], z["col"]
    elif which == "grid":
        _, rp, col = gen.grid_nd((12, 12, 12), "7")
        beg, end = rp[:-1], rp[1:]
    else:
        _, rp, col = gen.random_banded(3000, bw=6, extra=2, seed=9)
        beg, end = rp[:-1], rp[1:]
    n = beg.shape[0]
    r = O.rows(beg, end, col, pattern=True)
    nsup, flags = O.supernodes(r["nzU_ref"], r["lback"], 128)
    ref = _supernodal_reference(n, r, flags)
    m = ctx.load_csr(beg, end, col)
    res = ctx.factor(m, pattern=True)
    got = res.supernodal()
    np.testing.assert_array_equal(got["block_start"], ref["block_start"])
    for k in ("lptr", "lrows", "uptr", "ucols"):
        np.testing.assert_array_equal(got[k], np.array(ref[k]), err_msg=k)
    assert res.supernodal()["lrows"].shape == got["lrows"].shape  # cached, same answer
    res.close()
    m.close()


def test_forced_queue_overflow_is_an_error_and_the_context_survives(ctx):
    """Fault injection (GSOFA_DEBUG_QUEUE_CAP): 64-entry frontier queues make
    BC's long searches overflow; the bounds-checked queue turns that into
    GSOFA_ERR_OVERFLOW, and the next plain factorization is exact."""
    from gsofatpds_b200 import GsofaError
    from gsofatpds_b200 import _lib as C
    z = load_bc()
    m = ctx.load_csr(z["beg"], z["end"], z["col"])
    with pytest.raises(GsofaError) as e:
        ctx.factor(m, debug_queue_cap=True)
    assert e.value.status == C.ERR_OVERFLOW
    r = ctx.factor(m)
    assert r.counts["fill_count"] == 980136
    np.testing.assert_array_equal(r.row_counts()["nnz_u_row"], z["nnzU"])
    r.close()
    m.close()
