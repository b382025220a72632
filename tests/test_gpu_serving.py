"""Serving request loop (gsofa_server_*) against plain factorization.

Every served request must give exactly the result of factoring the same
matrix alone with gsofa_factor_symbolic (all quantities are integers):
totals, per-row counts, digests, L masks and the supernode partition.  The
mix is built so that requests overlap on the device: small requests are
submitted while a large one runs, and at least one of them must finish
before the large one does (a loop that served requests one at a time could
not do that).
"""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _mix():
    from gsofatpds_b200 import gen
    from tests.helpers import load_bc
    z = load_bc()
    reqs = []
    # one large request first: a 3D 27-point grid in nested-dissection order
    reqs.append(("grid3d_27_56", gen.grid_nd((56, 56, 56), "27")[1:]))
    reqs.append(("random_extra_20k", gen.random_extra(20000, 3, seed=1)[1:]))
    for i, side in enumerate([30, 64, 100, 150]):
        reqs.append(("grid2d_%d" % side, gen.grid_nd((side, side), "5" if i % 2 else "9")[1:]))
    for i, n in enumerate([1500, 4000, 9000, 25000]):
        reqs.append(("banded_%d" % n, gen.random_banded(n, bw=4 + 6 * i, extra=1 + i, seed=10 + i)[1:]))
    reqs.append(("grid3d_7_20", gen.grid_nd((20, 20, 20), "7")[1:]))
    reqs.append(("bc", (z["beg"], z["end"], z["col"])))
    return reqs


def _alone(ctx, spec, **kw):
    if len(spec) == 3:
        m = ctx.load_csr(*spec)
    else:
        m = ctx.load_rowptr(*spec)
    r = ctx.factor(m, **kw)
    out = dict(counts=r.counts, rows=r.row_counts(l_rows="l_row_stats" in kw), dig=r.digests(),
               lmask=r.lmask(), flags=r.supernodes()[0])
    r.close()
    m.close()
    return out


def _submit(srv, spec):
    if len(spec) == 3:
        return srv.submit(*spec)
    return srv.submit_rowptr(*spec)


def _same(name, got, ref):
    keys = ["fill_count", "nnz_l", "nnz_u", "nnz_lu", "n_supernodes", "edges_alg", "vertices_alg"]
    for k in keys:
        assert got.counts[k] == ref["counts"][k], (name, k, got.counts[k], ref["counts"][k])
    rc = got.row_counts(l_rows="nnz_l_row" in ref["rows"])
    for k, v in ref["rows"].items():
        np.testing.assert_array_equal(rc[k], v, err_msg="%s %s" % (name, k))
    dg = got.digests()
    for k, v in ref["dig"].items():
        np.testing.assert_array_equal(dg[k], v, err_msg="%s %s" % (name, k))
    np.testing.assert_array_equal(got.lmask(), ref["lmask"], err_msg=name + " lmask")
    np.testing.assert_array_equal(got.supernodes()[0], ref["flags"], err_msg=name + " flags")


@pytest.mark.parametrize("block", [256, 1024])
def test_served_results_equal_alone_and_overlap(block):
    _cuda()
    from gsofatpds_b200 import Context
    reqs = _mix()
    with Context(0) as ctx:
        refs = [_alone(ctx, spec) for _, spec in reqs]
        with ctx.server(max_n=200000, threads_per_source=block) as srv:
            tickets = [_submit(srv, reqs[0][1])]
            time.sleep(0.005)  # the large request is on the device now
            for _, spec in reqs[1:]:
                tickets.append(_submit(srv, spec))
                time.sleep(0.0005)
            got = [srv.wait(t, 120000) for t in tickets]
            info = [srv.info(t) for t in tickets]
            st = srv.stats()
        for (name, _), g, ref in zip(reqs, got, refs):
            assert g is not None, name
            _same(name, g, ref)
            g.close()
        assert refs[-1]["counts"]["fill_count"] == 980136
    big = info[0]
    overtook = [i for i in info[1:] if i["t_done_ms"] < big["t_done_ms"]]
    assert overtook, "no request finished while the large one ran"
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["max_in_flight"] >= 2


def test_served_global_bitmaps_and_l_rows():
    """Every bitmap in global memory (diagnostic flag), per-row L scatter on."""
    _cuda()
    from gsofatpds_b200 import Context
    reqs = _mix()[1:8]
    with Context(0) as ctx:
        refs = [_alone(ctx, spec, l_row_stats=True) for _, spec in reqs]
        with ctx.server(max_n=100000, l_row_stats=True, global_bitmap=True) as srv:
            tickets = [_submit(srv, spec) for _, spec in reqs]
            got = [srv.wait(t, 120000) for t in tickets]
        for (name, _), g, ref in zip(reqs, got, refs):
            _same(name, g, ref)
            g.close()


def test_served_errors_and_limits():
    _cuda()
    from gsofatpds_b200 import Context, GsofaError, gen
    from gsofatpds_b200 import _lib as C
    _, rp, col = gen.random_extra(3000, 2, seed=5)
    with Context(0) as ctx:
        ref = _alone(ctx, (rp, col))
        with ctx.server(max_n=5000) as srv:
            # column id outside [0, n): found by the device build, fails alone
            bad = col.copy()
            bad[7] = 999999
            t_bad = srv.submit_rowptr(rp, bad)
            # row interval outside the column array: found on the host
            beg = rp[:-1].copy()
            end = rp[1:].copy()
            end[3] = len(col) + 10
            t_rows = srv.submit(beg, end, col)
            t_ok = srv.submit_rowptr(rp, col)
            with pytest.raises(GsofaError) as e1:
                srv.wait(t_bad, 60000)
            assert e1.value.status == C.ERR_ARG
            with pytest.raises(GsofaError) as e2:
                srv.wait(t_rows, 60000)
            assert e2.value.status == C.ERR_ARG
            g = srv.wait(t_ok, 60000)
            _same("after errors", g, ref)
            g.close()
            # a result is handed out once
            with pytest.raises(GsofaError):
                srv.poll(t_ok)
            # larger than max_n
            _, rp2, col2 = gen.random_extra(6000, 2, seed=5)
            with pytest.raises(GsofaError) as e3:
                srv.submit_rowptr(rp2, col2)
            assert e3.value.status == C.ERR_UNSUPPORTED
            st = srv.stats()
            assert st["failed"] == 2 and st["completed"] == 1
        # a budget too small for the request (but not for the workspace)
        with ctx.server(max_n=5000, budget_bytes=64 << 20) as srv:
            _, rp3, col3 = gen.random_banded(5000, bw=60, extra=4, seed=1)
            big = np.repeat(col3, 40)  # duplicated columns inflate nnz, not n
            rpb = rp3 * 40
            with pytest.raises(GsofaError) as e4:
                srv.submit_rowptr(rpb, big)
            assert e4.value.status == C.ERR_OOM_BUDGET


def test_served_idle_restart():
    """The kernel exits when the loop is idle and is relaunched on demand."""
    _cuda()
    from gsofatpds_b200 import Context, gen
    _, rp, col = gen.random_banded(8000, bw=10, extra=2, seed=2)
    with Context(0) as ctx:
        ref = _alone(ctx, (rp, col))
        with ctx.server(max_n=10000) as srv:
            for _ in range(3):
                t = srv.submit_rowptr(rp, col)
                g = srv.wait(t, 60000)
                _same("restart", g, ref)
                g.close()
                time.sleep(0.05)
            assert srv.stats()["kernel_launches"] >= 2
