"""The no-allocation entry point (gsofa_factor_symbolic_noalloc) against the
regular one.

It serves callers that cannot call cudaMalloc while factoring (a host
framework that owns all device memory, or a loop that must not allocate after
set-up): the matrix is loaded beforehand, the outputs are caller-owned device
buffers, and the kernel's scratch lives in the library's static device array.
Here torch plays the caller that owns the output buffers.  Two calls in a row
must both reproduce the regular entry point's results exactly (every quantity
is an integer), since each call reuses the static array left by the last.

The file name sorts last so that a run stopping at its first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(ctx, mat, opts, n, torch, expect=None):
    """One call with fresh caller-owned output buffers; returns the outputs
    (or, with `expect`, checks that the call returns that status and
    returns None)."""
    from gsofatpds_b200 import _lib as C
    dev = torch.device("cuda", ctx.device)
    out = dict(nnz_u_row=torch.full((n,), -1, dtype=torch.int32, device=dev),
               nz_row_u=torch.full((n,), -1, dtype=torch.int32, device=dev),
               nnz_l_col=torch.full((n,), -1, dtype=torch.int32, device=dev),
               lmask=torch.full((n, 4), 7, dtype=torch.int32, device=dev),
               flags=torch.full((n,), 9, dtype=torch.int8, device=dev),
               counters=torch.full((8,), 5, dtype=torch.int64, device=dev))
    torch.cuda.synchronize()
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    rc = C.load().gsofa_factor_symbolic_noalloc(
        mat.handle, ctypes.byref(opts), None, p(out["nnz_u_row"]), p(out["nz_row_u"]),
        p(out["nnz_l_col"]), p(out["lmask"]), p(out["flags"]), p(out["counters"]))
    if expect is not None:
        assert rc == expect, C.load().gsofa_status_string(rc)
        return None
    assert rc == C.OK, C.load().gsofa_status_string(rc)
    return {k: v.cpu().numpy() for k, v in out.items()}


def _check_against(got, ref, call):
    rc, lm, fl, c = ref
    np.testing.assert_array_equal(got["nnz_u_row"], rc["nnz_u_row"], err_msg="call %d" % call)
    np.testing.assert_array_equal(got["nz_row_u"], rc["nz_row_u"], err_msg="call %d" % call)
    np.testing.assert_array_equal(got["nnz_l_col"], rc["nnz_l_col"], err_msg="call %d" % call)
    np.testing.assert_array_equal(got["lmask"].view(np.uint32), lm, err_msg="call %d" % call)
    np.testing.assert_array_equal(got["flags"], fl, err_msg="call %d" % call)
    k = got["counters"].view(np.uint64)
    assert int(k[0]) == c["fill_count"]
    assert int(k[1]) == c["edges_alg"] and int(k[2]) == c["vertices_alg"]
    assert int(k[4]) + 1 == c["n_supernodes"]
    assert int(k[5]) == c["nnz_u"] and int(k[6]) == c["nnz_l"]


def _regular(ctx, m, **kw):
    ref = ctx.factor(m, max_supernode_size=128, **kw)
    out = (ref.row_counts(), ref.lmask(), ref.supernodes()[0], ref.counts)
    ref.close()
    return out


@pytest.mark.parametrize("which", ["bc", "random_extra", "circuit_40k"])
def test_noalloc_matches_regular_entry_twice(which):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gsofatpds_b200 import Context, gen
    from tests.helpers import load_bc
    with Context(0) as ctx:
        if which == "bc":
            z = load_bc()
            m = ctx.load_csr(z["beg"], z["end"], z["col"])
        elif which == "random_extra":
            _, rp, col = gen.random_extra(20000, 3, seed=1)
            m = ctx.load_rowptr(rp, col)
        else:
            _, rp, col = gen.circuit_like(n=40000, target_nnz=int(5830000 * 40000 / 659033), seed=9)
            m = ctx.load_rowptr(rp, col)
        n = m.n
        ref = _regular(ctx, m)
        opts = ctx.opts(max_supernode_size=128, digests=False)
        for call in range(2):
            _check_against(_noalloc(ctx, m, opts, n, torch), ref, call)
        if which == "bc":
            assert ref[3]["fill_count"] == 980136
        m.close()


def test_noalloc_rejects_what_it_cannot_do():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gsofatpds_b200 import Context, gen
    from gsofatpds_b200 import _lib as C
    with Context(0) as ctx:
        _, rp, col = gen.random_extra(500, 2, seed=3)
        m = ctx.load_rowptr(rp, col)
        buf = torch.zeros(4096, dtype=torch.int64, device="cuda")
        p = ctypes.c_void_p(buf.data_ptr())
        L = C.load()
        # per-row L statistics need result storage the entry point does not have
        o = ctx.opts(l_row_stats=True)
        assert L.gsofa_factor_symbolic_noalloc(m.handle, ctypes.byref(o), None, p, p, p, p, p,
                                               p) == C.ERR_UNSUPPORTED
        # missing output buffer
        o = ctx.opts()
        assert L.gsofa_factor_symbolic_noalloc(m.handle, ctypes.byref(o), None, None, p, p, p, p,
                                               p) == C.ERR_ARG
        m.close()


def test_noalloc_variants_and_a_shrunken_grid():
    """The same answers from the global-bitmap layout, and on a 600,625-row
    grid where the fixed array holds only a few tens of CTAs' queues and
    rings (the grid shrinks to fit); each twice in a row."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gsofatpds_b200 import Context, gen
    from gsofatpds_b200 import _lib as C
    with Context(0) as ctx:
        _, rp, col = gen.random_banded(5000, bw=8, extra=2, seed=21)
        m = ctx.load_rowptr(rp, col)
        ref = _regular(ctx, m)
        o = ctx.opts(max_supernode_size=128, digests=False)
        o.flags |= C.FORCE_GLOBAL_BITMAP
        for call in range(2):
            _check_against(_noalloc(ctx, m, o, m.n, torch), ref, call)
        m.close()
        n, rp, col = gen.grid_nd((775, 775), "5")
        m = ctx.load_rowptr(rp, col)
        ref = _regular(ctx, m)
        o = ctx.opts(max_supernode_size=128, digests=False)
        for call in range(2):
            _check_against(_noalloc(ctx, m, o, n, torch), ref, call)
        m.close()


def test_noalloc_errors_leave_the_library_usable():
    """A forced 64-entry queue overflows (GSOFA_ERR_OVERFLOW, nothing written
    out of bounds) and a matrix whose one CTA does not fit the fixed array is
    GSOFA_ERR_SCRATCH; the next regular call gives the exact answer."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gsofatpds_b200 import Context
    from gsofatpds_b200 import _lib as C
    from tests.helpers import load_bc
    with Context(0) as ctx:
        z = load_bc()
        m = ctx.load_csr(z["beg"], z["end"], z["col"])
        o = ctx.opts(max_supernode_size=128, digests=False, debug_queue_cap=True)
        _noalloc(ctx, m, o, m.n, torch, expect=C.ERR_OVERFLOW)
        # 6M rows with a 64-deep ring: 24 MB of queue + 48 MB of ring per CTA
        big = 6000000
        mb = ctx.load_rowptr(np.arange(big + 1, dtype=np.int32), np.arange(big, dtype=np.int32))
        o = ctx.opts(max_supernode_size=128, digests=False, cached_closures=64)
        _noalloc(ctx, mb, o, big, torch, expect=C.ERR_SCRATCH)
        mb.close()
        ref = _regular(ctx, m)
        assert ref[3]["fill_count"] == 980136
        o = ctx.opts(max_supernode_size=128, digests=False)
        _check_against(_noalloc(ctx, m, o, m.n, torch), ref, 0)
        m.close()
