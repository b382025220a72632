"""Python host interface over the C-ABI (include/gsofa.h).

Mirrors the reference's interface for the symbolic-factorization path:
``symbfact_min_id(argv)`` takes the same argument vectors as the reference's
``symbfact_min_id(argc, argv, rank, fill_count, time, N_supernodes, TEPS)``
(gSoFa_SOAComparison/symbfact_warp_centric_new_scheduling.cuh:2529,
SpaceOptimization/symbfact.cuh:1553) and returns the same four outputs, while
``Context`` / ``Matrix`` / ``Result`` expose the handle-based calls for
callers that keep matrices device-resident.  Errors raise ``GsofaError``
carrying the library's status code; nothing here falls back to the CPU.
"""
import ctypes
import os

import numpy as np

from . import _lib as C

__all__ = ["GsofaError", "Context", "Matrix", "Result", "Batch", "Server", "symbfact_min_id",
           "write_binary", "read_binary", "convert_dat"]


class GsofaError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("%s (status %d)" % (message, status))
        self.status = status


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class Context:
    """One device context (memory budget, stream, workspace)."""

    def __init__(self, device=0, budget_bytes=0):
        self._L = C.load()
        h = ctypes.c_void_p()
        rc = self._L.gsofa_create(int(device), int(budget_bytes), ctypes.byref(h))
        if rc != C.OK:
            raise GsofaError(rc, "gsofa_create failed: %s" % self._L.gsofa_status_string(rc).decode())
        self._h = h
        self.device = device

    def _check(self, rc, what):
        if rc != C.OK:
            msg = self._L.gsofa_last_error(self._h).decode(errors="replace")
            raise GsofaError(rc, "%s: %s" % (what, msg))

    @property
    def handle(self):
        """The gsofa_ctx* handle (for calls through gsofatpds_b200._lib)."""
        return self._h

    def set_stream(self, stream_ptr):
        """Launch on this CUDA stream (an int cudaStream_t, e.g.
        torch.cuda.current_stream().cuda_stream); None = own stream."""
        self._check(self._L.gsofa_set_stream(self._h, ctypes.c_void_p(stream_ptr or 0)), "set_stream")

    def memory_used(self):
        """Device bytes the context holds now (matrices, results, workspace)."""
        v = ctypes.c_size_t()
        self._check(self._L.gsofa_memory_used(self._h, ctypes.byref(v)), "memory_used")
        return v.value

    def load_csr(self, row_begin, row_end, col):
        """Host arrays -> device-resident matrix.  Rows may be unsorted and
        non-contiguous (row v is col[row_begin[v]:row_end[v]])."""
        b = np.ascontiguousarray(row_begin, dtype=np.int32)
        e = np.ascontiguousarray(row_end, dtype=np.int32)
        c = np.ascontiguousarray(col, dtype=np.int32)
        if b.shape != e.shape:
            raise GsofaError(C.ERR_ARG, "row_begin and row_end differ in length")
        h = ctypes.c_void_p()
        self._check(self._L.gsofa_load_csr(self._h, b.shape[0], c.shape[0], _ptr(b), _ptr(e),
                                           _ptr(c), ctypes.byref(h)), "load_csr")
        return Matrix(self, h)

    def load_rowptr(self, rowptr, col):
        """load_csr for contiguous rows: row v is col[rowptr[v]:rowptr[v+1]]."""
        rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
        return self.load_csr(rowptr[:-1], rowptr[1:], col)

    def load_binary(self, path):
        """A matrix from a binary CSR file (see write_binary)."""
        h = ctypes.c_void_p()
        self._check(self._L.gsofa_load_csr_binary(self._h, os.fsencode(path), ctypes.byref(h)),
                    "load_csr_binary")
        return Matrix(self, h)

    def load_files(self, beg_file, end_file, csr_file):
        """The reference's three ASCII files (colbeg, colend, csr) -> matrix."""
        h = ctypes.c_void_p()
        self._check(self._L.gsofa_load_csr_files(self._h, beg_file.encode(), end_file.encode(),
                                                 csr_file.encode(), ctypes.byref(h)), "load_files")
        return Matrix(self, h)

    @staticmethod
    def opts(max_supernode_size=128, threads_per_source=0, sources_in_flight=0,
             supernodes=True, digests=True, l_row_stats=False, pattern=False,
             bu_alpha=0, bu_beta=0, heavy_row=0, bu_min_source=0, chunk_sources=0,
             merge=True, cached_closures=0, global_bitmap=False, debug_queue_cap=False,
             chain=True, chain_wait_us=0):
        """A gsofa_opts from keyword arguments (0 = library default); the
        launch-shape options change speed only, never results."""
        o = C.Opts()
        o.cached_closures = int(cached_closures)
        o.chain_wait_us = int(chain_wait_us)
        o.chunk_sources = int(chunk_sources)
        o.bu_min_source = int(bu_min_source)
        o.bu_alpha = int(bu_alpha)
        o.bu_beta = int(bu_beta)
        o.heavy_row = int(heavy_row)
        o.max_supernode_size = int(max_supernode_size)
        o.threads_per_source = int(threads_per_source)
        o.sources_in_flight = int(sources_in_flight)
        o.flags = ((C.SUPERNODES if supernodes else 0) | (C.DIGESTS if digests else 0) |
                   (C.L_ROW_STATS if l_row_stats else 0) | (C.PATTERN if pattern else 0) |
                   (0 if merge else C.NO_MERGE) | (C.FORCE_GLOBAL_BITMAP if global_bitmap else 0) |
                   (C.DEBUG_QUEUE_CAP if debug_queue_cap else 0) | (0 if chain else C.NO_CHAIN))
        return o

    def autotune(self, mat, **kw):
        """Fastest (threads_per_source, chunk_sources, cached_closures) for
        `mat`, measured on the device; returns them as keyword arguments."""
        o = self.opts(**kw)
        self._check(self._L.gsofa_autotune(self._h, mat.handle, ctypes.byref(o)), "autotune")
        return dict(threads_per_source=o.threads_per_source, chunk_sources=o.chunk_sources,
                    cached_closures=o.cached_closures, heavy_row=o.heavy_row)

    def autotune_batch(self, mats, **kw):
        """Fastest launch shape for one persistent launch over all `mats`."""
        o = self.opts(**kw)
        k = len(mats)
        arr = (ctypes.c_void_p * max(k, 1))(*[m.handle for m in mats])
        self._check(self._L.gsofa_autotune_batch(self._h, arr, k, ctypes.byref(o)), "autotune_batch")
        return dict(threads_per_source=o.threads_per_source, chunk_sources=o.chunk_sources,
                    cached_closures=o.cached_closures, heavy_row=o.heavy_row)

    def order_nd(self, mat, leaf_size=0, max_rounds=0):
        """Fill-reducing ordering of A + A^T by level-set nested dissection,
        computed on the device.  Returns (perm, stats): new index k holds
        old index perm[k]."""
        n = mat.n
        perm = np.zeros(max(n, 1), np.int32)
        st = C.OrderStats()
        self._check(self._L.gsofa_order_nd(self._h, mat.handle, int(leaf_size), int(max_rounds),
                                           _ptr(perm), ctypes.byref(st)), "order_nd")
        stats = {f: getattr(st, f) for f, _ in C.OrderStats._fields_ if f != "reserved"}
        return perm[:n], stats

    def order_hybrid(self, mat, leaf_size=0):
        """Fill-reducing ordering of A + A^T by hybrid nested dissection
        (level-set and multilevel separators, the smaller kept at each
        split), computed on the device.  Returns (perm, stats) as order_nd."""
        n = mat.n
        perm = np.zeros(max(n, 1), np.int32)
        st = C.OrderStats()
        self._check(self._L.gsofa_order_hybrid(self._h, mat.handle, int(leaf_size), _ptr(perm),
                                               ctypes.byref(st)), "order_hybrid")
        stats = {f: getattr(st, f) for f, _ in C.OrderStats._fields_ if f != "reserved"}
        return perm[:n], stats

    def permute(self, mat, perm):
        """P A P^T on the device: row k is row perm[k] of `mat`, columns renamed."""
        p = np.ascontiguousarray(perm, dtype=np.int32)
        if p.shape[0] != mat.n:
            raise GsofaError(C.ERR_ARG, "perm has %d entries, the matrix %d rows" %
                             (p.shape[0], mat.n))
        h = ctypes.c_void_p()
        self._check(self._L.gsofa_matrix_permute(self._h, mat.handle, _ptr(p), ctypes.byref(h)),
                    "matrix_permute")
        return Matrix(self, h)

    def factor(self, mat, **kw):
        """gsofa_factor_symbolic: the fill structure of `mat` (a Result);
        keyword arguments as for opts()."""
        o = self.opts(**kw)
        h = ctypes.c_void_p()
        self._check(self._L.gsofa_factor_symbolic(self._h, mat.handle, ctypes.byref(o),
                                                  ctypes.byref(h)), "factor_symbolic")
        return Result(self, h)

    def batch(self, mats, **kw):
        """Prepared graph-captured batch (see Batch)."""
        return Batch(self, mats, **kw)

    def server(self, max_n, budget_bytes=0, **kw):
        """Serving request loop (see Server)."""
        return Server(self, max_n, budget_bytes, **kw)

    def factor_batch(self, mats, **kw):
        """All `mats` in one persistent launch; one Result per matrix."""
        o = self.opts(**kw)
        k = len(mats)
        arr = (ctypes.c_void_p * max(k, 1))(*[m.handle for m in mats])
        outs = (ctypes.c_void_p * max(k, 1))()
        self._check(self._L.gsofa_factor_batch(self._h, arr, k, ctypes.byref(o), outs),
                    "factor_batch")
        return [Result(self, ctypes.c_void_p(outs[i])) for i in range(k)]

    def close(self):
        """Releases the context and everything it holds on the device."""
        if getattr(self, "_h", None):
            self._L.gsofa_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Batch:
    """Many matrices in one persistent launch captured in a CUDA graph;
    run() replays it.  Results are owned by the batch."""

    def __init__(self, ctx, mats, **kw):
        self.ctx = ctx
        self.mats = list(mats)  # keep the matrices alive while the batch lives
        o = ctx.opts(**kw)
        k = len(self.mats)
        arr = (ctypes.c_void_p * max(k, 1))(*[m.handle for m in self.mats])
        h = ctypes.c_void_p()
        ctx._check(ctx._L.gsofa_batch_create(ctx.handle, arr, k, ctypes.byref(o), ctypes.byref(h)),
                   "batch_create")
        self._h = h

    def run(self):
        """Replays the captured launch; results are refreshed in place."""
        self.ctx._check(self.ctx._L.gsofa_batch_run(self._h), "batch_run")
        return self

    def result(self, i):
        """The i-th matrix's Result (owned by the batch)."""
        h = ctypes.c_void_p()
        self.ctx._check(self.ctx._L.gsofa_batch_result(self._h, int(i), ctypes.byref(h)), "batch_result")
        return Result(self.ctx, h, owned=False)

    def close(self):
        if getattr(self, "_h", None):
            self.ctx._L.gsofa_batch_destroy(self._h)
            self._h = None


class Server:
    """Continuous-batching request loop: submit() queues a host CSR matrix and
    returns a ticket; wait()/poll() hand out its Result.  The submitted
    arrays are kept referenced here until their ticket completes (the library
    reads them when it admits the request)."""

    def __init__(self, ctx, max_n, budget_bytes=0, **kw):
        self.ctx = ctx
        self._L = ctx._L
        o = ctx.opts(**kw)
        h = ctypes.c_void_p()
        ctx._check(self._L.gsofa_server_create(ctx.handle, ctypes.byref(o), int(max_n),
                                               int(budget_bytes), ctypes.byref(h)), "server_create")
        self._h = h
        self._held = {}

    def _raise(self, rc, what):
        msg = self._L.gsofa_server_last_error(self._h).decode(errors="replace")
        raise GsofaError(rc, "%s: %s" % (what, msg or self._L.gsofa_status_string(rc).decode()))

    def submit(self, row_begin, row_end, col):
        """Queue one request (rows col[row_begin[v]:row_end[v]]); returns its ticket."""
        beg = np.ascontiguousarray(row_begin, dtype=np.int32)
        end = np.ascontiguousarray(row_end, dtype=np.int32)
        c = np.ascontiguousarray(col, dtype=np.int32)
        t = ctypes.c_uint64()
        rc = self._L.gsofa_server_submit(self._h, beg.shape[0], c.shape[0], _ptr(beg), _ptr(end),
                                         _ptr(c), ctypes.byref(t))
        if rc != C.OK:
            self._raise(rc, "server_submit")
        self._held[t.value] = (beg, end, c)
        return t.value

    def submit_rowptr(self, rowptr, col):
        """submit() for contiguous rows (rowptr of n+1 entries)."""
        rowptr = np.asarray(rowptr)
        return self.submit(rowptr[:-1], rowptr[1:], col)

    def _finish(self, ticket, rc, h):
        if rc == C.ERR_BUSY or rc == C.ERR_TIMEOUT:
            return None
        self._held.pop(ticket, None)
        if rc != C.OK:
            self._raise(rc, "ticket %d" % ticket)
        return Result(self.ctx, h)

    def poll(self, ticket):
        """The Result if the ticket is complete, else None."""
        h = ctypes.c_void_p()
        return self._finish(ticket, self._L.gsofa_server_poll(self._h, int(ticket), ctypes.byref(h)), h)

    def wait(self, ticket, timeout_ms=-1.0):
        """Blocks until the ticket completes (None on timeout)."""
        h = ctypes.c_void_p()
        rc = self._L.gsofa_server_wait(self._h, int(ticket), float(timeout_ms), ctypes.byref(h))
        return self._finish(ticket, rc, h)

    def info(self, ticket):
        """A ticket's times (submit, admit, publish, done; ms), footprint and status."""
        i = C.TicketInfo()
        rc = self._L.gsofa_server_ticket_info(self._h, int(ticket), ctypes.byref(i))
        if rc != C.OK:
            self._raise(rc, "ticket_info")
        return {f: getattr(i, f) for f, _ in C.TicketInfo._fields_}

    def stats(self):
        """The loop's counters: requests, launches, memory in use and peak."""
        st = C.ServerStats()
        rc = self._L.gsofa_server_get_stats(self._h, ctypes.byref(st))
        if rc != C.OK:
            self._raise(rc, "server_stats")
        return {f: getattr(st, f) for f, _ in C.ServerStats._fields_ if f != "reserved"}

    def close(self):
        if getattr(self, "_h", None):
            self._L.gsofa_server_destroy(self._h)
            self._h = None
            self._held.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Matrix:
    def __init__(self, ctx, h):
        self.ctx = ctx
        self._h = h
        n = ctypes.c_int32()
        nnz = ctypes.c_int64()
        ctx._check(ctx._L.gsofa_matrix_info(h, ctypes.byref(n), ctypes.byref(nnz)), "matrix_info")
        self.n = n.value
        self.nnz = nnz.value

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            self.ctx._L.gsofa_matrix_destroy(self._h)
            self._h = None


class Result:
    def __init__(self, ctx, h, owned=True):
        self.ctx = ctx
        self._h = h
        self._owned = owned
        c = C.Counts()
        ctx._check(ctx._L.gsofa_result_counts(h, ctypes.byref(c)), "result_counts")
        self.counts = {f: getattr(c, f) for f, _ in C.Counts._fields_ if f != "reserved"}
        self.n = c.n

    def row_counts(self, l_rows=False):
        """Per-row arrays: |U row|, the reference's nz_row_U, |L column| and,
        with l_rows (needs the l_row_stats option), |L row|."""
        n = self.n
        u = np.zeros(n, np.int32)
        nzu = np.zeros(n, np.int32)
        lc = np.zeros(n, np.int32)
        lr = np.zeros(n, np.int32) if l_rows else None
        self.ctx._check(self.ctx._L.gsofa_result_row_counts(self._h, _ptr(u), _ptr(nzu), _ptr(lc),
                                                            _ptr(lr)), "row_counts")
        out = dict(nnz_u_row=u, nz_row_u=nzu, nnz_l_col=lc)
        if l_rows:
            out["nnz_l_row"] = lr
        return out

    def digests(self, l_rows=False):
        """64-bit column-set digests per U row and L column (and L row)."""
        n = self.n
        du = np.zeros(n, np.uint64)
        dl = np.zeros(n, np.uint64)
        dr = np.zeros(n, np.uint64) if l_rows else None
        self.ctx._check(self.ctx._L.gsofa_result_digests(self._h, _ptr(du), _ptr(dl), _ptr(dr)),
                        "digests")
        out = dict(dig_u_row=du, dig_l_col=dl)
        if l_rows:
            out["dig_l_row"] = dr
        return out

    def supernodes(self):
        """(flags int8[n], boundaries): non-zero flags start a supernode."""
        flags = np.zeros(self.n, np.int8)
        cnt = ctypes.c_int64()
        self.ctx._check(self.ctx._L.gsofa_result_supernodes(self._h, _ptr(flags), None, 0,
                                                            ctypes.byref(cnt)), "supernodes")
        return flags, np.nonzero(flags)[0].astype(np.int32)

    def lmask(self):
        """(n, 4) uint32: bit j of column f's mask is L(f+1+j, f) != 0."""
        m = np.zeros((self.n, 4), np.uint32)
        self.ctx._check(self.ctx._L.gsofa_result_lmask(self._h, _ptr(m)), "lmask")
        return m

    def _pattern(self, fn):
        ptr = np.zeros(self.n + 1, np.int64)
        self.ctx._check(fn(self._h, _ptr(ptr), None, 0), "pattern")
        ids = np.zeros(max(int(ptr[-1]), 1), np.int32)
        self.ctx._check(fn(self._h, _ptr(ptr), _ptr(ids), ids.shape[0]), "pattern")
        return ptr, ids[:ptr[-1]]

    def supernodal(self):
        """Supernodal block form: block_start (nblocks + 1), and per block the
        sorted off-block L rows (lptr, lrows) and U columns (uptr, ucols)."""
        nb, nl, nu = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        f = self.ctx._L.gsofa_result_supernodal
        self.ctx._check(f(self._h, ctypes.byref(nb), ctypes.byref(nl), ctypes.byref(nu), None, None,
                          None, None, None), "supernodal")
        start = np.zeros(nb.value + 1, np.int32)
        lptr = np.zeros(nb.value + 1, np.int64)
        uptr = np.zeros(nb.value + 1, np.int64)
        lrows = np.zeros(max(nl.value, 1), np.int32)
        ucols = np.zeros(max(nu.value, 1), np.int32)
        self.ctx._check(f(self._h, None, None, None, _ptr(start), _ptr(lptr), _ptr(lrows), _ptr(uptr),
                          _ptr(ucols)), "supernodal")
        return dict(block_start=start, lptr=lptr, lrows=lrows[:nl.value], uptr=uptr,
                    ucols=ucols[:nu.value])

    def pattern_u(self):
        """U by rows: (rowptr[n+1], sorted column ids)."""
        return self._pattern(self.ctx._L.gsofa_result_pattern_u)

    def pattern_l(self):
        """L by columns: (colptr[n+1], sorted row ids)."""
        return self._pattern(self.ctx._L.gsofa_result_pattern_l)

    def close(self):
        if getattr(self, "_h", None):
            if self._owned:
                self.ctx._L.gsofa_result_destroy(self._h)
            self._h = None


def write_binary(path, row_begin, row_end, col):
    """Binary CSR file (row v = col[row_begin[v]:row_end[v]]); no GPU needed."""
    beg = np.ascontiguousarray(row_begin, dtype=np.int32)
    end = np.ascontiguousarray(row_end, dtype=np.int32)
    c = np.ascontiguousarray(col, dtype=np.int32)
    rc = C.load().gsofa_write_csr_binary(os.fsencode(path), beg.shape[0], c.shape[0], _ptr(beg),
                                         _ptr(end), _ptr(c))
    if rc != C.OK:
        raise GsofaError(rc, "write_csr_binary %s" % path)


def read_binary(path):
    """(row_begin, row_end, col) of a binary CSR file; no GPU needed."""
    L = C.load()
    n, nnz = ctypes.c_int32(), ctypes.c_int64()
    rc = L.gsofa_read_csr_binary(os.fsencode(path), ctypes.byref(n), ctypes.byref(nnz), None, None,
                                 None)
    if rc != C.OK:
        raise GsofaError(rc, "read_csr_binary %s" % path)
    beg = np.zeros(n.value, np.int32)
    end = np.zeros(n.value, np.int32)
    col = np.zeros(max(nnz.value, 1), np.int32)
    rc = L.gsofa_read_csr_binary(os.fsencode(path), ctypes.byref(n), ctypes.byref(nnz), _ptr(beg),
                                 _ptr(end), _ptr(col))
    if rc != C.OK:
        raise GsofaError(rc, "read_csr_binary %s" % path)
    return beg, end, col[:nnz.value]


def convert_dat(beg_file, end_file, csr_file, out_path):
    """The reference's three ASCII files into one binary CSR file."""
    rc = C.load().gsofa_convert_dat_to_binary(os.fsencode(beg_file), os.fsencode(end_file),
                                              os.fsencode(csr_file), os.fsencode(out_path))
    if rc != C.OK:
        raise GsofaError(rc, "convert_dat_to_binary -> %s" % out_path)


def symbfact_min_id(argv, rank=0):
    """The reference's entry point: argv is the full vector including the
    program name (11 entries: SOA layout; 6 entries: SPO layout).
    Returns (fill_count, time_ms, N_supernodes, TEPS_edges)."""
    L = C.load()
    args = [a.encode() if isinstance(a, str) else a for a in argv]
    arr = (ctypes.c_char_p * len(args))(*args)
    fill = ctypes.c_uint64()
    ms = ctypes.c_double()
    nsup = ctypes.c_int32()
    teps = ctypes.c_uint64()
    rc = L.gsofa_symbfact_min_id(len(args), arr, int(rank), ctypes.byref(fill), ctypes.byref(ms),
                                 ctypes.byref(nsup), ctypes.byref(teps))
    if rc != C.OK:
        raise GsofaError(rc, "symbfact_min_id failed: %s" % L.gsofa_status_string(rc).decode())
    return fill.value, ms.value, nsup.value, teps.value
