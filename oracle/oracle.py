"""ctypes binding of the CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only as the checker.  The product library never calls it.
The algorithm and its reference citations are in gsofa_oracle.c.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "libgsofa_oracle.so")
_lib = None

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        L = ctypes.CDLL(_SO)
        vp = ctypes.c_void_p
        L.or_rows.restype = ctypes.c_int
        L.or_rows.argtypes = [ctypes.c_int32, vp, vp, vp, vp, ctypes.c_int64, ctypes.c_int,
                              vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
        L.or_supernodes.restype = ctypes.c_int64
        L.or_supernodes.argtypes = [ctypes.c_int32, vp, vp, ctypes.c_int32, vp]
        L.or_mix64.restype = ctypes.c_uint64
        L.or_mix64.argtypes = [ctypes.c_uint64]
        L.or_read_dat.restype = ctypes.c_int
        L.or_read_dat.argtypes = [ctypes.c_char_p] * 3 + [ctypes.POINTER(ctypes.c_int32),
                                                          ctypes.POINTER(ctypes.c_int64)] + \
            [ctypes.POINTER(ctypes.POINTER(ctypes.c_int32))] * 3
        L.or_free.argtypes = [vp]
        L.or_order_hybrid.restype = ctypes.c_int
        L.or_order_hybrid.argtypes = [ctypes.c_int32, vp, vp, vp, ctypes.c_int32, vp, vp]
        L.or_order_hybrid_trace.restype = ctypes.c_int
        L.or_order_hybrid_trace.argtypes = [ctypes.c_int32, vp, vp, vp, ctypes.c_int32, vp, vp,
                                            vp, ctypes.c_int64, vp]
        L.or_order_nd.restype = ctypes.c_int
        L.or_order_nd.argtypes = [ctypes.c_int32, vp, vp, vp, ctypes.c_int32, ctypes.c_int32, vp,
                                  vp]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def mix64(x):
    return lib().or_mix64(int(x))


def rows(beg, end, col, rows=None, nthreads=0, pattern=False):
    """Run the per-source label search for `rows` (default: every row).

    Returns a dict of numpy arrays indexed like `rows`: nnzL, nnzU, nzU_ref,
    digL, digU, fills, e_alg, v_alg, lback (shape (k,4)); with pattern=True
    also Lptr/Lcols and Uptr/Ucols (sorted column ids per row, CSR layout).
    """
    beg = np.ascontiguousarray(beg, dtype=np.int32)
    end = np.ascontiguousarray(end, dtype=np.int32)
    col = np.ascontiguousarray(col, dtype=np.int32)
    n = beg.shape[0]
    if rows is None:
        k = n
        rws = None
    else:
        rws = np.ascontiguousarray(rows, dtype=np.int32)
        k = rws.shape[0]
    out = dict(
        nnzL=np.zeros(k, np.int32), nnzU=np.zeros(k, np.int32), nzU_ref=np.zeros(k, np.int32),
        digL=np.zeros(k, np.uint64), digU=np.zeros(k, np.uint64), fills=np.zeros(k, np.uint64),
        e_alg=np.zeros(k, np.uint64), v_alg=np.zeros(k, np.uint64),
        lback=np.zeros((k, 4), np.uint32))
    rc = lib().or_rows(n, _p(beg), _p(end), _p(col), _p(rws), k, int(nthreads),
                       _p(out["nnzL"]), _p(out["nnzU"]), _p(out["nzU_ref"]),
                       _p(out["digL"]), _p(out["digU"]), _p(out["fills"]),
                       _p(out["e_alg"]), _p(out["v_alg"]), _p(out["lback"]),
                       None, None, None, None)
    if rc != 0:
        raise ValueError("oracle: invalid CSR input or out of memory")
    if pattern:
        Lptr = np.zeros(k + 1, np.int64)
        Uptr = np.zeros(k + 1, np.int64)
        np.cumsum(out["nnzL"], out=Lptr[1:])
        np.cumsum(out["nnzU"], out=Uptr[1:])
        Lcols = np.zeros(max(int(Lptr[-1]), 1), np.int32)
        Ucols = np.zeros(max(int(Uptr[-1]), 1), np.int32)
        rc = lib().or_rows(n, _p(beg), _p(end), _p(col), _p(rws), k, int(nthreads),
                           None, None, None, None, None, None, None, None, None,
                           _p(Lptr), _p(Lcols), _p(Uptr), _p(Ucols))
        if rc != 0:
            raise ValueError("oracle: pattern pass failed")
        out.update(Lptr=Lptr, Lcols=Lcols[:Lptr[-1]], Uptr=Uptr, Ucols=Ucols[:Uptr[-1]])
    return out


def supernodes(nzU_ref, lback, mss):
    """Reference supernode rule; returns (detected_count, flags int8[n])."""
    nz = np.ascontiguousarray(nzU_ref, dtype=np.int32)
    lb = np.ascontiguousarray(lback, dtype=np.uint32)
    n = nz.shape[0]
    flags = np.zeros(n, np.int8)
    c = lib().or_supernodes(n, _p(nz), _p(lb), int(mss), _p(flags))
    if c < 0:
        raise ValueError("oracle: bad supernode arguments")
    return int(c), flags


def order_nd(beg, end, col, leaf=32, max_rounds=512):
    """Level-set nested dissection of A + A^T (gsofa_order_oracle.c).
    Returns (perm, stats): new index k <- old perm[k]; stats = (rounds,
    splits, separator vertices, largest separator)."""
    b = np.ascontiguousarray(beg, dtype=np.int32)
    e = np.ascontiguousarray(end, dtype=np.int32)
    c = np.ascontiguousarray(col, dtype=np.int32)
    n = b.shape[0]
    perm = np.zeros(max(n, 1), np.int32)
    stats = np.zeros(4, np.int64)
    rc = lib().or_order_nd(n, _p(b), _p(e), _p(c), int(leaf), int(max_rounds), _p(perm),
                           _p(stats))
    if rc != 0:
        raise ValueError("oracle: bad ordering arguments")
    return perm[:n], tuple(int(x) for x in stats)


def order_hybrid(beg, end, col, leaf=32):
    """The hybrid nested-dissection rule (gsofa_order_hybrid_oracle.c):
    level-set ND where, at each split, a multilevel separator is also
    computed and the smaller one used.  Returns (perm, stats) like order_nd."""
    b = np.ascontiguousarray(beg, dtype=np.int32)
    e = np.ascontiguousarray(end, dtype=np.int32)
    c = np.ascontiguousarray(col, dtype=np.int32)
    n = b.shape[0]
    perm = np.zeros(max(n, 1), np.int32)
    stats = np.zeros(4, np.int64)
    rc = lib().or_order_hybrid(n, _p(b), _p(e), _p(c), int(leaf), _p(perm), _p(stats))
    if rc != 0:
        raise ValueError("oracle: bad ordering arguments")
    return perm[:n], tuple(int(x) for x in stats)


def order_hybrid_trace(beg, end, col, leaf=32):
    """order_hybrid, also returning every split: an int32 array of rows
    (range start, component size, |A|, |B|, |S|, rule 0 level-set / 1
    multilevel, the level-set separator's size).  The component's range holds
    A, then B, then S."""
    b = np.ascontiguousarray(beg, dtype=np.int32)
    e = np.ascontiguousarray(end, dtype=np.int32)
    c = np.ascontiguousarray(col, dtype=np.int32)
    n = b.shape[0]
    perm = np.zeros(max(n, 1), np.int32)
    stats = np.zeros(4, np.int64)
    cap = max(n, 1)
    trace = np.zeros((cap, 7), np.int32)
    cnt = np.zeros(1, np.int64)
    rc = lib().or_order_hybrid_trace(n, _p(b), _p(e), _p(c), int(leaf), _p(perm), _p(stats),
                                     _p(trace), cap, _p(cnt))
    if rc != 0 or cnt[0] > cap:
        raise ValueError("oracle: bad ordering arguments")
    return perm[:n], tuple(int(x) for x in stats), trace[:int(cnt[0])]


def read_dat(beg_file, end_file, csr_file):
    """Reference ASCII reader -> (beg, end, col) int32 arrays."""
    L = lib()
    n = ctypes.c_int32()
    nnz = ctypes.c_int64()
    pb, pe, pc = (ctypes.POINTER(ctypes.c_int32)() for _ in range(3))
    rc = L.or_read_dat(beg_file.encode(), end_file.encode(), csr_file.encode(),
                       ctypes.byref(n), ctypes.byref(nnz), ctypes.byref(pb),
                       ctypes.byref(pe), ctypes.byref(pc))
    if rc != 0:
        raise ValueError("oracle: cannot parse %s/%s/%s" % (beg_file, end_file, csr_file))
    try:
        beg = np.ctypeslib.as_array(pb, shape=(n.value,)).copy()
        end = np.ctypeslib.as_array(pe, shape=(n.value,)).copy()
        col = np.ctypeslib.as_array(pc, shape=(max(nnz.value, 1),)).copy()[:nnz.value]
    finally:
        L.or_free(ctypes.cast(pb, ctypes.c_void_p))
        L.or_free(ctypes.cast(pe, ctypes.c_void_p))
        L.or_free(ctypes.cast(pc, ctypes.c_void_p))
    return beg, end, col


def transpose(beg, end, col):
    """CSR of A^T (rows contiguous) from the possibly non-contiguous CSR of A."""
    beg = np.asarray(beg, np.int64)
    end = np.asarray(end, np.int64)
    n = beg.shape[0]
    deg = end - beg
    rows = np.repeat(np.arange(n, dtype=np.int32), deg)
    idx = np.concatenate([np.arange(b, e) for b, e in zip(beg, end)]) if n else np.zeros(0, np.int64)
    cols = np.asarray(col)[idx] if idx.size else np.zeros(0, np.int32)
    order = np.argsort(cols, kind="stable")
    tcol = rows[order].astype(np.int32)
    cnt = np.bincount(cols, minlength=n).astype(np.int64)
    tptr = np.zeros(n + 1, np.int64)
    np.cumsum(cnt, out=tptr[1:])
    return tptr[:-1].astype(np.int32), tptr[1:].astype(np.int32), tcol
