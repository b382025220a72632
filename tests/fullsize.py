"""Full-size parity records: what the oracle and the device produce for one
matrix, reduced to totals and hashes of every per-row array so that
full-size answers can be committed as small fixtures.

A record holds
  totals  fill_count, nnz_u, nnz_l, edges_alg, vertices_alg, n_supernodes
          (printed form: detected + 1, SOA symbfact_warp_centric_new_scheduling.cuh:3549)
  hashes  the first 16 hex digits of SHA-256 over the little-endian bytes
          of each per-row array (HASHED below, with its dtype): U-row and
          L-column/L-row counts, the reference's nz_row_U counter, the
          64-bit digests, the 128-bit L-column masks and the supernode flags.

The oracle side (oracle_record) runs the CPU label search over every row of
A and, for an unsymmetric pattern, every row of A^T (its U rows are the L
columns of A).  The device side (device_record) reads the same arrays from a
gsofatpds_b200 Result.  Test infrastructure only.
"""
import hashlib

import numpy as np

# name -> dtype of the hashed array
HASHED = {
    "nnz_u_row": np.int32, "nz_row_u": np.int32, "nnz_l_col": np.int32, "nnz_l_row": np.int32,
    "dig_u_row": np.uint64, "dig_l_col": np.uint64, "dig_l_row": np.uint64,
    "lmask": np.uint32, "sn_flags": np.int8,
}
TOTALS = ("fill_count", "nnz_u", "nnz_l", "edges_alg", "vertices_alg", "n_supernodes")


def h16(a, dtype):
    a = np.ascontiguousarray(np.asarray(a).astype(np.dtype(dtype).newbyteorder("<")))
    return hashlib.sha256(a.tobytes()).hexdigest()[:16]


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


def pattern_symmetric(beg, end, col):
    """True when the pattern of A (duplicates ignored) equals that of A^T."""
    beg = np.asarray(beg, np.int64)
    end = np.asarray(end, np.int64)
    n = beg.shape[0]
    deg = end - beg
    rows = np.repeat(np.arange(n, dtype=np.int64), deg)
    idx = np.concatenate([np.arange(b, e) for b, e in zip(beg, end)]) if n else np.zeros(0, np.int64)
    cols = np.asarray(col, np.int64)[idx]
    k1 = np.unique(rows * n + cols)
    k2 = np.unique(cols * n + rows)
    return k1.shape == k2.shape and bool(np.all(k1 == k2))


def oracle_record(beg, end, col, mss, nthreads=0, symmetric=None):
    """Totals and hashes from the CPU oracle (every row of A, and every row
    of A^T unless the pattern is symmetric)."""
    from oracle import oracle as O
    r = O.rows(beg, end, col, nthreads=nthreads)
    if symmetric is None:
        symmetric = pattern_symmetric(beg, end, col)
    if symmetric:
        rt = r
    else:
        tb, te, tc = O.transpose(beg, end, col)
        rt = O.rows(tb, te, tc, nthreads=nthreads)
    nsup, flags = O.supernodes(r["nzU_ref"], r["lback"], mss)
    arrays = {
        "nnz_u_row": r["nnzU"], "nz_row_u": r["nzU_ref"], "nnz_l_col": rt["nnzU"],
        "nnz_l_row": r["nnzL"], "dig_u_row": r["digU"], "dig_l_col": rt["digU"],
        "dig_l_row": r["digL"], "lmask": colmask_from_lback(r["lback"]), "sn_flags": flags,
    }
    return {
        "n": int(np.asarray(beg).shape[0]), "nnz": int(np.asarray(col).shape[0]), "mss": int(mss),
        "symmetric": bool(symmetric),
        "totals": {"fill_count": int(r["fills"].sum()), "nnz_u": int(r["nnzU"].sum()),
                   "nnz_l": int(r["nnzL"].sum()), "edges_alg": int(r["e_alg"].sum()),
                   "vertices_alg": int(r["v_alg"].sum()), "n_supernodes": nsup + 1},
        "hashes": {k: h16(v, HASHED[k]) for k, v in arrays.items()},
    }


def device_record(res, l_rows=True):
    """The same record from a device Result (l_rows: the factorization ran
    with l_row_stats, so the L-row counts and digests exist)."""
    rc = res.row_counts(l_rows=l_rows)
    dg = res.digests(l_rows=l_rows)
    flags, _ = res.supernodes()
    arrays = {"nnz_u_row": rc["nnz_u_row"], "nz_row_u": rc["nz_row_u"],
              "nnz_l_col": rc["nnz_l_col"], "dig_u_row": dg["dig_u_row"],
              "dig_l_col": dg["dig_l_col"], "lmask": res.lmask(), "sn_flags": flags}
    if l_rows:
        arrays["nnz_l_row"] = rc["nnz_l_row"]
        arrays["dig_l_row"] = dg["dig_l_row"]
    c = res.counts
    return {"totals": {k: int(c[k]) for k in TOTALS},
            "hashes": {k: h16(v, HASHED[k]) for k, v in arrays.items()}}


def compare(dev, ref, what=""):
    """Assert every total and every hash the device record has equals the
    oracle's."""
    for k in TOTALS:
        assert dev["totals"][k] == ref["totals"][k], "%s %s: device %d, oracle %d" % (
            what, k, dev["totals"][k], ref["totals"][k])
    for k, v in dev["hashes"].items():
        assert v == ref["hashes"][k], "%s per-row array %s differs from the oracle's" % (what, k)
