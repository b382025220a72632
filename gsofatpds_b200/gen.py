"""Seeded synthetic sparsity patterns standing in for the reference's
SuperLU_DIST-reordered inputs (the reference's own large test graph, pre2,
n=659,033, is not available).  Every generator returns ``(n, rowptr, col)``:
an int32 CSR with contiguous rows, full diagonal, no duplicate entries and
sorted column ids.  ``write_dat`` writes the reference's ASCII layout.

Workloads (the five benchmark shapes):
  * ``random_extra``   n=20,000: diagonal + tridiagonal + 3 uniform columns/row
  * ``circuit_like``   n=659,033, ~5.83M nnz: diagonal, band |i-j|<=8 kept
                       with p=0.3, Zipf(1.2) long-range degrees capped at 2,000
                       on a calibrated fraction of rows, uniform columns, one
                       seeded symmetric permutation
  * ``grid_nd``        2D/3D 5/7/9/27-point grid patterns in nested-dissection
                       order from deterministic recursive coordinate bisection
                       (separator planes numbered last)
  * ``random_banded``  unsymmetric band (half-bandwidth bw, entries kept with
                       p=0.5) plus uniform off-band entries per row
  * ``batch_mix`` / ``request_stream``: the batched and serving mixes.
"""
import math

import numpy as np

__all__ = ["random_extra", "circuit_like", "circuit_like_calibration", "grid_nd",
           "random_banded", "batch_mix", "request_stream", "write_dat", "from_coo",
           "csr_to_beg_end"]


def from_coo(n, r, c):
    """Deduplicated, row-sorted, column-sorted CSR from coordinate lists."""
    r = np.asarray(r, np.int64)
    c = np.asarray(c, np.int64)
    key = np.sort(r * n + c)
    if key.size:
        key = key[np.concatenate(([True], key[1:] != key[:-1]))]
    rows = (key // n).astype(np.int64)
    col = (key % n).astype(np.int32)
    cnt = np.bincount(rows, minlength=n)
    rowptr = np.zeros(n + 1, np.int64)
    np.cumsum(cnt, out=rowptr[1:])
    if rowptr[-1] >= 2**31:
        raise ValueError("nnz does not fit int32 row pointers")
    return n, rowptr.astype(np.int32), col


def csr_to_beg_end(rowptr):
    rowptr = np.asarray(rowptr, np.int32)
    return rowptr[:-1].copy(), rowptr[1:].copy()


def random_extra(n=20000, extra=3, seed=1):
    """Diagonal + tridiagonal band + `extra` uniform columns per row."""
    rng = np.random.default_rng(seed)
    i = np.arange(n, dtype=np.int64)
    rs = [i, i[1:], i[:-1]]
    cs = [i, i[1:] - 1, i[:-1] + 1]
    rs.append(np.repeat(i, extra))
    cs.append(rng.integers(0, n, size=n * extra))
    return from_coo(n, np.concatenate(rs), np.concatenate(cs))


def _zipf_capped(rng, size, a=1.2, cap=2000):
    k = np.arange(1, cap + 1, dtype=np.float64)
    p = k ** (-a)
    p /= p.sum()
    return rng.choice(np.arange(1, cap + 1), size=size, p=p)


def circuit_like_calibration(n=659033, target_nnz=5830000, band=8, p_band=0.3,
                             a=1.2, cap=2000):
    """Fraction of rows that receive Zipf(a)-distributed long-range links so
    that the expected nnz (before deduplication) equals `target_nnz`.

    Zipf(1.2) capped at 2,000 has mean ~121 links per row, so giving every row
    a Zipf degree would produce ~80M entries instead of ~5.83M; the law is
    therefore applied to a calibrated fraction q of the rows."""
    k = np.arange(1, cap + 1, dtype=np.float64)
    p = k ** (-a)
    mean = float((k * p).sum() / p.sum())
    band_expected = p_band * sum(2 * (n - d) for d in range(1, band + 1))
    remaining = target_nnz - n - band_expected
    q = remaining / (n * mean)
    return max(0.0, min(1.0, q)), mean


def circuit_like(n=659033, target_nnz=5830000, seed=2, band=8, p_band=0.3, a=1.2, cap=2000):
    """Circuit-like unsymmetric pattern of the reference test graph's shape."""
    rng = np.random.default_rng(seed)
    q, _ = circuit_like_calibration(n, target_nnz, band, p_band, a, cap)
    i = np.arange(n, dtype=np.int64)
    rs = [i]
    cs = [i]
    for d in range(1, band + 1):
        for sgn in (1, -1):
            src = i[:-d] if sgn > 0 else i[d:]
            dst = src + sgn * d
            keep = rng.random(src.shape[0]) < p_band
            rs.append(src[keep])
            cs.append(dst[keep])
    has = rng.random(n) < q
    lr_rows = i[has]
    deg = _zipf_capped(rng, lr_rows.shape[0], a, cap)
    rs.append(np.repeat(lr_rows, deg))
    cs.append(rng.integers(0, n, size=int(deg.sum())))
    r = np.concatenate(rs)
    c = np.concatenate(cs)
    perm = rng.permutation(n)  # one seeded symmetric permutation P A P^T
    return from_coo(n, perm[r], perm[c])


def _nd_order(dims, leaf=64):
    """Recursive coordinate bisection order of the cells of a box grid.
    Returns `order`: new id -> old linear (C-order) cell index."""
    dims = tuple(int(d) for d in dims)
    strides = np.cumprod((1,) + dims[::-1][:-1])[::-1]
    out = []

    def cells(lo, hi):
        axes = [np.arange(lo[d], hi[d]) for d in range(len(dims))]
        g = np.meshgrid(*axes, indexing="ij")
        lin = np.zeros(g[0].shape, np.int64)
        for d in range(len(dims)):
            lin += g[d] * strides[d]
        return lin.ravel()

    stack = [(tuple(0 for _ in dims), dims, False)]
    while stack:
        lo, hi, emit = stack.pop()
        ext = [hi[d] - lo[d] for d in range(len(dims))]
        if emit or math.prod(ext) <= leaf or max(ext) < 3:
            if math.prod(ext) > 0:
                out.append(cells(lo, hi))
            continue
        d = int(np.argmax(ext))
        mid = lo[d] + ext[d] // 2
        left_hi = list(hi)
        left_hi[d] = mid
        right_lo = list(lo)
        right_lo[d] = mid + 1
        sep_lo = list(lo)
        sep_lo[d] = mid
        sep_hi = list(hi)
        sep_hi[d] = mid + 1
        # pushed in reverse: left half, right half, then the separator last
        stack.append((tuple(sep_lo), tuple(sep_hi), True))
        stack.append((tuple(right_lo), tuple(hi), False))
        stack.append((tuple(lo), tuple(left_hi), False))
    return np.concatenate(out)


def grid_nd(dims, stencil="7", leaf=64, natural=False):
    """Grid-graph pattern (symmetric) in nested-dissection order.

    dims: (nx, ny) or (nx, ny, nz).  stencil: "5"/"9" for 2D, "7"/"27" for 3D.
    """
    dims = tuple(int(d) for d in dims)
    nd = len(dims)
    n = math.prod(dims)
    if nd == 2:
        offs = [(0, 0), (1, 0), (-1, 0), (0, 1), (0, -1)] if stencil == "5" else \
            [(a, b) for a in (-1, 0, 1) for b in (-1, 0, 1)]
    else:
        offs = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)] \
            if stencil == "7" else [(a, b, c) for a in (-1, 0, 1) for b in (-1, 0, 1) for c in (-1, 0, 1)]
    coords = np.indices(dims).reshape(nd, -1)
    strides = np.cumprod((1,) + dims[::-1][:-1])[::-1]
    lin = np.arange(n, dtype=np.int64)
    rs, cs = [], []
    for o in offs:
        nb = coords + np.array(o).reshape(nd, 1)
        ok = np.all((nb >= 0) & (nb < np.array(dims).reshape(nd, 1)), axis=0)
        nl = (nb[:, ok] * strides.reshape(nd, 1)).sum(axis=0)
        rs.append(lin[ok])
        cs.append(nl)
    r = np.concatenate(rs)
    c = np.concatenate(cs)
    if natural:
        return from_coo(n, r, c)
    order = _nd_order(dims, leaf)
    inv = np.empty(n, np.int64)
    inv[order] = np.arange(n)
    return from_coo(n, inv[r], inv[c])


def random_banded(n, bw=8, extra=2, p_band=0.5, seed=3):
    """Unsymmetric band: diagonal, |i-j|<=bw kept with p_band, plus `extra`
    uniform off-band columns per row."""
    rng = np.random.default_rng(seed)
    i = np.arange(n, dtype=np.int64)
    rs = [i]
    cs = [i]
    for d in range(1, bw + 1):
        for sgn in (1, -1):
            src = i[:-d] if sgn > 0 else i[d:]
            keep = rng.random(src.shape[0]) < p_band
            rs.append(src[keep])
            cs.append(src[keep] + sgn * d)
    rs.append(np.repeat(i, extra))
    cs.append(rng.integers(0, n, size=n * extra))
    return from_coo(n, np.concatenate(rs), np.concatenate(cs))


def batch_mix(count=512, nmin=2000, nmax=60000, seed=4):
    """Batched workload: n log-uniform in [nmin, nmax]; even entries are 2D
    5-point grids in nested-dissection order, odd entries random-banded
    unsymmetric (bandwidth 4-32, 1-4 uniform off-band entries per row)."""
    rng = np.random.default_rng(seed)
    mats = []
    for k in range(count):
        n_t = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
        if k % 2 == 0:
            side = max(2, int(round(math.sqrt(n_t))))
            mats.append(grid_nd((side, side), "5"))
        else:
            bw = int(rng.integers(4, 33))
            extra = int(rng.integers(1, 5))
            mats.append(random_banded(n_t, bw=bw, extra=extra, seed=int(rng.integers(1 << 30))))
    return mats


def request_stream(count=64, rate_hz=20.0, nmin=1000, nmax=1000000, seed=5, max_rb_n=None,
                   big_n=None):
    """Serving stream: Poisson arrivals at `rate_hz`; each request is a seeded
    matrix with n log-uniform in [nmin, nmax] and 5-27 nnz/row: 2D 5/9-point
    and 3D 7/27-point grid patterns in nested-dissection order, or
    random-banded unsymmetric.  Random-banded requests are capped at
    `max_rb_n` rows (their fill grows as n^2).  A draw of at least `big_n`
    rows becomes the stream's largest request kind, the 3D 27-point grid of
    side round(nmax^(1/3)) (100^3: n = 1,000,000, ~26.5M nnz).  Returns
    [(arrival_s, kind, spec)] where spec is passed to ``make_request``."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    kinds = ["grid2d_5", "grid2d_9", "grid3d_7", "grid3d_27", "banded"]
    for _ in range(count):
        t += float(rng.exponential(1.0 / rate_hz))
        n_t = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
        kind = kinds[int(rng.integers(0, len(kinds)))]
        if kind == "banded" and max_rb_n is not None:
            n_t = min(n_t, max_rb_n)
        if big_n is not None and n_t >= big_n:
            kind = "grid3d_27"
            n_t = int(round(nmax ** (1.0 / 3.0))) ** 3
        out.append((t, kind, dict(n=n_t, seed=int(rng.integers(1 << 30)))))
    return out


# the serving benchmark's stream: 48 requests at 20/s, random-banded
# requests capped at 100,000 rows, draws of 500,000 rows or more become
# 100^3 27-point grids
SERVE_STREAM = dict(count=48, rate_hz=20.0, nmin=1000, nmax=1000000, seed=5, max_rb_n=100000,
                    big_n=500000)


def make_request(kind, spec):
    n_t = spec["n"]
    if kind.startswith("grid2d"):
        side = max(2, int(round(math.sqrt(n_t))))
        return grid_nd((side, side), kind.split("_")[1])
    if kind.startswith("grid3d"):
        side = max(2, int(round(n_t ** (1.0 / 3.0))))
        return grid_nd((side, side, side), kind.split("_")[1])
    rng = np.random.default_rng(spec["seed"])
    # 5-27 nnz/row: 1 + 2*bw*0.5 + extra
    bw = int(rng.integers(2, 24))
    extra = int(rng.integers(1, 5))
    return random_banded(n_t, bw=bw, extra=extra, seed=spec["seed"])


def write_dat(path_prefix, n, rowptr, col):
    """Write the reference's ASCII files: <prefix>colbeg_<n>.dat,
    <prefix>colend_<n>.dat, <prefix>csr_<n>.dat.  Returns the three paths."""
    beg, end = csr_to_beg_end(rowptr)
    pb = "%scolbeg_%d.dat" % (path_prefix, n)
    pe = "%scolend_%d.dat" % (path_prefix, n)
    pc = "%scsr_%d.dat" % (path_prefix, n)
    with open(pc, "w") as f:
        f.write("%d\n%d\n" % (col.shape[0], n))
        f.write(" ".join(map(str, col.tolist())))
        f.write("\n")
    with open(pb, "w") as f:
        f.write(" ".join(map(str, beg.tolist())))
        f.write("\n")
    with open(pe, "w") as f:
        f.write(" ".join(map(str, end.tolist())))
        f.write("\n")
    return pb, pe, pc
