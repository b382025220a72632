"""The seeded generators behind every benchmark input (CPU only): the CSR
contract their docstring states, determinism, the nested-dissection order
of the grids, the circuit-like calibration, the batched and serving mixes,
and the reference ASCII writer."""
import numpy as np
import pytest

from gsofatpds_b200 import gen


def _check_csr(n, rp, col):
    assert rp.dtype == np.int32 and col.dtype == np.int32
    assert rp.shape == (n + 1,) and rp[0] == 0 and rp[-1] == col.shape[0]
    assert np.all(np.diff(rp) >= 1)
    rows = np.repeat(np.arange(n), np.diff(rp))
    assert np.all((col >= 0) & (col < n))
    same = rows[1:] == rows[:-1]
    assert np.all(np.diff(col.astype(np.int64))[same] > 0), "columns sorted, no duplicates"
    diag = np.zeros(n, bool)
    diag[rows[col == rows]] = True
    assert diag.all(), "full diagonal"


def _components_without(n, rp, col, removed):
    keep = np.ones(n, bool)
    keep[removed] = False
    seen = ~keep
    comps = 0
    for s in range(n):
        if seen[s]:
            continue
        comps += 1
        seen[s] = True
        stack = [s]
        while stack:
            u = stack.pop()
            for w in col[rp[u]:rp[u + 1]]:
                if not seen[w]:
                    seen[w] = True
                    stack.append(w)
    return comps


@pytest.mark.parametrize("spec", [
    ("random_extra", dict(n=3000, extra=3, seed=1)),
    ("random_banded", dict(n=2500, bw=6, extra=2, seed=4)),
    ("circuit_like", dict(n=20000, target_nnz=177000, seed=2)),
    ("grid2d_5", None), ("grid2d_9", None), ("grid3d_7", None), ("grid3d_27", None)])
def test_csr_contract(spec):
    name, kw = spec
    if name.startswith("grid"):
        dims = (23, 17) if name.startswith("grid2d") else (9, 8, 7)
        n, rp, col = gen.grid_nd(dims, name.split("_")[1])
    else:
        n, rp, col = getattr(gen, name)(**kw)
    _check_csr(n, rp, col)


def test_seeded_and_deterministic():
    a = gen.random_banded(3000, bw=5, extra=2, seed=7)
    b = gen.random_banded(3000, bw=5, extra=2, seed=7)
    c = gen.random_banded(3000, bw=5, extra=2, seed=8)
    for x, y in zip(a[1:], b[1:]):
        np.testing.assert_array_equal(x, y)
    assert not np.array_equal(a[2], c[2])


@pytest.mark.parametrize("dims,stencil", [((16, 16), "5"), ((15, 20), "9"), ((8, 8, 8), "7")])
def test_grids_symmetric_and_nested_dissection(dims, stencil):
    n, rp, col = gen.grid_nd(dims, stencil)
    nn, rpn, coln = gen.grid_nd(dims, stencil, natural=True)
    assert n == nn == int(np.prod(dims))
    # symmetric pattern
    rows = np.repeat(np.arange(n), np.diff(rp))
    fwd = set(zip(rows.tolist(), col.tolist()))
    assert all((c, r) in fwd for r, c in fwd)
    # the same graph renumbered: equal degree multisets
    np.testing.assert_array_equal(np.sort(np.diff(rp)), np.sort(np.diff(rpn)))
    # separator last: without the last plane of vertices the graph falls apart
    plane = int(np.prod(sorted(dims)[:-1])) if len(dims) == 3 else min(dims)
    assert _components_without(n, rp, col, np.arange(n - plane, n)) >= 2
    # natural order does not have that property
    assert _components_without(nn, rpn, coln, np.arange(nn - plane, nn)) == 1


def test_circuit_like_calibration():
    q, mean = gen.circuit_like_calibration()
    assert 0.024 < q < 0.026 and 110 < mean < 130
    n = 50000
    target = int(5830000 * n / 659033)
    _, rp, col = gen.circuit_like(n=n, target_nnz=target, seed=2)
    assert abs(col.shape[0] - target) / target < 0.06
    deg = np.diff(rp)
    assert deg.max() > 100  # long-range Zipf rows exist


def test_batch_mix_and_request_stream():
    mats = gen.batch_mix(12, nmin=1000, nmax=8000, seed=3)
    assert len(mats) == 12
    for k, (n, rp, col) in enumerate(mats):
        assert 800 <= n <= 8200
        _check_csr(n, rp, col)
        sym = np.array_equal(np.sort(np.diff(rp)), np.sort(np.diff(gen.from_coo(
            n, col, np.repeat(np.arange(n), np.diff(rp)))[1])))
        if k % 2 == 0:
            assert sym  # even entries are grids (symmetric)
    reqs = gen.request_stream(count=40, rate_hz=10.0, nmin=1000, nmax=50000, seed=5,
                              max_rb_n=20000)
    t = [r[0] for r in reqs]
    assert all(b > a for a, b in zip(t, t[1:]))
    assert abs(np.mean(np.diff([0.0] + t)) - 0.1) < 0.06  # Poisson at 10/s
    for _, kind, spec in reqs:
        assert 1000 <= spec["n"] <= 50000
        if kind == "banded":
            assert spec["n"] <= 20000
    n, rp, col = gen.make_request(*reqs[0][1:])
    _check_csr(n, rp, col)


def test_write_dat_reads_back_with_the_reference_layout(tmp_path):
    from oracle import oracle as O
    n, rp, col = gen.random_extra(500, 2, seed=3)
    pb, pe, pc = gen.write_dat(str(tmp_path) + "/", n, rp, col)
    b, e, c = O.read_dat(pb, pe, pc)
    np.testing.assert_array_equal(b, rp[:-1])
    np.testing.assert_array_equal(e, rp[1:])
    np.testing.assert_array_equal(c, col)
