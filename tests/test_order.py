"""Fill-reducing ordering (gsofa_order_nd) and the symmetric permutation
(gsofa_matrix_permute).

The reference has no ordering code (its inputs arrive permuted by
SuperLU_DIST, README.md:27-33), so the oracle is pinned three ways: known
answers derived by hand from the published level-set nested dissection rule,
a second restatement of the rule written independently below (recursive,
pure Python, small graphs only) that must agree with the C oracle exactly,
and fill properties (the ordering must cut the fill of scrambled grids).
The device ordering must then equal the oracle's permutation bit for bit.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import load_bc


def _csr(rows):
    n = len(rows)
    beg = np.zeros(n, np.int32)
    end = np.zeros(n, np.int32)
    col = []
    for i, r in enumerate(rows):
        beg[i] = len(col)
        col.extend(r)
        end[i] = len(col)
    return beg, end, np.array(col, np.int32)


def _sym_adj(beg, end, col):
    n = len(beg)
    adj = [set() for _ in range(n)]
    for v in range(n):
        for w in col[beg[v]:end[v]]:
            w = int(w)
            if w != v:
                adj[v].add(w)
                adj[w].add(v)
    return adj


def _sym_csr(beg, end, col):
    """A + A^T as (row starts, neighbour ids): distinct, no loops."""
    adj = _sym_adj(beg, end, col)
    rp = np.zeros(len(adj) + 1, np.int64)
    rp[1:] = np.cumsum([len(a) for a in adj])
    flat = np.array([w for a in adj for w in sorted(a)], np.int64)
    return rp, flat


def nd_python(beg, end, col, leaf, max_rounds=512):
    """Level-set nested dissection, restated recursively from the rule:
    components in root order; a component above `leaf` is cut at the middle
    level m of a BFS from r1 (smallest id at the largest distance from its
    smallest id), m = first level where twice the running count reaches
    |c|, capped at e - 1; separator = level-m vertices next to level m + 1;
    layout [A | B | S]."""
    n = len(beg)
    adj = _sym_adj(beg, end, col)
    perm = [None] * n
    st = dict(rounds=0, splits=0, sep=0, maxsep=0)

    def place(vs, lo):
        for i, v in enumerate(sorted(vs)):
            perm[lo + i] = v

    def components(vs):
        left, out = set(vs), []
        for r in sorted(vs):
            if r not in left:
                continue
            comp, stack = {r}, [r]
            left.discard(r)
            while stack:
                u = stack.pop()
                for w in adj[u]:
                    if w in left:
                        left.discard(w)
                        comp.add(w)
                        stack.append(w)
            out.append(comp)
        return out

    def bfs(src, c):
        d, frontier = {src: 0}, [src]
        while frontier:
            nxt = []
            for u in frontier:
                for w in adj[u]:
                    if w in c and w not in d:
                        d[w] = d[u] + 1
                        nxt.append(w)
            frontier = nxt
        return d

    def solve(vs, lo, depth):
        st["rounds"] = max(st["rounds"], depth + 1)
        off = lo
        for c in components(vs):
            if len(c) <= leaf or depth == max_rounds - 1:
                place(c, off)
            else:
                d1 = bfs(min(c), c)
                e1 = max(d1.values())
                r1 = min(v for v in c if d1[v] == e1)
                d = bfs(r1, c)
                e = max(d.values())
                cum, m = 0, 0
                for m in range(e + 1):
                    cum += sum(1 for v in c if d[v] == m)
                    if 2 * cum >= len(c):
                        break
                m = min(m, e - 1)
                S = {v for v in c if d[v] == m and any(w in c and d[w] == m + 1 for w in adj[v])}
                A = {v for v in c if d[v] < m or (d[v] == m and v not in S)}
                B = {v for v in c if d[v] > m}
                place(S, off + len(c) - len(S))
                st["splits"] += 1
                st["sep"] += len(S)
                st["maxsep"] = max(st["maxsep"], len(S))
                if A:
                    solve(A, off, depth + 1)
                if B:
                    solve(B, off + len(A), depth + 1)
            off += len(c)

    if n:
        solve(set(range(n)), 0, 0)
    return np.array(perm, np.int32), (st["rounds"], st["splits"], st["sep"], st["maxsep"])


def _path(n):
    return _csr([[j for j in (i - 1, i + 1) if 0 <= j < n] for i in range(n)])


def _grid2d(nx, ny, rng=None):
    """5-point grid, optionally with its vertices renumbered at random."""
    idx = np.arange(nx * ny).reshape(nx, ny)
    if rng is not None:
        idx = rng.permutation(nx * ny).reshape(nx, ny)
    rows = [[] for _ in range(nx * ny)]
    for i in range(nx):
        for j in range(ny):
            v = idx[i, j]
            rows[v].append(v)
            for di, dj in ((1, 0), (-1, 0), (0, 1), (0, -1)):
                a, b = i + di, j + dj
                if 0 <= a < nx and 0 <= b < ny:
                    rows[v].append(idx[a, b])
    return _csr(rows)


def permuted(beg, end, col, perm):
    """Host P A P^T: row k = row perm[k], column c renamed to iperm[c]."""
    n = len(beg)
    iperm = np.empty(n, np.int32)
    iperm[perm] = np.arange(n, dtype=np.int32)
    rows = [iperm[col[beg[v]:end[v]]] for v in perm]
    return _csr([r.tolist() for r in rows])


def _fill(beg, end, col):
    return int(O.rows(beg, end, col)["fills"].sum())


# ---- the oracle pinned (CPU) ----------------------------------------------------

def test_path_known_answer():
    # 0-1-2-3-4-5-6, leaf 1: BFS from 0 ends at 6; from 6 the levels are
    # 6,5,4,3,2,1,0; m = 3 (2*4 >= 7): S = {3}, A = {6,5,4}, B = {2,1,0};
    # each side of 3 splits again at its middle vertex
    perm, st = O.order_nd(*_path(7), leaf=1)
    assert perm.tolist() == [6, 4, 5, 2, 0, 1, 3]
    assert st == (3, 3, 3, 1)


def test_star_known_answer():
    # centre 0, leaves 1..5: from 1 the levels are {1}, {0}, {2..5}; m = 2
    # capped at e - 1 = 1: S = {0}, A = {1}, B = {2,3,4,5} (four components)
    rows = [[1, 2, 3, 4, 5], [0], [0], [0], [0], [0]]
    perm, st = O.order_nd(*_csr(rows), leaf=1)
    assert perm.tolist() == [1, 2, 3, 4, 5, 0]
    assert st == (2, 1, 1, 1)


def test_no_edges_and_round_cap():
    n = 9
    perm, st = O.order_nd(*_csr([[i] for i in range(n)]), leaf=1)
    assert perm.tolist() == list(range(n)) and st == (1, 0, 0, 0)
    # one round only: the connected path is placed whole, in id order
    perm, st = O.order_nd(*_path(12), leaf=1, max_rounds=1)
    assert perm.tolist() == list(range(12)) and st[0] == 1 and st[1] == 0


@pytest.mark.parametrize("seed", range(24))
def test_oracle_equals_python_restatement(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 70))
    dens = float(rng.uniform(0.0, 0.12))
    rows = []
    for i in range(n):
        r = [int(j) for j in np.nonzero(rng.random(n) < dens)[0]]
        if seed % 3 and rng.random() < 0.7:
            r.append(i)
        rows.append(r)
    b, e, c = _csr(rows)
    leaf = int(rng.choice([1, 2, 4, 8]))
    max_rounds = int(rng.choice([512, 2, 3]))
    pp, sp = nd_python(b, e, c, leaf, max_rounds)
    po, so = O.order_nd(b, e, c, leaf=leaf, max_rounds=max_rounds)
    np.testing.assert_array_equal(po, pp)
    assert so == sp


def test_oracle_cuts_the_fill_of_a_scrambled_grid():
    rng = np.random.default_rng(7)
    b, e, c = _grid2d(40, 40, rng)
    perm, st = O.order_nd(b, e, c, leaf=8)
    assert sorted(perm.tolist()) == list(range(1600))
    f_scr = _fill(b, e, c)
    f_nat = _fill(*_grid2d(40, 40))
    f_nd = _fill(*permuted(b, e, c, perm))
    assert f_nd < f_nat < f_scr, (f_nd, f_nat, f_scr)
    assert st[1] > 50 and st[3] <= 80


# ---- the device ordering (GPU) --------------------------------------------------

def _cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.fixture(scope="module")
def ctx():
    _cuda()
    from gsofatpds_b200 import Context
    c = Context(0)
    yield c
    c.close()


def _cases():
    from gsofatpds_b200 import gen
    from gsofatpds_b200.gen import csr_to_beg_end
    rng = np.random.default_rng(11)
    out = {}
    z = load_bc()
    out["bc"] = (z["beg"], z["end"], z["col"])
    out["grid2d_scrambled"] = _grid2d(90, 70, rng)
    _, rp, col = gen.grid_nd((24, 24, 24), "7")
    b, e = csr_to_beg_end(rp)
    p = np.random.default_rng(3).permutation(len(b)).astype(np.int32)
    out["grid3d_scrambled"] = permuted(b, e, col, p)
    _, rp, col = gen.random_extra(20000, 3, seed=1)
    out["random_extra_20k"] = (*csr_to_beg_end(rp), col)
    _, rp, col = gen.random_banded(20000, bw=2, extra=0, p_band=1.0, seed=5)
    out["banded_long_diameter"] = (*csr_to_beg_end(rp), col)
    out["no_edges"] = _csr([[i] for i in range(300)])
    out["empty_rows"] = _csr([[] for _ in range(50)] + [[0, 1, 2]])
    out["star"] = _csr([list(range(1, 400))] + [[0]] * 399)
    pieces = [[j for j in (i - 1, i + 1) if 0 <= j < 2000 and (i // 100) == (j // 100)]
              for i in range(2000)]
    out["disconnected_paths"] = _csr(pieces)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("leaf", [1, 8, 32])
def test_device_ordering_equals_oracle(ctx, leaf):
    for name, (b, e, c) in _cases().items():
        m = ctx.load_csr(b, e, c)
        perm, st = ctx.order_nd(m, leaf_size=leaf)
        ref, rst = O.order_nd(b, e, c, leaf=leaf)
        np.testing.assert_array_equal(perm, ref, err_msg="%s leaf %d" % (name, leaf))
        assert (st["rounds"], st["splits"], st["separator_vertices"],
                st["max_separator"]) == rst, (name, leaf, st, rst)
        m.close()


@pytest.mark.gpu
def test_device_ordering_round_cap(ctx):
    b, e, c = _grid2d(50, 50, np.random.default_rng(2))
    m = ctx.load_csr(b, e, c)
    for cap in (1, 2, 5):
        perm, st = ctx.order_nd(m, leaf_size=4, max_rounds=cap)
        ref, rst = O.order_nd(b, e, c, leaf=4, max_rounds=cap)
        np.testing.assert_array_equal(perm, ref, err_msg="cap %d" % cap)
        assert st["rounds"] == rst[0] <= cap
    m.close()


@pytest.mark.gpu
def test_permute_then_factor(ctx):
    """P A P^T built on the device factors exactly like the same matrix
    permuted on the host, and the device ordering cuts the grid's fill."""
    rng = np.random.default_rng(5)
    b, e, c = _grid2d(60, 60, rng)
    m = ctx.load_csr(b, e, c)
    perm, _ = ctx.order_nd(m, leaf_size=16)
    pm = ctx.permute(m, perm)
    r = ctx.factor(pm)
    hb, he, hc = permuted(b, e, c, perm)
    ref = O.rows(hb, he, hc)
    assert r.counts["fill_count"] == int(ref["fills"].sum())
    assert r.counts["nnz_l"] == int(ref["nnzL"].sum())
    np.testing.assert_array_equal(r.row_counts()["nnz_u_row"], ref["nnzU"])
    r0 = ctx.factor(m)
    assert r.counts["fill_count"] * 4 < r0.counts["fill_count"]
    for x in (r, r0, pm, m):
        x.close()
    # a permutation that is not one is refused
    m = ctx.load_csr(b, e, c)
    from gsofatpds_b200 import GsofaError
    bad = np.arange(len(b), dtype=np.int32)
    bad[3] = 4
    with pytest.raises(GsofaError):
        ctx.permute(m, bad)
    m.close()


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["--order", "--order-hybrid"])
def test_cli_order_mode(tmp_path, mode):
    """gsofa_cli --order / --order-hybrid: binary file -> device ordering ->
    P A P^T -> factor; the fill equals the oracle's on the same permutation."""
    import subprocess
    _cuda()
    from gsofatpds_b200 import _lib, write_binary
    b, e, c = _grid2d(50, 40, np.random.default_rng(9))
    path = str(tmp_path / "g.gsofacsr")
    write_binary(path, b, e, c)
    out = subprocess.run([_lib.CLI_PATH, mode, path, "128"], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr
    if mode == "--order":
        perm, _ = O.order_nd(b, e, c, leaf=32)
    else:
        perm, _ = O.order_hybrid(b, e, c, leaf=32)
    ref = _fill(*permuted(b, e, c, perm))
    assert "Final Number of fill-ins detected: %d" % ref in out.stdout, out.stdout
    rule = "level-set" if mode == "--order" else "hybrid"
    assert "Ordering (%s nested dissection on the device)" % rule in out.stdout


@pytest.mark.gpu
def test_grid_barrier_wait_runs_out_and_context_survives(ctx):
    """The ordering's grid barrier waits with a time limit: launched waiting
    for one block more than it has, every wait gives up, the kernel returns,
    the host reports GSOFA_ERR_TIMEOUT, and the context still orders."""
    import time
    from gsofatpds_b200 import _lib
    L = _lib.load()
    t0 = time.perf_counter()
    rc = L.gsofa_order_wait_selftest(ctx.handle, 50.0)
    dt = time.perf_counter() - t0
    assert rc == _lib.ERR_TIMEOUT, rc
    assert dt < 5.0, dt
    assert L.gsofa_order_wait_selftest(ctx.handle, 0.0) == _lib.ERR_ARG
    b, e, c = _grid2d(30, 30, np.random.default_rng(4))
    m = ctx.load_csr(b, e, c)
    perm, _ = ctx.order_nd(m, leaf_size=8)
    ref, _ = O.order_nd(b, e, c, leaf=8)
    np.testing.assert_array_equal(perm, ref)
    m.close()


# ---- the hybrid rule ---------------------------------------------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("leaf", [1, 8, 32])
def test_device_hybrid_equals_oracle(ctx, leaf):
    """gsofa_order_hybrid against or_order_hybrid: the same permutation and
    the same statistics on every graph of the battery."""
    for name, (b, e, c) in _cases().items():
        m = ctx.load_csr(b, e, c)
        perm, st = ctx.order_hybrid(m, leaf_size=leaf)
        ref, rst = O.order_hybrid(b, e, c, leaf=leaf)
        np.testing.assert_array_equal(perm, ref, err_msg="%s leaf %d" % (name, leaf))
        assert (st["rounds"], st["splits"], st["separator_vertices"],
                st["max_separator"]) == rst, (name, leaf, st, rst)
        m.close()


@pytest.mark.gpu
def test_device_hybrid_circuit_like_and_grid():
    """A circuit-like matrix (multilevel separators win) and an unscrambled
    3D grid (coarsening stops at once: the whole-device BFS in queue order):
    identical to the oracle, and the circuit-like fill is cut."""
    _cuda()
    from gsofatpds_b200 import Context, gen
    from gsofatpds_b200.gen import csr_to_beg_end
    _, rp, col = gen_circuit(30000)
    b, e = csr_to_beg_end(rp)
    _, grp, gcol = gen.grid_nd((32, 32, 32), "7")
    gb, ge = csr_to_beg_end(grp)
    got = {}
    with Context(0) as c:
        for name, (bb, ee, cc) in (("circuit30k", (b, e, col)), ("grid32", (gb, ge, gcol))):
            m = c.load_csr(bb, ee, cc)
            perm, st = c.order_hybrid(m, leaf_size=32)
            ref, rst = O.order_hybrid(bb, ee, cc, leaf=32)
            np.testing.assert_array_equal(perm, ref, err_msg=name)
            assert (st["rounds"], st["splits"], st["separator_vertices"],
                    st["max_separator"]) == rst, (name, st, rst)
            got[name] = perm
            m.close()
    pl, _ = O.order_nd(b, e, col, leaf=32)
    assert _fill(*permuted(b, e, col, got["circuit30k"])) < _fill(*permuted(b, e, col, pl))


# ---- the hybrid rule's oracle -------------------------------------------------------

@pytest.mark.parametrize("seed", range(12))
def test_hybrid_oracle_is_a_deterministic_permutation(seed):
    rng = np.random.default_rng(700 + seed)
    n = int(rng.integers(1, 900))
    dens = float(rng.uniform(0.0, 0.02))
    rows = [[int(j) for j in np.nonzero(rng.random(n) < dens)[0]] for _ in range(n)]
    b, e, c = _csr(rows)
    leaf = int(rng.choice([1, 8, 32]))
    p1, s1 = O.order_hybrid(b, e, c, leaf=leaf)
    assert sorted(p1.tolist()) == list(range(n))
    p2, s2 = O.order_hybrid(b, e, c, leaf=leaf)
    np.testing.assert_array_equal(p1, p2)
    assert s1 == s2


def test_hybrid_equals_level_set_when_level_sets_win():
    # a path: the level-set separator is one vertex, which no other can beat
    for n in (7, 50, 301):
        b, e, c = _path(n)
        ph, sh = O.order_hybrid(b, e, c, leaf=1)
        pl, sl = O.order_nd(b, e, c, leaf=1)
        np.testing.assert_array_equal(ph, pl)
        assert sh == sl


def test_hybrid_cuts_circuit_like_fill():
    _, rp, col = gen_circuit(12000)
    b, e = rp[:-1], rp[1:]
    pl, _ = O.order_nd(b, e, col, leaf=32)
    ph, _ = O.order_hybrid(b, e, col, leaf=32)
    f_l = _fill(*permuted(b, e, col, pl))
    f_h = _fill(*permuted(b, e, col, ph))
    assert f_h < f_l, (f_h, f_l)


def _trace_graphs():
    from gsofatpds_b200 import gen
    from gsofatpds_b200.gen import csr_to_beg_end
    rng = np.random.default_rng(41)
    out = {}
    n = 700
    rows = [[int(j) for j in np.nonzero(rng.random(n) < 0.006)[0]] for _ in range(n)]
    out["random"] = _csr(rows)
    _, rp, col = gen_circuit(6000)
    out["circuit"] = (*csr_to_beg_end(rp), col)
    out["grid_scrambled"] = _grid2d(40, 30, rng)
    return out


@pytest.mark.parametrize("name", ["random", "circuit", "grid_scrambled"])
def test_hybrid_oracle_splits_separate(name):
    """Every split the hybrid oracle makes, checked on the permutation it
    returns: the component's range holds A, B and S; no edge of A + A^T
    joins A and B; a split with both sides non-empty has a separator; a
    multilevel split is taken only when its separator is smaller than the
    level-set one and leaves both sides non-empty, and each of its separator
    vertices borders A or B; a level-set split keeps the level-set separator;
    the statistics add up.  (The 40..60 % balance bounds each refinement move,
    not the start that BFS growth gives on a weighted coarse graph, so the
    final balance is not a property to assert.)"""
    b, e, c = _trace_graphs()[name]
    n = len(b)
    perm, st, tr = O.order_hybrid_trace(b, e, c, leaf=8)
    assert sorted(perm.tolist()) == list(range(n))
    rp, adj = _sym_csr(b, e, c)
    rule_seen = set()
    for lo, k, na, nb, ns, rule, nls in tr.tolist():
        assert na + nb + ns == k and ns >= 0
        side = np.full(n, -1, np.int8)
        side[perm[lo:lo + na]] = 0
        side[perm[lo + na:lo + na + nb]] = 1
        side[perm[lo + k - ns:lo + k]] = 2
        for v in perm[lo:lo + na]:
            assert not np.any(side[adj[rp[v]:rp[v + 1]]] == 1), (name, lo, v)
        if na and nb:
            assert ns > 0
        if rule == 1:
            assert ns < nls and na > 0 and nb > 0
            for v in perm[lo + k - ns:lo + k]:
                nb_sides = side[adj[rp[v]:rp[v + 1]]]
                assert np.any((nb_sides == 0) | (nb_sides == 1)), (name, lo, v)
        else:
            assert ns == nls
        rule_seen.add(rule)
    assert st[1] == len(tr) and st[2] == int(tr[:, 4].sum()) and st[3] == int(tr[:, 4].max())
    if name == "circuit":
        assert 1 in rule_seen  # the multilevel rule wins somewhere on a small-world graph


def gen_circuit(n):
    from gsofatpds_b200 import gen
    return gen.circuit_like(n=n, target_nnz=int(5830000 * n / 659033), seed=2)


@pytest.mark.parametrize("nx,ny", [(3, 3), (4, 4), (5, 3)])
def test_hybrid_grid_known_answer(nx, ny):
    """Hand-worked: on an nx x ny 5-point grid (vertex i*ny + j) the search
    for a pseudo-peripheral start ends at a corner, the level sets from a
    corner are the anti-diagonals i + j = d, and the middle one,
    d = (nx + ny - 2) // 2, is the top separator: no multilevel separator of
    a grid this small is smaller, so the hybrid keeps it.  It is ordered
    last; the two triangles it cuts off come first."""
    b, e, c = _grid2d(nx, ny)
    n = nx * ny
    perm, _, tr = O.order_hybrid_trace(b, e, c, leaf=1)
    d = (nx + ny - 2) // 2
    diag = {i * ny + j for i in range(nx) for j in range(ny) if i + j == d}
    near = {i * ny + j for i in range(nx) for j in range(ny) if i + j < d}
    far = {i * ny + j for i in range(nx) for j in range(ny) if i + j > d}
    k = len(diag)
    assert set(perm[n - k:].tolist()) == diag
    assert len(near) == len(far)  # the middle level of these shapes halves the rest
    halves = {frozenset(perm[:len(near)].tolist()), frozenset(perm[len(near):n - k].tolist())}
    assert halves == {frozenset(near), frozenset(far)}
    lo, kk, na, nb, ns, rule, nls = tr[0].tolist()
    assert (lo, kk, ns, rule, nls) == (0, n, k, 0, k)
    pl, _ = O.order_nd(b, e, c, leaf=1)
    assert np.array_equal(perm, pl)


def test_hybrid_barbell_known_answer():
    """Hand-worked: two 5-cliques joined through one bridge vertex.  The bridge
    is the only one-vertex separator, so it is ordered last, with each clique
    whole on one side before it.  A clique cannot be split, so inside each
    the splits peel one vertex off as the separator."""
    m = 5
    rows = [[] for _ in range(2 * m + 1)]
    for a in range(m):
        for c in range(m):
            if a != c:
                rows[a].append(c)
                rows[m + 1 + a].append(m + 1 + c)
    rows[m - 1].append(m)
    rows[m] += [m - 1, m + 1]
    rows[m + 1].append(m)
    b, e, c = _csr([sorted(r) for r in rows])
    perm, _, tr = O.order_hybrid_trace(b, e, c, leaf=1)
    assert perm[-1] == m
    first, second = set(perm[:m].tolist()), set(perm[m:2 * m].tolist())
    cliques = {frozenset(range(m)), frozenset(range(m + 1, 2 * m + 1))}
    assert {frozenset(first), frozenset(second)} == cliques
    assert tr[0].tolist()[:5] == [0, 2 * m + 1, m, m, 1]
    for lo, k, na, nb, ns, rule, nls in tr[1:].tolist():
        if k > 1:
            assert ns >= 1 and min(na, nb) == 0, (lo, k, na, nb, ns)
