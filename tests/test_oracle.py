"""The CPU oracle pinned: against the reference's logged BC answer, against
the committed golden vectors, and against symbolic Gaussian elimination."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import load_bc, random_pattern, scrambled_csr, symbolic_elimination

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))


def test_bc_fill_count_matches_reference_log():
    z = load_bc()
    r = O.rows(z["beg"], z["end"], z["col"])
    # SpaceOptimization/with_supernodes/space_optimization_log_1_264_GPU_warp_centric.dat:2
    assert int(r["fills"].sum()) == 980136
    g = GOLD["bc_11948"]
    assert int(r["nnzL"].sum()) == g["nnz_l"] and int(r["nnzU"].sum()) == g["nnz_u"]
    assert int(r["e_alg"].sum()) == g["edges_alg"]
    assert int(r["v_alg"].sum()) == g["vertices_alg"]


def test_bc_golden_vectors():
    z = load_bc()
    r = O.rows(z["beg"], z["end"], z["col"])
    for k in ("nnzL", "nnzU", "nzU_ref", "digL", "digU", "lback"):
        np.testing.assert_array_equal(r[k], z[k], err_msg=k)
    nsup, flags = O.supernodes(r["nzU_ref"], r["lback"], 128)
    assert nsup + 1 == GOLD["bc_11948"]["supernodes_mss128_printed"]
    np.testing.assert_array_equal(flags, z["sflags"])


def test_bc_sampled_rows_equal_full_run():
    z = load_bc()
    full = O.rows(z["beg"], z["end"], z["col"])
    rows = np.array([0, 1, 17, 5000, 11946, 11947], np.int32)
    part = O.rows(z["beg"], z["end"], z["col"], rows=rows)
    for k in ("nnzL", "nnzU", "digU", "fills", "e_alg"):
        np.testing.assert_array_equal(part[k], full[k][rows])


@pytest.mark.parametrize("seed", range(12))
def test_oracle_equals_symbolic_elimination(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 48))
    pat = random_pattern(rng, n, rng.uniform(0.02, 0.25), diag=bool(seed % 3))
    beg, end, col = scrambled_csr(rng, pat, dup_prob=0.2 if seed % 4 == 0 else 0.0)
    r = O.rows(beg, end, col, pattern=True)
    F = symbolic_elimination(n, pat)
    for s in range(n):
        L = list(r["Lcols"][r["Lptr"][s]:r["Lptr"][s + 1]])
        U = list(r["Ucols"][r["Uptr"][s]:r["Uptr"][s + 1]])
        assert L == [j for j in range(s) if F[s, j]], (seed, s)
        assert U == [j for j in range(s + 1, n) if F[s, j]], (seed, s)
    orig = sum(len(p - {i}) for i, p in enumerate(pat))
    assert int(r["fills"].sum()) == int(F.sum()) - n - orig


def test_nz_row_u_counts_duplicates_like_reference():
    # row 0 holds column 2 twice: the reference's seeding counts CSR entries
    # above the diagonal with multiplicity (SOA :895-903)
    beg = np.array([0, 3, 4], np.int32)
    end = np.array([3, 4, 5], np.int32)
    col = np.array([0, 2, 2, 1, 2], np.int32)
    r = O.rows(beg, end, col)
    assert r["nnzU"][0] == 1 and r["nzU_ref"][0] == 2


def test_empty_and_single():
    r = O.rows(np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0, np.int32))
    assert r["fills"].shape == (0,)
    r = O.rows(np.array([0], np.int32), np.array([0], np.int32), np.zeros(0, np.int32))
    assert int(r["nnzL"][0]) == 0 and int(r["nnzU"][0]) == 0


def test_invalid_column_rejected():
    with pytest.raises(ValueError):
        O.rows(np.array([0], np.int32), np.array([1], np.int32), np.array([5], np.int32))


def _lback_from_pattern(F):
    n = F.shape[0]
    lb = np.zeros((n, 4), np.uint32)
    for r in range(n):
        for j in range(min(r, 128)):
            if F[r, r - 1 - j]:
                lb[r, j >> 5] |= np.uint32(1 << (j & 31))
    return lb


def test_supernode_rule_hand_case():
    # nzU = 5,4,3,9,8 with mss 8: rows 0 (chunk head) and 3 (nzU jump) start;
    # rows 1,2,4 pass through; L(2,0) missing -> one split at row 2
    nzU = np.array([5, 4, 3, 9, 8], np.int32)
    F = np.eye(5, dtype=bool)
    F[1, 0] = True      # L(1,0)
    F[4, 3] = True      # L(4,3)
    c, flags = O.supernodes(nzU, _lback_from_pattern(F), 8)
    assert list(flags) == [1, 0, 2, 1, 0] and c == 3


def test_supernode_split_keeps_first_row():
    # after a failed test at row 2, row 3 is still compared with row 0
    nzU = np.array([9, 8, 7, 6], np.int32)
    F = np.eye(4, dtype=bool)
    F[1, 0] = True
    F[3, 0] = True      # L(3,0) present, L(3,2) absent
    c, flags = O.supernodes(nzU, _lback_from_pattern(F), 16)
    assert list(flags) == [1, 0, 2, 0] and c == 2


def test_supernode_forced_start_every_128_rows():
    # a block of 128 threads handles chunk offsets t, t+128, ...; thread 0
    # always opens a supernode, so offset 128 of a 256-row chunk is a start
    n = 300
    nzU = np.arange(n, 0, -1).astype(np.int32)
    F = np.eye(n, dtype=bool)
    for r in range(1, n):
        F[r, :r] = True
    c, flags = O.supernodes(nzU, _lback_from_pattern(F), 256)
    assert flags[0] == 1 and flags[128] == 1 and flags[256] == 1
    assert c == 3 and flags.sum() == 3


def test_transposed_reachability_equals_labels():
    # the GPU kernels' formulation: U row s = BFS from s in A through ids < s;
    # L column m = BFS from m in A^T through ids < m
    rng = np.random.default_rng(7)
    for _ in range(6):
        n = int(rng.integers(2, 40))
        pat = random_pattern(rng, n, 0.12)
        beg, end, col = scrambled_csr(rng, pat)
        r = O.rows(beg, end, col, pattern=True)
        tb, te, tc = O.transpose(beg, end, col)
        rt = O.rows(tb, te, tc, pattern=True)
        # U rows of A^T are the L columns of A
        Lcol = [[] for _ in range(n)]
        for s in range(n):
            for m in r["Lcols"][r["Lptr"][s]:r["Lptr"][s + 1]]:
                Lcol[m].append(s)
        for m in range(n):
            assert sorted(Lcol[m]) == list(rt["Ucols"][rt["Uptr"][m]:rt["Uptr"][m + 1]])


@pytest.mark.parametrize("seed", range(4))
def test_digest_definitions(seed):
    """U-row digests sum splitmix64((w << 32) | mask) over the row's non-zero
    32-column words; L-row digests sum splitmix64(column) over its columns."""
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(40, 200))
    pat = random_pattern(rng, n, rng.uniform(0.02, 0.1), diag=True)
    beg, end, col = scrambled_csr(rng, pat)
    r = O.rows(beg, end, col, pattern=True)
    M = (1 << 64) - 1
    for s in range(n):
        U = r["Ucols"][r["Uptr"][s]:r["Uptr"][s + 1]]
        words = {}
        for c in U:
            words[int(c) >> 5] = words.get(int(c) >> 5, 0) | (1 << (int(c) & 31))
        du = sum(O.mix64((w << 32) | m) for w, m in words.items()) & M
        assert du == int(r["digU"][s]), (seed, s)
        L = r["Lcols"][r["Lptr"][s]:r["Lptr"][s + 1]]
        dl = sum(O.mix64(int(c)) for c in L) & M
        assert dl == int(r["digL"][s]), (seed, s)


@pytest.mark.parametrize("seed", range(8))
def test_supernodal_form_reference_equals_elimination(seed):
    """The restatement the GPU handoff test compares against
    (`_supernodal_reference`: per-block unions from the oracle's patterns)
    equals the same unions read off symbolic Gaussian elimination."""
    from tests.test_gpu_parity import _supernodal_reference
    rng = np.random.default_rng(300 + seed)
    n = int(rng.integers(2, 60))
    pat = random_pattern(rng, n, float(rng.uniform(0.02, 0.12)))
    beg, end, col = scrambled_csr(rng, pat)
    r = O.rows(beg, end, col, pattern=True)
    mss = [4, 8, 128][seed % 3]
    _, flags = O.supernodes(r["nzU_ref"], r["lback"], mss)
    got = _supernodal_reference(n, r, flags)
    F = symbolic_elimination(n, pat)
    starts = list(np.nonzero(flags)[0]) + [n]
    np.testing.assert_array_equal(got["block_start"], starts)
    for k in range(len(starts) - 1):
        f, l = starts[k], starts[k + 1]
        rows = sorted({i for i in range(l, n) for c in range(f, l) if F[i, c]})
        cols = sorted({j for j in range(l, n) for i in range(f, l) if F[i, j]})
        assert got["lrows"][got["lptr"][k]:got["lptr"][k + 1]] == rows, (seed, k)
        assert got["ucols"][got["uptr"][k]:got["uptr"][k + 1]] == cols, (seed, k)
