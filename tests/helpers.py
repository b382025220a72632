"""Shared test helpers: small seeded patterns in the reference's input shapes
and an independent definitional check of the fill structure."""
import numpy as np


def symbolic_elimination(n, pattern):
    """Structure of L+U by symbolic Gaussian elimination without pivoting:
    eliminating vertex k adds (i,j) for every i,j > k with (i,k) and (k,j)
    present.  Equivalent to the fill-path rule; O(n^3), tiny n only.
    Returns a boolean n x n matrix (diagonal included)."""
    F = np.zeros((n, n), dtype=bool)
    for i, row in enumerate(pattern):
        F[i, list(row)] = True
    np.fill_diagonal(F, True)
    for k in range(n):
        rows = np.nonzero(F[k + 1:, k])[0] + k + 1
        cols = np.nonzero(F[k, k + 1:])[0] + k + 1
        if rows.size and cols.size:
            F[np.ix_(rows, cols)] = True
    return F


def scrambled_csr(rng, pattern, shuffle_rows=True, dup_prob=0.0):
    """Reference-style CSR: rows stored in a random order (non-contiguous
    begin/end), columns unsorted, optional duplicate entries."""
    n = len(pattern)
    order = rng.permutation(n) if shuffle_rows else np.arange(n)
    beg = np.zeros(n, np.int32)
    end = np.zeros(n, np.int32)
    col = []
    for i in order:
        r = list(rng.permutation(sorted(pattern[i])))
        if dup_prob and r:
            r += [c for c in r if rng.random() < dup_prob]
        beg[i] = len(col)
        col.extend(r)
        end[i] = len(col)
    return beg, end, np.array(col, dtype=np.int32)


def random_pattern(rng, n, density, diag=True):
    A = rng.random((n, n)) < density
    if diag:
        np.fill_diagonal(A, True)
    return [set(np.nonzero(A[i])[0].tolist()) for i in range(n)]


def load_bc():
    import os
    d = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "bc_11948.npz")
    return np.load(d)
