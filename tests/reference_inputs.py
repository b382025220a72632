"""Matrices on which the reference's own SPO build was run
(tests/golden/make_reference_spo.py) and on which the oracle is checked
against its answers (tests/test_reference_spo.py).  Each is rebuilt from a
seed; `build(label)` returns (row_begin, row_end, col) in the reference's
layout.

  bc_264        the reference's bundled BC matrix with the reference's own
                logged parameters (264 virtual GPUs, 5 GB)
  bc            BC again with one virtual GPU
  random_extra  n=20,000 + 3 uniform columns/row (the plain-call benchmark)
  grid3d_64     64^3 7-point grid in nested-dissection order
  circuit_20k   circuit-like, n=20,000
  banded_3000   random-banded unsymmetric, n=3,000
  grid2d_45     45x45 5-point grid in nested-dissection order
  rand_<k>      small random patterns in the reference's raw layout: rows
                stored out of order, columns unsorted, some duplicates
"""
import numpy as np

INPUTS = {
    "bc_264": dict(virtual_gpus=264, memory_gb=5.0),
    "bc": dict(),
    "random_extra": dict(),
    "grid3d_64": dict(timeout=1500),
    "circuit_20k": dict(),
    "banded_3000": dict(),
    "grid2d_45": dict(),
}
for _k in range(8):
    INPUTS["rand_%d" % _k] = dict()


def build(label):
    from gsofatpds_b200 import gen
    from tests.helpers import load_bc, random_pattern, scrambled_csr
    if label.startswith("bc"):
        z = load_bc()
        return z["beg"], z["end"], z["col"]
    if label.startswith("rand_"):
        k = int(label.split("_")[1])
        rng = np.random.default_rng(500 + k)
        n = int(rng.integers(40, 400))
        pat = random_pattern(rng, n, float(rng.uniform(0.01, 0.06)), diag=True)
        return scrambled_csr(rng, pat, dup_prob=0.2 if k % 2 else 0.0)
    if label == "random_extra":
        n, rp, col = gen.random_extra(20000, 3, seed=1)
    elif label == "grid3d_64":
        n, rp, col = gen.grid_nd((64, 64, 64), "7")
    elif label == "circuit_20k":
        n, rp, col = gen.circuit_like(n=20000, target_nnz=int(5830000 * 20000 / 659033), seed=7)
    elif label == "banded_3000":
        n, rp, col = gen.random_banded(3000, bw=6, extra=2, seed=13)
    elif label == "grid2d_45":
        n, rp, col = gen.grid_nd((45, 45), "5")
    else:
        raise KeyError(label)
    beg, end = gen.csr_to_beg_end(rp)
    return beg, end, col
