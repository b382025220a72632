"""Generates the committed golden fixtures (run in a checkout that has the
reference tree; the fixtures themselves travel without it).

  bc_11948.npz   the reference's bundled BC matrix (SpaceOptimization/dataset/
                 {colbeg,colend,csr}_11948.dat) as int32 beg/end/col arrays,
                 plus the oracle's per-row answers (nnzL, nnzU, nzU_ref,
                 digests, lback, supernode flags for mss=128)
  golden.json    pinned totals: the reference's logged fill count (980,136,
                 SpaceOptimization/with_supernodes/
                 space_optimization_log_1_264_GPU_warp_centric.dat:2) and the
                 oracle's derived totals

Usage: python tests/golden/make_golden.py /path/to/gSoFaTPDS
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402

PUBLISHED_BC_FILLS = 980136


def main():
    if len(sys.argv) != 2:
        raise SystemExit("usage: make_golden.py /path/to/gSoFaTPDS (the reference checkout)")
    ref = sys.argv[1]
    d = os.path.join(ref, "SpaceOptimization", "dataset")
    beg, end, col = O.read_dat(os.path.join(d, "colbeg_11948.dat"),
                               os.path.join(d, "colend_11948.dat"),
                               os.path.join(d, "csr_11948.dat"))
    r = O.rows(beg, end, col)
    if int(r["fills"].sum()) != PUBLISHED_BC_FILLS:
        raise SystemExit("oracle disagrees with the reference's logged fill count")
    nsup, flags = O.supernodes(r["nzU_ref"], r["lback"], 128)
    tb, te, tc = O.transpose(beg, end, col)
    rt = O.rows(tb, te, tc)  # U rows of A^T = L columns of A
    np.savez_compressed(os.path.join(HERE, "bc_11948.npz"), beg=beg, end=end, col=col,
                        nnzL=r["nnzL"], nnzU=r["nnzU"], nzU_ref=r["nzU_ref"],
                        digL=r["digL"], digU=r["digU"], lback=r["lback"],
                        nnzLcol=rt["nnzU"], digLcol=rt["digU"], sflags=flags)
    gold = {
        "bc_11948": {
            "n": int(beg.shape[0]), "nnz": int(col.shape[0]),
            "fill_count": int(r["fills"].sum()),
            "fill_count_source": "reference log space_optimization_log_1_264_GPU_warp_centric.dat:2",
            "nnz_l": int(r["nnzL"].sum()), "nnz_u": int(r["nnzU"].sum()),
            "edges_alg": int(r["e_alg"].sum()), "vertices_alg": int(r["v_alg"].sum()),
            "supernodes_mss128_printed": nsup + 1,
            "supernodes_source": "oracle restatement of the SOA kernel rule (not logged by the reference)",
        }
    }
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(gold, f, indent=1)
    print(json.dumps(gold, indent=1))


if __name__ == "__main__":
    main()
