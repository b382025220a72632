"""The reference's own SOA supernode kernel, run as a second checker of the
supernode rule.  TEST INFRASTRUCTURE ONLY: used by
tests/golden/make_reference_soa.py (on a GPU machine), never by the product.

oracle/_ref/soa_supernodes (oracle/Makefile, target `ref`) is our harness
around the reference's unmodified kernel warpcentric_local_detection_test
(gSoFa_SOAComparison/symbfact_warp_centric_new_scheduling.cuh:1790-2123),
launched as the reference launches it, <<<1,128>>> with (mss + 1) ints of
shared memory, one chunk of max_supernode_size rows per launch.  The kernel
is one block, so it has no inter-block wait, and every array it indexes is
sized by the harness for the chunk it reads (its rows' counters, mss x n
markers, mss pass-through flags).

The inputs are the oracle's per-row nz_row_U counters and L rows (the fill
structure, which the reference's SPO build already confirms); the kernel's
count of detected supernodes (the reference prints it + 1, :3549) and its
starts per chunk must equal the oracle's restatement of the rule
(or_supernodes).
"""
import os
import re
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BINARY = os.path.join(HERE, "_ref", "soa_supernodes")


def write_input(path, nz_row_u, lptr, lcols, mss):
    n = int(np.asarray(nz_row_u).shape[0])
    with open(path, "wb") as f:
        np.array([n, mss], np.int32).tofile(f)
        np.ascontiguousarray(nz_row_u, np.int32).tofile(f)
        np.ascontiguousarray(lptr, np.int64).tofile(f)
        np.ascontiguousarray(lcols, np.int32).tofile(f)


def run(nz_row_u, lptr, lcols, mss, timeout=600):
    """Returns (detected supernodes, starts per chunk) from the reference
    kernel."""
    if not os.path.exists(BINARY):
        raise FileNotFoundError(BINARY + " (build it with make -C oracle ref)")
    if not 1 <= mss <= 1024:
        raise ValueError("max_supernode_size outside 1..1024")
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "in.bin")
        write_input(p, nz_row_u, lptr, lcols, mss)
        out = subprocess.run([BINARY, p], capture_output=True, text=True, timeout=timeout)
    if out.returncode != 0:
        raise RuntimeError("harness exited %d: %s" % (out.returncode, out.stderr[-2000:]))
    m = re.search(r"Nsup_detected (\d+)", out.stdout)
    if not m:
        raise RuntimeError("no count in the harness output")
    starts = [int(x) for x in re.findall(r"chunk_starts \d+ (\d+)", out.stdout)]
    return int(m.group(1)), starts
