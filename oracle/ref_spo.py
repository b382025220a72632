"""The reference's own CUDA build (SpaceOptimization, "SPO"), run as a second
checker of the fill counts.  TEST INFRASTRUCTURE ONLY: used by
tests/golden/make_reference_spo.py (on a GPU machine) to record the
reference's answers, never by the product.

The binary oracle/_ref/spo_symbfact is compiled unmodified from the
reference's sources (oracle/Makefile, target `ref`: SpaceOptimization/main.cu,
which includes symbfact.cuh, for sm_100a).  It prints "Total Number of
fill-ins detected: N" (symbfact.cuh:2526).

Before any run, `check` restates SPO's own sizing on the host and refuses an
input whose device writes the binary does not bound by itself:
  * concurrency: Compute_Src_group_original (symbfact.cuh:1101-1119) and the
    per-group reduction Get_Max_id_efficent_N_SourceGroup (:1465-1507,
    threshold max_id_fraction * pool, :57, :1683-1687), carried across
    groups and virtual GPUs exactly as the host loop does (:2042, :2415);
  * the pool split (:2079-2124): labels, fill markers, four queues of
    real_allocation words each, and the assert of :2124;
  * the 32-bit label offset s*(2(first+1)+(s-1)V)/2 (:661, :695, :922) and
    the fill offset s*n (:696, :924) must not wrap, and every label index
    (offset + vertex <= source) must stay inside the label region;
  * the seeding kernel (:639-721) appends the source rows' lower neighbours
    to the queue without a bound check: their total per group must fit
    real_allocation (the level kernel checks its own appends, :1030);
  * the row files are read in loops of E iterations into n-entry arrays
    (:1609-1640; fscanf stops at end of file), so E >= n is required;
  * the pinned host buffers, 4 * C * n words (:1871), must fit an int
    product and the host budget.
Only inputs and parameters that pass are run; the runs use one virtual GPU
and a pool large enough that no frontier is spilled to the host.
"""
import math
import os
import re
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BINARY = os.path.join(HERE, "_ref", "spo_symbfact")
MAX_ID_FRACTION = 0.999       # symbfact.cuh:57
REAL_ALLOCATION_FACTOR = 1.1  # symbfact.cuh:77


def compute_src_group_original(n):
    """symbfact.cuh:1101-1119 (log_2 via natural logs, truncated)."""
    temp = 3758096384 / float(5 * n)
    if temp > n:
        temp = float(int(math.log(n / 2.0) / 0.693147180559945309417))
    else:
        temp = float(int(math.log(temp) / 0.693147180559945309417))
    return int(2.0 ** temp)


def max_id_group(c, end_group, v, begin, threshold, n):
    """symbfact.cuh:1465-1507: shrink the group until labels + markers fit;
    returns (C, label words).  first_term is an unsigned int there."""
    while True:
        first_term = ((begin + 1 + v) + (end_group + 1)) & 0xFFFFFFFF
        need = (first_term * c) // 2 + c * n
        if need <= threshold:
            return c, (first_term * c) // 2
        c -= 1
        if c <= 0:
            return 0, 0
        end_group = begin + c * v


def check(beg, end, col, virtual_gpus=1, memory_gb=4.0, host_budget=32 << 30):
    """None when the reference binary bounds every device write for this
    input and these parameters, else the reason it would not."""
    beg = np.asarray(beg, np.int64)
    end = np.asarray(end, np.int64)
    n = int(beg.shape[0])
    nnz = int(np.asarray(col).shape[0])
    if n < 2:
        return "n < 2"
    if nnz < n:
        return "fewer entries than rows: the row files would be read short (:1609-1640)"
    if nnz >= 2 ** 31:
        return "nnz does not fit int"
    deg = end - beg
    if np.any(deg < 0) or np.any(beg < 0) or np.any(end > nnz):
        return "row interval outside the entry array"
    colv = np.asarray(col, np.int64)
    if colv.size and (colv.min() < 0 or colv.max() >= n):
        return "column id outside [0, n)"
    v = int(virtual_gpus)
    total = int(memory_gb * 1024 * 1024 * 1024) // 4          # :1683
    threshold = int(MAX_ID_FRACTION * total)                   # :1687
    c0 = compute_src_group_original(n)
    if c0 * n >= 2 ** 31:
        return "pinned buffer size C*n overflows int (:1871)"
    if 16 * c0 * n > host_budget:
        return "pinned host buffers above the host budget"
    c = c0
    for g in range(v):
        begin = 0
        while begin < n:
            end_group = begin + c * v
            c, maxid = max_id_group(c, end_group, v, begin, threshold, n)
            if c <= 0:
                return "no group size fits the pool"
            fill = c * n
            real = (total - (maxid + fill)) // 4
            if real < 1 or maxid + fill + 4 * real > total:
                return "pool split fails (:2124)"
            first = begin + g
            s_max = c - 1
            prod = s_max * (2 * (first + 1) + (s_max - 1) * v)
            if prod >= 2 ** 32:
                return "32-bit label offset wraps (:661)"
            if s_max * n >= 2 ** 31:
                return "int fill offset wraps (:924)"
            srcs = np.arange(c, dtype=np.int64) * v + g + begin
            valid = srcs < n
            k = np.arange(c, dtype=np.int64)
            off = (k * (2 * (first + 1) + (k - 1) * v)) // 2
            if np.any(off[valid] + srcs[valid] >= maxid):
                return "label index outside the label region"
            if int(deg[srcs[valid]].sum()) > real - 1:
                return "seeding queue above real_allocation"
            begin += c * v
    return None


def write_dat(d, beg, end, col):
    """The reference's three ASCII files in directory d; returns the paths."""
    n = len(beg)
    pb, pe, pc = (os.path.join(d, "%s_%d.dat" % (k, n)) for k in ("colbeg", "colend", "csr"))
    with open(pc, "w") as f:
        f.write("%d\n%d\n" % (len(col), n))
        f.write(" ".join(map(str, np.asarray(col).tolist())) + "\n")
    with open(pb, "w") as f:
        f.write(" ".join(map(str, np.asarray(beg).tolist())) + "\n")
    with open(pe, "w") as f:
        f.write(" ".join(map(str, np.asarray(end).tolist())) + "\n")
    return pb, pe, pc


def run(beg, end, col, virtual_gpus=1, memory_gb=4.0, timeout=600):
    """Runs the reference binary (after `check`) in a scratch directory (it
    appends log files to its working directory); returns (fills, stdout)."""
    why = check(beg, end, col, virtual_gpus, memory_gb)
    if why:
        raise ValueError("refused: " + why)
    if not os.path.exists(BINARY):
        raise FileNotFoundError(BINARY + " (build it with make -C oracle ref)")
    with tempfile.TemporaryDirectory() as d:
        pb, pe, pc = write_dat(d, beg, end, col)
        out = subprocess.run([BINARY, pb, pe, pc, str(int(virtual_gpus)), repr(float(memory_gb))],
                             cwd=d, capture_output=True, text=True, timeout=timeout)
    if out.returncode != 0:
        raise RuntimeError("reference exited %d: %s" % (out.returncode, out.stdout[-2000:]))
    m = re.search(r"Total Number of fill-ins detected: (\d+)", out.stdout)
    if not m:
        raise RuntimeError("no fill count in the reference's output")
    return int(m.group(1)), out.stdout


def min_memory_gb(beg, end, col):
    """Smallest whole-GB pool with one virtual GPU whose queues hold the
    largest group's worst case (C*n entries plus the 10 % slack), so that no
    frontier is spilled to the host."""
    n = len(beg)
    c = compute_src_group_original(n)
    words = c * c // 2 + c * n + 4 * REAL_ALLOCATION_FACTOR * c * n
    return max(1, int(math.ceil(words * 4 / (1024 ** 3) / MAX_ID_FRACTION)) + 1)
