"""Benchmark of the fill-path symbolic factorization on B200.

One step = one full symbolic factorization (every source row, both halves
of L+U, supernode detection) of the circuit-like matrix n=659,033 with
~5.84M nonzeros (the reference's pre2 test graph shape; seeded synthetic
stand-in), max supernode size 128.

  value   fill-path GTEPS = edges_alg / device time, inputs resident in HBM
  e2e     the same metric through the C-ABI with host buffers: H2D of the
          CSR, device ingest/transpose, factorization, D2H of the per-row
          counts, every step
  roofline  traversal kernel: algorithmic bytes (8*E_alg + 16*V_alg +
          4*W_out) per launch / its CUDA-event duration vs measured HBM peak

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
N > 1 runs under torchrun as independent replicas (one matrix per GPU, no
collective on the data path); value = all ranks' edges / max-over-ranks time.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "circuit_like": "circuit-like n=659033 ~5.84M nnz, Zipf(1.2) long links, symmetric permutation, mss 128",
    "random_extra": "n=20000 diagonal+tridiagonal+3 uniform columns/row, mss 128",
    "grid3d_64": "64^3 7-point grid, nested-dissection order, mss 256",
    "circuit_like_100k": "circuit-like n=100000 ~0.89M nnz (profiling size), mss 128",
    "batch512": "512 matrices, n log-uniform [2000, 60000]: 2D 5-point ND grids and random-banded "
                "unsymmetric (bandwidth 4-32, 1-4 uniform off-band entries/row), mss 128",
    "ingest": "circuit-like n=659033 ~5.84M nnz loaded from the reference's ASCII .dat files, from a "
              "binary CSR file and from host memory (upload, padded CSR of A and A^T, checks)",
    "handoff": "supernodal block form (gsofa_result_supernodal) of the n=20000 random matrix and the "
               "64^3 ND grid, from their materialised patterns, mss 128",
    "order": "fill-reducing ordering (gsofa_order_nd, level-set nested dissection of A + A^T, and "
             "gsofa_order_hybrid, level-set or multilevel separator per split; leaf 32) "
             "of the 64^3 7-point grid under a seeded random symmetric permutation (n=262144), "
             "the n=20000 random matrix and the circuit-like n=659033 matrix",
    "steal": "the 512-matrix batch mix as 32 chunks of 16 matrices spread over the ranks by "
             "longest-first per-rank queues with work stealing; each claimed chunk is one batched "
             "launch (shape from gsofa_autotune_batch)",
    "reference_build": "the matrices the reference's own CUDA build (SpaceOptimization, unmodified, "
                       "sm_100a) was timed on: BC n=11948, n=20000 random, 64^3 ND grid, circuit-like "
                       "n=20000, banded, grid and small raw-layout patterns",
    "serve": "Poisson request stream, n log-uniform [1000, 1000000], 5-27 nnz/row: 2D 5/9-point and "
             "3D 7/27-point ND grids, random-banded unsymmetric (n capped), 40 GB budget, mss 128",
}


def make_workload(name):
    from gsofatpds_b200 import gen
    if name == "circuit_like":
        return gen.circuit_like(), 128
    if name == "random_extra":
        return gen.random_extra(20000, 3, seed=1), 128
    if name == "grid3d_64":
        return gen.grid_nd((64, 64, 64), "7"), 256
    if name == "circuit_like_100k":
        return gen.circuit_like(n=100000, target_nnz=int(5830000 * 100000 / 659033)), 128
    raise SystemExit("unknown workload " + name)


def read_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def roofline_entry(edges, vertices_alg, edges_trav, n, kernel_ms, peak, peak_kind, traffic):
    """The line's roofline object for the traversal kernel, whose bound is
    HBM (an irregular integer traversal; no tensor cores).  `achieved` is the
    DRAM bytes one launch really moves (`traffic`: ncu dram__bytes_read.sum +
    dram__bytes_write.sum of one full-size launch, from the committed
    profile of this workload) per second of the kernel's CUDA-event time, and
    frac = achieved / the measured HBM peak.  `work_equivalent` gives the
    algorithmic bytes 8 E_alg + 16 V_alg + 4 W_out of a search that expands
    every reachable vertex of every source, per second: closure reuse and
    chained starts do far less than that work, so that figure exceeds the
    peak and is not a bandwidth fraction."""
    w_out = 11 * n  # nnz_u, nz_row_u, nnz_lc, 2 digests (u64), 128-bit L-mask per row
    bytes_alg = 8 * edges + 16 * vertices_alg + 4 * w_out
    t = kernel_ms / 1e3
    roof = {"bound": "hbm", "achieved": None, "peak": peak, "unit": "GB/s", "frac": None,
            "traffic": traffic, "peak_kind": peak_kind + " (MEASURED_PEAKS hbm_gbs)",
            "kernel": "traverse_kernel", "kernel_ms": kernel_ms,
            "traffic_source": "ncu, one full-size launch (profiles/traverse_<workload>.md)",
            "inspected_edges_per_s": edges_trav / t,
            "work_equivalent": {"bytes_alg": bytes_alg, "gbs": bytes_alg / t / 1e9,
                                "note": "algorithmic bytes of an ideal label search per second; "
                                        "the kernel reuses closures, so this exceeds the peak"}}
    if traffic:
        roof["achieved"] = traffic / t / 1e9
        roof["frac"] = roof["achieved"] / peak
    return roof


def read_traffic(workload):
    """dram bytes per traversal launch from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "traverse_%s.md" % workload)
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("dram_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)),
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_sample(rp, col, seconds, seed=0):
    """Oracle (label search, all host threads) on random source rows of the
    same matrix until `seconds` of work; returns GTEPS over the sample."""
    from oracle import oracle as O
    from gsofatpds_b200 import gen
    beg, end = gen.csr_to_beg_end(rp)
    n = beg.shape[0]
    rng = np.random.default_rng(seed)
    perm = rng.permutation(n).astype(np.int32)
    done = 0
    edges = 0
    t0 = time.perf_counter()
    batch = 64
    while done < n and time.perf_counter() - t0 < seconds:
        rows = np.sort(perm[done:done + batch])
        r = O.rows(beg, end, col, rows=rows)
        edges += int(r["e_alg"].sum())
        done += rows.shape[0]
        batch = min(batch * 2, 4096)
    dt = time.perf_counter() - t0
    cores = os.cpu_count() or 1
    return dict(value=edges / dt / 1e9, unit="GTEPS", cores=cores, kind="port",
                sample="%d random source rows of %d (%.1f%%), %.3g edges_alg, %.1f s" %
                       (done, n, 100.0 * done / n, edges, dt))


def run_reference(args, rank, world):
    """Reference arm: the CPU restatement of the reference's traversal on the
    host cores (the reference's own implementation of this path exists only
    as CUDA kernels; its GPU build is not run here)."""
    if rank != 0:
        return
    if args.workload not in ("circuit_like", "random_extra", "grid3d_64", "circuit_like_100k"):
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no counterpart "
                          "of the %s workload (it factors one matrix per run)" % args.workload}),
              flush=True)
        return
    (n, rp, col), mss = make_workload(args.workload)
    per_step = max(2.0, min(20.0, 60.0 / max(args.steps + args.warmup, 1)))
    for i in range(args.warmup):
        cpu_sample(rp, col, per_step / 2, seed=100 + i)
    vals = []
    last = None
    for i in range(args.steps):
        last = cpu_sample(rp, col, per_step, seed=i)
        vals.append(last["value"])
    v = float(np.median(vals))
    cb = dict(last)
    cb["value"] = v
    line = {"impl": "reference", "metric": "fill_path_gteps", "value": v, "unit": "GTEPS",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic", "config": {"workload": WORKLOADS[args.workload], "n": n,
                                            "nnz": int(rp[-1]), "mss": mss},
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_reference_build(args, local):
    """Beside the reference's own CUDA build on the same GPU model: the fill
    detection times that the unmodified SPO binary's own timer reported
    (symbfact.cuh:2004, :2420), recorded by tests/golden/make_reference_spo.py
    in tests/golden/reference_spo.json, against this library's plain
    factorization of the same matrices (device time, CUDA events on the
    launching stream, L2 flushed, library defaults, supernodes included).
    Each matrix's fill count is checked against the reference's."""
    import torch
    from gsofatpds_b200 import Context
    from tests import reference_inputs as RI
    recs = json.load(open(os.path.join(ROOT, "tests", "golden", "reference_spo.json")))["records"]
    torch.cuda.set_device(local)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    rows = []
    with Context(local) as ctx:
        stream = torch.cuda.Stream()
        torch.cuda.set_stream(stream)
        ctx.set_stream(stream.cuda_stream)
        for label, rec in sorted(recs.items()):
            if not rec.get("ms_reference"):
                continue
            beg, end, col = RI.build(label)
            m = ctx.load_csr(beg, end, col)
            for _ in range(args.warmup):
                ctx.factor(m, max_supernode_size=128).close()
            ts, fills = [], None
            for _ in range(args.steps):
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                r = ctx.factor(m, max_supernode_size=128)
                e1.record(stream)
                torch.cuda.synchronize()
                ts.append(e0.elapsed_time(e1))
                fills = r.counts["fill_count"]
                r.close()
            m.close()
            if fills != rec["fills_reference"]:
                raise SystemExit("%s: fills %d, the reference build printed %d" %
                                 (label, fills, rec["fills_reference"]))
            ms = float(np.median(ts))
            rows.append({"input": label, "n": rec["n"], "nnz": rec["nnz"],
                         "virtual_gpus": rec["virtual_gpus"], "memory_gb": rec["memory_gb"],
                         "ms_reference_build": rec["ms_reference"], "ms": ms,
                         "speedup": rec["ms_reference"] / ms, "fills": fills})
    sp = [r["speedup"] for r in rows]
    line = {"metric": "speedup_vs_reference_build", "unit": "x",
            "value": float(np.exp(np.mean(np.log(sp)))) if sp else None,
            "value_kind": "geometric mean over the inputs of the reference build's own fill-detection "
                          "time / this library's device time",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "dtype": "int32", "data": "synthetic and the reference's BC matrix",
            "config": {"workload": WORKLOADS["reference_build"],
                       "l2": "flushed (256 MB write) before every timed step"},
            "rows": rows}
    print(json.dumps(line), flush=True)


def measure_batch(ctx, stream, steps, warmup, tune=True):
    """Config 4: the 512-matrix mix factored as one graph-captured persistent
    launch, against the same matrices factored back to back by plain calls
    (each with its own autotuned shape, and with library defaults).  Device
    time of each arm with CUDA events on `stream`, median over `steps`."""
    import torch
    from gsofatpds_b200 import gen
    mats_np = gen.batch_mix(512)
    mats = [ctx.load_rowptr(rp, col) for (_, rp, col) in mats_np]
    kw = dict(max_supernode_size=128)
    if tune:
        kw.update(ctx.autotune_batch(mats, **kw))
    batch = ctx.batch(mats, **kw)

    def timed(fn):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    # plain arm: one call per matrix, each with its own tuned shape (the
    # tuner caches per size class), or the library defaults without tuning
    base = dict(max_supernode_size=128)
    plain_kw = [dict(base, **ctx.autotune(m, **base)) for m in mats] if tune else [base] * len(mats)

    def plain():
        for m, k in zip(mats, plain_kw):
            ctx.factor(m, **k).close()

    def plain_defaults():  # what a caller gets without the tuner
        for m in mats:
            ctx.factor(m, **base).close()

    for _ in range(warmup):
        plain()
        plain_defaults()
        batch.run()
    plain_ms = [timed(plain) for _ in range(steps)]
    plain_def_ms = [timed(plain_defaults) for _ in range(steps)]
    batch_ms = [timed(batch.run) for _ in range(steps)]
    edges = sum(batch.result(i).counts["edges_alg"] for i in range(len(mats)))
    pm, bm = float(np.median(plain_ms)), float(np.median(batch_ms))
    pdm = float(np.median(plain_def_ms))
    out = {"workload": WORKLOADS["batch512"], "matrices": len(mats),
           "launch": {k: v for k, v in kw.items()},
           "ms_per_batch": bm, "matrices_per_s": len(mats) / (bm / 1e3),
           "plain_ms_per_batch": pm, "plain_matrices_per_s": len(mats) / (pm / 1e3),
           "plain_shapes": "per-matrix autotuned" if tune else "library defaults",
           "speedup_vs_plain": pm / bm,
           "plain_defaults_ms_per_batch": pdm, "speedup_vs_plain_defaults": pdm / bm,
           "edges_alg": edges, "gteps": edges / (bm / 1e3) / 1e9}
    batch.close()
    for m in mats:
        m.close()
    return out


def run_batch(args, local):
    """Batched form on its own line (see measure_batch)."""
    import torch
    from gsofatpds_b200 import Context
    torch.cuda.set_device(local)
    ctx = Context(local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    r = measure_batch(ctx, stream, args.steps, args.warmup, tune=not args.no_tune)
    line = {"metric": "matrices_per_s", "value": r["matrices_per_s"], "unit": "matrices/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_batch"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic", "config": {"workload": r["workload"], "launch": r["launch"]},
            "gpu_launches": 1}
    line.update({k: v for k, v in r.items() if k not in ("workload", "launch")})
    print(json.dumps(line), flush=True)
    ctx.close()


def run_ingest(args, local):
    """Input pipeline: the same matrix loaded onto the device from the
    reference's three ASCII files (parse + build), from one binary CSR file
    and from host arrays; each timed end to end on the host clock, median of
    the steps."""
    import tempfile
    import torch
    from gsofatpds_b200 import Context, convert_dat, gen
    torch.cuda.set_device(local)
    n, rp, col = gen.circuit_like()
    with tempfile.TemporaryDirectory() as d:
        gen.write_dat(os.path.join(d, ""), n, rp, col)
        paths = [os.path.join(d, "%s_%d.dat" % (k, n)) for k in ("colbeg", "colend", "csr")]
        binp = os.path.join(d, "m.gsofacsr")
        t0 = time.perf_counter()
        convert_dat(*paths, binp)
        convert_ms = (time.perf_counter() - t0) * 1e3
        dat_bytes = sum(os.path.getsize(p) for p in paths)
        bin_bytes = os.path.getsize(binp)
        with Context(local) as ctx:
            loaders = {"ascii": lambda: ctx.load_files(*paths),
                       "binary": lambda: ctx.load_binary(binp),
                       "memory": lambda: ctx.load_rowptr(rp, col)}
            res = {}
            for name, fn in loaders.items():
                for _ in range(args.warmup):
                    fn().close()
                ts = []
                for _ in range(args.steps):
                    t0 = time.perf_counter()
                    m = fn()
                    ts.append((time.perf_counter() - t0) * 1e3)
                    m.close()
                res[name] = float(np.median(ts))
    line = {"metric": "ingest_ms", "value": res["binary"], "unit": "ms", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["binary"],
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic", "config": {"workload": WORKLOADS["ingest"], "n": n,
                                            "nnz": int(col.shape[0])},
            "ascii_ms": res["ascii"], "binary_ms": res["binary"], "memory_ms": res["memory"],
            "convert_ms": convert_ms, "dat_bytes": dat_bytes, "binary_bytes": bin_bytes,
            "speedup_binary_vs_ascii": res["ascii"] / res["binary"]}
    print(json.dumps(line), flush=True)


def run_handoff(args, local):
    """Symbolic-to-numeric handoff: factor with the pattern materialised,
    then time building the supernodal block form on the device (first call
    of gsofa_result_supernodal, read-back of the arrays included)."""
    import ctypes
    import torch
    from gsofatpds_b200 import Context, gen
    torch.cuda.set_device(local)
    out = {}
    with Context(local) as ctx:
        for name, (n, rp, col) in [("random_extra_20k", gen.random_extra(20000, 3, seed=1)),
                                   ("grid3d_64", gen.grid_nd((64, 64, 64), "7"))]:
            m = ctx.load_rowptr(rp, col)
            ts, pairs = [], 0
            for it in range(args.warmup + args.steps):
                r = ctx.factor(m, pattern=True)
                nb, nl, nu = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
                t0 = time.perf_counter()
                rc = ctx._L.gsofa_result_supernodal(r._h, ctypes.byref(nb), ctypes.byref(nl),
                                                    ctypes.byref(nu), None, None, None, None, None)
                ms = (time.perf_counter() - t0) * 1e3
                assert rc == 0
                pairs = r.counts["nnz_l"] + r.counts["nnz_u"]
                if it >= args.warmup:
                    ts.append(ms)
                out[name] = dict(build_ms=float(np.median(ts)) if ts else None, blocks=nb.value,
                                 l_rows=nl.value, u_cols=nu.value, pattern_entries=pairs)
                r.close()
            m.close()
            out[name]["pattern_entries_per_s"] = out[name]["pattern_entries"] / (
                out[name]["build_ms"] / 1e3)
    tot = sum(v["build_ms"] for v in out.values())
    line = {"metric": "handoff_ms", "value": tot, "unit": "ms", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tot, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": WORKLOADS["handoff"]}, "cases": out}
    print(json.dumps(line), flush=True)


def run_order(args, local):
    """Ordering on the device against the oracle's single-thread ordering,
    for both rules (level-set nested dissection, gsofa_order_nd, and the
    hybrid with multilevel separators, gsofa_order_hybrid); the fill of each
    ordered matrix is measured by factoring it on the device (the 64^3 grid
    also against its coordinate-bisection ND order)."""
    import torch
    from gsofatpds_b200 import Context, gen
    from gsofatpds_b200.gen import csr_to_beg_end
    from oracle import oracle as O  # the CPU-baseline leg: timed and compared, never shipped
    torch.cuda.set_device(local)
    out = {}
    rng = np.random.default_rng(3)
    _, rp, col = gen.grid_nd((64, 64, 64), "7")
    gb, ge = csr_to_beg_end(rp)
    p = rng.permutation(len(gb)).astype(np.int32)
    ip = np.empty_like(p)
    ip[p] = np.arange(len(p), dtype=np.int32)
    deg = (ge - gb)[p]
    srp = np.zeros(len(p) + 1, np.int64)
    np.cumsum(deg, out=srp[1:])
    scol = np.concatenate([ip[col[gb[v]:ge[v]]] for v in p]).astype(np.int32)
    cases = [("grid3d_64_scrambled", srp.astype(np.int32), scol, (rp, col)),
             ("random_extra_20k",) + tuple(gen.random_extra(20000, 3, seed=1)[1:]) + (None,),
             ("circuit_like",) + tuple(gen.circuit_like()[1:]) + (None,)]
    with Context(local) as ctx:
        for name, crp, ccol, nd_ref in cases:
            m = ctx.load_rowptr(crp, ccol)
            ms, wall = [], []
            for it in range(args.warmup + args.steps):
                t0 = time.perf_counter()
                perm, st = ctx.order_nd(m)
                w = (time.perf_counter() - t0) * 1e3
                if it >= args.warmup:
                    ms.append(st["ms"])
                    wall.append(w)
            row = dict(n=int(m.n), ms_device=float(np.median(ms)), ms_call=float(np.median(wall)),
                       rounds=st["rounds"], splits=st["splits"],
                       separator_vertices=st["separator_vertices"],
                       max_separator=st["max_separator"])
            b, e = csr_to_beg_end(crp)
            t0 = time.perf_counter()
            ref, _ = O.order_nd(b, e, ccol)
            row["cpu_oracle_ms"] = (time.perf_counter() - t0) * 1e3
            row["equal_to_oracle"] = bool(np.array_equal(ref, perm))
            pm = ctx.permute(m, perm)
            r = ctx.factor(pm)
            row["fill_ordered"] = int(r.counts["fill_count"])
            row["factor_ms_ordered"] = float(r.counts["ms_device"])
            r.close()
            pm.close()
            # the hybrid rule
            hms, hwall = [], []
            for it in range(1 + max(1, min(args.steps, 3))):
                t0 = time.perf_counter()
                hperm, hst = ctx.order_hybrid(m)
                w = (time.perf_counter() - t0) * 1e3
                if it >= 1:
                    hms.append(hst["ms"])
                    hwall.append(w)
            hy = dict(ms_device=float(np.median(hms)), ms_call=float(np.median(hwall)),
                      rounds=hst["rounds"], splits=hst["splits"],
                      separator_vertices=hst["separator_vertices"],
                      max_separator=hst["max_separator"])
            t0 = time.perf_counter()
            href, _ = O.order_hybrid(b, e, ccol)
            hy["cpu_oracle_ms"] = (time.perf_counter() - t0) * 1e3
            hy["equal_to_oracle"] = bool(np.array_equal(href, hperm))
            pm = ctx.permute(m, hperm)
            r = ctx.factor(pm)
            hy["fill_ordered"] = int(r.counts["fill_count"])
            hy["factor_ms_ordered"] = float(r.counts["ms_device"])
            r.close()
            pm.close()
            row["hybrid"] = hy
            if nd_ref is not None:
                m2 = ctx.load_rowptr(*nd_ref)
                r = ctx.factor(m2)
                row["fill_coordinate_nd"] = int(r.counts["fill_count"])
                r.close()
                m2.close()
            else:
                r = ctx.factor(m)
                row["fill_given_order"] = int(r.counts["fill_count"])
                r.close()
            m.close()
            out[name] = row
    head = out["grid3d_64_scrambled"]
    line = {"metric": "ordering_ms", "value": head["ms_device"], "unit": "ms", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": head["ms_device"],
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic", "config": {"workload": WORKLOADS["order"]},
            "cpu_baseline": {"value": head["cpu_oracle_ms"], "unit": "ms", "cores": 1,
                             "kind": "port", "sample": "the same ordering by the oracle"},
            "cases": out}
    print(json.dumps(line), flush=True)


def run_steal(args, rank, world, local):
    """Replicas with per-rank request queues and work stealing: each step
    spreads the 512-matrix mix (32 chunks of 16) over the ranks; a rank
    factors its own chunks, then steals from the others' queue heads.  The
    queue heads live in a TCPStore (host fetch-and-add); the only
    collectives are the barrier and the max over ranks of the step time."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    from gsofatpds_b200 import Context, gen, replicas
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
        host = os.environ.get("MASTER_ADDR", "127.0.0.1")
        port = int(os.environ["MASTER_PORT"]) + 1
    else:
        import socket
        sk = socket.socket()
        sk.bind(("127.0.0.1", 0))
        host, port = "127.0.0.1", sk.getsockname()[1]
        sk.close()
    store = dist.TCPStore(host, port, world, rank == 0, timeout=timedelta(seconds=600))
    mats_np = gen.batch_mix(512)
    chunk = 16
    chunks = [list(range(i, min(i + chunk, len(mats_np)))) for i in range(0, len(mats_np), chunk)]
    costs = [sum(int(mats_np[j][2].shape[0]) for j in c) for c in chunks]
    queues = replicas.assign_queues(costs, world)
    ctx = Context(local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    mats = [ctx.load_rowptr(rp, col) for (_, rp, col) in mats_np]
    kw = dict(max_supernode_size=128)
    if not args.no_tune:
        kw.update(ctx.autotune_batch(mats, **kw))
    stolen = []

    def step(tag):
        sq = replicas.StealingQueue(store, rank, world, queues, prefix="bench/steal/%s" % tag)
        for c in sq:
            for r in ctx.factor_batch([mats[j] for j in chunks[c]], **kw):
                r.close()
        return sq.stolen

    for w in range(args.warmup):
        if world > 1:
            dist.barrier()
        step("w%d" % w)
    step_ms = []
    for s_ in range(args.steps):
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st = step("s%d" % s_)
        e1.record(stream)
        torch.cuda.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        stolen.append(st)
    local_ms = float(sum(step_ms))
    max_ms = replicas.max_over_ranks(local_ms, dist if world > 1 else None, "cuda")
    stolen_total = int(store.add("bench/steal/stolen", int(sum(stolen))))
    if world > 1:
        dist.barrier()
        stolen_total = int(store.add("bench/steal/stolen", 0))
    value = replicas.job_throughput(1, args.steps, len(mats), max_ms)
    if rank == 0:
        line = {"metric": "matrices_per_s", "value": value, "unit": "matrices/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": max_ms / args.steps,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
                "dtype": "int32", "data": "synthetic",
                "config": {"workload": WORKLOADS["steal"], "launch": kw,
                           "parallelism": "replicas with work stealing"},
                "chunks_stolen": stolen_total, "chunks_per_step": len(chunks)}
        print(json.dumps(line), flush=True)
    for m in mats:
        m.close()
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def _pct(xs, q):
    return float(np.percentile(np.asarray(xs, dtype=np.float64), q)) if len(xs) else None


def measure_serve(ctx, local, warmup, rate_hz, count, sampler=None):
    """Config 5: the seeded request stream (gen.SERVE_STREAM: n log-uniform in
    [1e3, 1e6], the largest requests 100^3 27-point grids) through the
    request loop, against plain calls (load + factor, one at a time), both
    measured on the host clock with host CSR in and results out:
      saturated  every request submitted at once: makespan, matrices/s and
                 latency from the common start, served vs plain back to back;
      at_rate    Poisson arrivals at rate_hz replayed in real time: each arm
                 measured as it runs (the plain arm starts a request when it
                 has arrived and the previous one is done).
    Both arms are warmed up with the stream's largest request and a few
    small ones, so that the library's workspace and memory pool have grown to
    the stream's largest matrix before timing: growing them (gigabytes of
    closure ring at n = 10^6) is a one-time cost per process, which otherwise
    lands on whichever arm meets the largest request first."""
    from gsofatpds_b200 import gen
    cfg = dict(gen.SERVE_STREAM, count=count, rate_hz=rate_hz)
    spec = gen.request_stream(**cfg)
    reqs = [(t, gen.make_request(kind, sp)) for (t, kind, sp) in spec]
    nmax = max(r[1][0] for r in reqs)
    kw = dict(max_supernode_size=128)
    largest = max(reqs, key=lambda r: r[1][0])
    warm = [largest] + [r for r in reqs if r[1][0] < 20000][:max(warmup, 1)]

    def plain_one(rp, col):
        m = ctx.load_rowptr(rp, col)
        r = ctx.factor(m, **kw)
        c = r.counts
        r.close()
        m.close()
        return c

    def plain_arm(arrivals):
        start = time.perf_counter()
        lat, counts, done = [], [], 0.0
        for t_arr, (_, rp, col) in zip(arrivals, [r[1] for r in reqs]):
            d = start + t_arr - time.perf_counter()
            if d > 0:
                time.sleep(d)
            counts.append(plain_one(rp, col))
            done = time.perf_counter() - start
            lat.append(done - t_arr)
        return lat, done - min(arrivals), counts

    def served_arm(srv, arrivals):
        start = time.perf_counter()
        tickets = []
        for t_arr, (_, rp, col) in zip(arrivals, [r[1] for r in reqs]):
            d = start + t_arr - time.perf_counter()
            if d > 0:
                time.sleep(d)
            tickets.append(srv.submit_rowptr(rp, col))
        counts = []
        for t in tickets:
            r = srv.wait(t)
            counts.append(r.counts)
            r.close()
        info = [srv.info(t) for t in tickets]
        t0 = min(i["t_submit_ms"] for i in info) - 1e3 * arrivals[0]
        lat = [(i["t_done_ms"] - (t0 + 1e3 * a)) / 1e3 for i, a in zip(info, arrivals)]
        makespan = (max(i["t_done_ms"] for i in info) - min(i["t_submit_ms"] for i in info)) / 1e3
        return lat, makespan, counts, info

    for r in warm:
        plain_one(r[1][1], r[1][2])
    k = len(reqs)
    zero = [0.0] * k
    arr = [r[0] for r in reqs]
    p_lat0, p_span0, p_counts = plain_arm(zero)
    p_lat1, p_span1, _ = plain_arm(arr)
    srv = ctx.server(max_n=nmax, budget_bytes=40 << 30, **kw)
    for r in warm:
        srv.wait(srv.submit_rowptr(r[1][1], r[1][2])).close()
    if sampler:
        sampler.start()
    s_lat0, s_span0, s_counts, _ = served_arm(srv, zero)
    s_lat1, s_span1, _, info1 = served_arm(srv, arr)
    clk = sampler.stop() if sampler else None
    st = srv.stats()
    srv.close()
    same = all(a["fill_count"] == b["fill_count"] and a["n_supernodes"] == b["n_supernodes"]
               and a["edges_alg"] == b["edges_alg"] for a, b in zip(s_counts, p_counts))
    edges = sum(c["edges_alg"] for c in s_counts)
    h2d = sum(4 * (r[1][0] * 2 + r[1][2].shape[0]) for r in reqs)
    ms = lambda x, q: _pct(x, q) * 1e3  # noqa: E731
    out = {"workload": WORKLOADS["serve"], "requests": k, "max_n": nmax,
           "largest": "100^3 27-point grid (n=1,000,000)" if nmax >= 1000000 else None,
           "banded_n_cap": cfg["max_rb_n"], "budget_gb": 40, "grid": st["grid"], "block": st["block"],
           "identical_to_plain": same, "edges_alg": edges,
           "saturated": {"matrices_per_s": k / s_span0, "plain_matrices_per_s": k / p_span0,
                         "speedup_vs_plain": p_span0 / s_span0, "makespan_s": s_span0,
                         "plain_makespan_s": p_span0, "p50_ms": ms(s_lat0, 50),
                         "p99_ms": ms(s_lat0, 99), "plain_p50_ms": ms(p_lat0, 50),
                         "plain_p99_ms": ms(p_lat0, 99), "gteps": edges / s_span0 / 1e9},
           "at_rate": {"rate_hz": rate_hz, "matrices_per_s": k / s_span1,
                       "plain_matrices_per_s": k / p_span1, "p50_ms": ms(s_lat1, 50),
                       "p99_ms": ms(s_lat1, 99), "plain_p50_ms": ms(p_lat1, 50),
                       "plain_p99_ms": ms(p_lat1, 99),
                       "run_p50_ms": _pct([i["t_done_ms"] - i["t_publish_ms"] for i in info1], 50)},
           "latency": "host clock from each request's arrival to its result; the plain arm "
                      "measured in real time, not replayed",
           "warmup": "both arms: the largest request and %d small ones" % (len(warm) - 1),
           "max_in_flight": st["max_in_flight"], "kernel_launches": st["kernel_launches"],
           "peak_bytes": st["peak_bytes"], "h2d_bytes": h2d}
    if clk:
        out["clocks"] = clk
    return out


def run_serve(args, local):
    """Serving form on its own line (see measure_serve)."""
    import torch
    from gsofatpds_b200 import Context
    torch.cuda.set_device(local)
    with Context(local) as ctx:
        r = measure_serve(ctx, local, args.warmup, args.serve_rate, args.serve_count,
                          ClockSampler(local))
    sat = r["saturated"]
    line = {"metric": "matrices_per_s", "value": sat["matrices_per_s"], "unit": "matrices/s",
            "n_gpus": 1, "steps": 1, "warmup": args.warmup, "ms_per_step": sat["makespan_s"] * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic", "config": {"workload": r["workload"], "requests": r["requests"],
                                            "rate_hz": args.serve_rate, "max_n": r["max_n"]},
            "e2e": {"value": sat["matrices_per_s"], "unit": "matrices/s",
                    "h2d_bytes_per_step": r["h2d_bytes"], "d2h_bytes_per_step": 8 * 8 * r["requests"]},
            "clocks": r.get("clocks"), "gpu_launches": r["kernel_launches"]}
    line.update({k: v for k, v in r.items() if k not in ("workload", "clocks")})
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="circuit_like", choices=sorted(WORKLOADS))
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--threads-per-source", type=int, default=0)
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner (library defaults)")
    ap.add_argument("--launch", default="",
                    help="explicit launch shape threads,chunk,ring,heavy_row (skips the autotuner)")
    ap.add_argument("--serve-count", type=int, default=48)
    ap.add_argument("--serve-rate", type=float, default=20.0, help="Poisson arrivals per second")
    ap.add_argument("--no-mix", action="store_true",
                    help="default workload: skip the batch (config 4) and serving (config 5) "
                         "measurements embedded in the line")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload == "batch512":
        run_batch(args, local)
        return
    if args.workload == "serve":
        run_serve(args, local)
        return
    if args.workload == "ingest":
        run_ingest(args, local)
        return
    if args.workload == "handoff":
        run_handoff(args, local)
        return
    if args.workload == "order":
        run_order(args, local)
        return
    if args.workload == "reference_build":
        run_reference_build(args, local)
        return
    if args.workload == "steal":
        run_steal(args, rank, world, local)
        return

    import torch
    import torch.distributed as dist
    from datetime import timedelta

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))

    from gsofatpds_b200 import Context, replicas

    (n, rp, col), mss = make_workload(args.workload)
    if world > 1:
        chk = int(np.bitwise_xor.reduce(col.astype(np.int64) * 2654435761 + np.arange(col.size)))
        if not replicas.same_input_on_all_ranks(chk, dist, "cuda"):
            raise SystemExit("ranks built different inputs")
    nnz = int(rp[-1])
    ctx = Context(local)
    stream = torch.cuda.Stream()  # events and the library share this stream
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    kw = dict(max_supernode_size=mss, threads_per_source=args.threads_per_source)

    m = ctx.load_rowptr(rp, col)
    if args.launch:
        tps, chunk, ring, heavy = (int(x) for x in args.launch.split(","))
        kw.update(threads_per_source=tps, chunk_sources=chunk, cached_closures=ring,
                  heavy_row=heavy)
    elif not args.no_tune and args.threads_per_source == 0:
        # the library's autotuner picks the launch shape (untimed, cached)
        kw.update(ctx.autotune(m, max_supernode_size=mss))
    # L2 flush buffer (> 126 MB L2) written between timed steps
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        r = ctx.factor(m, **kw)
        r.close()

    # ---- device-resident timing
    clocks = ClockSampler(local)
    barrier()
    clocks.start()
    step_ms, trav_ms = [], []
    counts = None
    for _ in range(args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = ctx.factor(m, **kw)
        e1.record(stream)
        torch.cuda.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        trav_ms.append(r.counts["ms_traverse"])
        counts = r.counts
        r.close()
    barrier()
    clk = clocks.stop()
    max_ms = replicas.max_over_ranks(float(sum(step_ms)), dist if world > 1 else None, "cuda")
    edges = counts["edges_alg"]
    value = replicas.job_throughput(world, args.steps, edges, max_ms) / 1e9

    # ---- end to end through the C-ABI with host buffers
    beg = torch.from_numpy(np.ascontiguousarray(rp[:-1])).pin_memory()
    end = torch.from_numpy(np.ascontiguousarray(rp[1:])).pin_memory()
    colp = torch.from_numpy(np.ascontiguousarray(col)).pin_memory()
    out_u = torch.empty(n, dtype=torch.int32).pin_memory()
    out_l = torch.empty(n, dtype=torch.int32).pin_memory()
    out_z = torch.empty(n, dtype=torch.int32).pin_memory()
    import ctypes
    L = ctx._L
    e2e_ms = []
    barrier()
    # warm-up iterations too: the first calls through the C-ABI grow the
    # context's workspace and the allocator's pool
    for it in range(args.warmup + args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        mh = ctypes.c_void_p()
        ctx._check(L.gsofa_load_csr(ctx.handle, n, nnz, ctypes.c_void_p(beg.data_ptr()),
                                    ctypes.c_void_p(end.data_ptr()), ctypes.c_void_p(colp.data_ptr()),
                                    ctypes.byref(mh)), "load_csr")
        o = ctx.opts(**kw)
        rh = ctypes.c_void_p()
        ctx._check(L.gsofa_factor_symbolic(ctx.handle, mh, ctypes.byref(o), ctypes.byref(rh)), "factor")
        ctx._check(L.gsofa_result_row_counts(rh, ctypes.c_void_p(out_u.data_ptr()),
                                             ctypes.c_void_p(out_z.data_ptr()),
                                             ctypes.c_void_p(out_l.data_ptr()), None), "row_counts")
        e1.record(stream)
        torch.cuda.synchronize()
        if it >= args.warmup:
            e2e_ms.append(e0.elapsed_time(e1))
        L.gsofa_result_destroy(rh)
        L.gsofa_matrix_destroy(mh)
    barrier()
    e2e_max = replicas.max_over_ranks(float(sum(e2e_ms)), dist if world > 1 else None, "cuda")
    e2e_value = replicas.job_throughput(world, args.steps, edges, e2e_max) / 1e9
    h2d = (2 * n + nnz) * 4
    d2h = 3 * n * 4

    if rank == 0:
        peak, peak_kind = read_peaks()
        trav = float(np.mean(trav_ms))
        roof = roofline_entry(edges, counts["vertices_alg"], counts["edges_traversed"], n, trav,
                              peak, peak_kind, read_traffic(args.workload))
        line = {"metric": "fill_path_gteps", "value": value, "unit": "GTEPS", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": max_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
                "config": {"workload": WORKLOADS[args.workload], "n": n, "nnz": nnz, "mss": mss,
                           "l2": "flushed (256 MB write) before every timed step",
                           "launch": {k: v for k, v in kw.items() if k != "max_supernode_size"},
                           "parallelism": "replicas" if world > 1 else "single"},
                "ms_per_matrix": max_ms / args.steps, "matrices_per_s": world * args.steps / (max_ms / 1e3),
                "fill_count": counts["fill_count"], "nnz_lu": counts["nnz_lu"],
                "n_supernodes": counts["n_supernodes"], "edges_alg": edges,
                "value_kind": "work-equivalent GTEPS: edges_alg (the reference's traversed-edge "
                              "count without re-expansions) per second of device time",
                "inspected_gteps": counts["edges_traversed"] / (max_ms / args.steps / 1e3) / 1e9,
                "sources_chained": counts["sources_chained"],
                "roofline": roof,
                "e2e": {"value": e2e_value, "unit": "GTEPS", "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h, "ms_per_step": float(np.mean(e2e_ms))},
                "clocks": clk,
                "gpu_launches": 2 * args.steps}
        if world == 1 and args.cpu_seconds > 0:
            line["cpu_baseline"] = cpu_sample(rp, col, args.cpu_seconds)
        if world == 1 and args.workload == "circuit_like" and not args.no_mix:
            # the batched (config 4) and served (config 5) forms against plain
            # calls, measured in the same run
            line["batch"] = measure_batch(ctx, stream, args.steps, args.warmup,
                                          tune=not args.no_tune)
            line["serve"] = measure_serve(ctx, local, args.warmup, args.serve_rate,
                                          args.serve_count)
        print(json.dumps(line), flush=True)

    m.close()
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
