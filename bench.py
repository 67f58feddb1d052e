#!/usr/bin/env python
"""Benchmark of the all-vs-all scoring path on B200 (one JSON line on rank 0).

Headline workload (the one the metric is quoted on): gap-block ``score_matrix``, 1,000 query x
10,000 reference CDR3-like junctions ('CASS' + uniform middle + 'F', length uniform 10-20; numpy
PCG64 seed 1 for queries, seed 0 for refs), BLOSUM62 penalties, gap_open 8, gap_extend 1,
central_prior(21); int32 output bit-identical to seqtree's C++.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]
                    [--no-suite]

At N = 1 the headline line also carries, under ``workloads``, one complete line for each other
named configuration (unless ``--no-suite``): ``hamming`` / ``levenshtein`` (20,000 x 20,000 ACGT),
``nw`` / ``sw`` (4,096 x 4,096 proteins, distance matrix), ``sparse`` / ``sparse_structural``
(100,000 x 1,000,000 CDR3-like, thresholded at max_penalty 24 into CSR rows; the dense matrix would
be 400 GB) and ``learned`` (1,000,000 x 1,000,000, learned proposal + exact rescore).
``--workload int_peak`` prints the measured instruction peaks alone.

* ``value``: pairs/s with inputs resident in HBM (device sets) and the result written to HBM,
  device-timed with CUDA events on the launching stream; the L2 is flushed (a 256 MiB write)
  between timed steps.  N > 1 (torchrun): every rank scores its own query block (weak scaling,
  no data-path collective); value = all ranks' pairs / max over ranks of the device time.
* ``e2e``: the same metric through the public API (``seqtree_b200.gapblock.score_matrix`` etc. on
  Python lists): packing, host->device copy, kernels and the device->host copy of the result.
* ``cpu_baseline``: the reference's own C++ (``oracle/_ref``) on the host cores, rank 0, N = 1, on
  evenly spaced query rows; those rows of the GPU result are compared with it (``parity``).
* ``kernel_roofline``: the dominant kernel against its own bound, with the instruction peaks
  measured in this process (``int_peaks``).
* ``--impl reference``: times that CPU implementation alone, on the same workloads; it imports
  nothing that loads this library.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from seqtree_b200 import workloads as W  # noqa: E402  (numpy only: loads no compiled code)

SUITE = ["hamming", "levenshtein", "nw", "sw", "sparse", "sparse_structural", "learned"]
PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0
FALLBACK_BF16_TFLOPS = 1590.0
L2_NOTE = ("GPU arm: L2 flushed between timed steps (256 MiB write); CPU reference arm: "
           "not applicable")
# DRAM bytes (read + write) per launch of the dominant kernel on the named workload, from the ncu
# captures summarised in profiles/ (None until captured).
TRAFFIC: dict[str, float | None] = {
    "gapblock": 1.92e6,     # 1.88 MB read + 0.03 MB write (the result stays in L2)
    "hamming": 1.31e9,      # 262 MB per 4,000 rows, scaled to 20,000 rows
    "levenshtein": 1.03e9,  # 102.5 MB per 2,000 rows, scaled to 20,000 rows
    "align": 1.05e6,        # one row-bucket launch of the wavefront kernel
}


# ----------------------------------------------------------------------------- workloads ----
def make_workload(name: str, rank: int, nq: int | None = None, nr: int | None = None):
    """The named workload (queries, refs, kind, config, metric); nq / nr shrink it for
    profiling captures of the same kernels on a smaller case."""
    w = _make_workload(name, rank)
    if w.pop("_lazy_strings", False):  # code arrays first; strings for the CPU reference
        if nq is not None:
            w["q_codes"], w["q_lens"] = w["q_codes"][:nq], w["q_lens"][:nq]
        if nr is not None:
            w["r_codes"], w["r_lens"] = w["r_codes"][:nr], w["r_lens"][:nr]
        w["queries"] = W.codes_to_strings(w["q_codes"], w["q_lens"])
        w["refs"] = W.codes_to_strings(w["r_codes"], w["r_lens"])
    if nq is not None or nr is not None:
        w["queries"] = w["queries"][:nq] if nq is not None else w["queries"]
        w["refs"] = w["refs"][:nr] if nr is not None else w["refs"]
        w["config"] = dict(w["config"], queries=len(w["queries"]), refs=len(w["refs"]),
                           workload="REDUCED " + w["config"]["workload"])
    return w


def _make_workload(name: str, rank: int):
    qseed = 1 + 1000 * rank  # rank 0 scores exactly the named workload
    if name in ("sparse", "sparse_structural"):
        mat = "blosum62" if name == "sparse" else "structural"
        return dict(kind="sparse", matrix=mat, thresh=24, queries=W.cdr3_skewed(qseed, 100000),
                    refs=W.cdr3_skewed(0, 1000000),
                    config={"workload": f"gapblock score_sparse 100000x1000000 CDR3-like (len 8-25, "
                                        f"mode 14), {mat}, gap_open 8, gap_extend 1, no prior, "
                                        "max_penalty 24, CSR (ref_id int32, score int32) output",
                            "queries": 100000, "refs": 1000000, "matrix": mat, "gap_open": 8,
                            "gap_extend": 1, "prior": None, "max_penalty": 24},
                    metric="gapblock thresholded sparse pairs/s")
    if name == "learned":
        qc, ql = W.cdr3_codes(qseed, 1000000)
        rc, rl = W.cdr3_codes(0, 1000000)
        return dict(kind="learned", matrix="blosum62", thresh=24, q_codes=qc, q_lens=ql,
                    r_codes=rc, r_lens=rl, _lazy_strings=True,
                    config={"workload": "learned proposal + exact rescore, 1000000x1000000 "
                                        "CDR3-like (len 8-25, mode 14), BLOSUM62, gap_open 8, "
                                        "gap_extend 1, no prior, max_penalty 24, top-256, "
                                        "recall bound 0.99",
                            "queries": 1000000, "refs": 1000000, "matrix": "blosum62",
                            "gap_open": 8, "gap_extend": 1, "prior": None, "max_penalty": 24,
                            "k": 256, "encoder": "2 conv + 2 attention, width 128, 64-d bf16"},
                    metric="learned-proposal effective pairs/s (exact rescore, recall >= 0.99)")
    if name == "gapblock":
        return dict(kind="gapblock", queries=W.cdr3(qseed, 1000), refs=W.cdr3(0, 10000),
                    config={"workload": "gapblock score_matrix 1000x10000 CDR3 junctions (len 10-20), "
                                        "BLOSUM62, gap_open 8, gap_extend 1, central_prior(21)",
                            "queries": 1000, "refs": 10000, "matrix": "BLOSUM62",
                            "gap_open": 8, "gap_extend": 1, "prior": "central_prior(21)"},
                    metric="gapblock score_matrix pairs/s")
    if name == "hamming":
        return dict(kind="hamming", queries=W.uniform_strings(qseed, 20000, 12, 12, "ACGT"),
                    refs=W.uniform_strings(0, 20000, 12, 12, "ACGT"),
                    config={"workload": "hamming_matrix 20000x20000 ACGT L=12", "queries": 20000,
                            "refs": 20000}, metric="hamming_matrix pairs/s")
    if name == "levenshtein":
        return dict(kind="levenshtein", queries=W.uniform_strings(qseed, 20000, 30, 60, "ACGT"),
                    refs=W.uniform_strings(0, 20000, 30, 60, "ACGT"),
                    config={"workload": "levenshtein_matrix 20000x20000 ACGT len 30-60",
                            "queries": 20000, "refs": 20000}, metric="levenshtein_matrix pairs/s")
    if name in ("nw", "sw"):
        mode = "global" if name == "nw" else "local"
        return dict(kind="align", mode=mode, queries=W.proteins(qseed, 4096),
                    refs=W.proteins(0, 4096),
                    config={"workload": f"align_dist_matrix {mode} 4096x4096 proteins (log-normal "
                                        "median 180, 50-500), BLOSUM62, gap 11/1",
                            "queries": 4096, "refs": 4096, "mode": mode},
                    metric=f"align_dist_matrix ({mode}) pairs/s")
    raise SystemExit(f"unknown workload {name}")


def line_config(w, world: int) -> dict:
    """The ``config`` object, identical in both arms for the same workload and N."""
    return dict(w["config"], l2=L2_NOTE,
                parallelism=f"{world} independent query blocks" if world > 1 else "single GPU")


def cells_of(w) -> float:
    """Algorithmic cells: gap block 2*min(m,n) (min(m,n) at d == 0); DP m*n; Hamming L."""
    lq = np.array([len(s) for s in w["queries"]], dtype=np.float64)
    lr = np.array([len(s) for s in w["refs"]], dtype=np.float64)
    if w["kind"] in ("gapblock", "sparse", "learned"):
        vq, cq = np.unique(lq, return_counts=True)
        vr, cr = np.unique(lr, return_counts=True)
        L = np.minimum(vq[:, None], vr[None, :])
        mult = np.where(vq[:, None] == vr[None, :], 1.0, 2.0)
        return float((cq[:, None] * cr[None, :] * L * mult).sum())
    if w["kind"] == "hamming":
        return float(lq.sum() * len(lr)) if len(lr) else 0.0
    return float(lq.sum() * lr.sum())


def fallback_cells(q_lens, r_lens, query_fallback, ref_fallback) -> tuple[float, float]:
    """(pairs, gap-block cells) the learned search scores exhaustively: fallback-length queries
    against every ref, and the other queries against fallback-length refs (cells as cells_of)."""
    vq, cq = np.unique(np.asarray(q_lens, np.int64), return_counts=True)
    vr, cr = np.unique(np.asarray(r_lens, np.int64), return_counts=True)
    fq = np.isin(vq, list(query_fallback))[:, None]
    fr = np.isin(vr, list(ref_fallback))[None, :]
    on = fq | fr
    n = cq[:, None].astype(np.float64) * cr[None, :]
    L = np.minimum(vq[:, None], vr[None, :]).astype(np.float64)
    mult = np.where(vq[:, None] == vr[None, :], 1.0, 2.0)
    return float((n * on).sum()), float((n * L * mult * on).sum())


# ----------------------------------------------------------------------------- helpers ------
def peaks() -> tuple[float, str]:
    try:
        return float(json.loads(PEAKS_FILE.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self._summary = None
        fd, name = tempfile.mkstemp(prefix="seqtree_b200_clocks_", suffix=".csv")
        os.close(fd)
        self.path = Path(name)  # scratch: read by summary(), then removed

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            if getattr(self, "fh", None) is not None:
                self.fh.close()
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self._summary is None and self.path.exists():
            if self.proc is not None:
                self._summary = self._read()
            self.path.unlink(missing_ok=True)
        return self._summary

    def _read(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def _peak_rate(int_peaks, op: str) -> tuple[float | None, float | None]:
    """(lane-ops/s on all SMs, lane-ops per SM clock) of a measured probe, or (None, None)."""
    try:
        p = int_peaks[op]["all_sms"]
        return float(p["lane_ops_per_s"]), float(p["per_sm_clk"])
    except Exception:
        return None, None


def kernel_roofline(w, cells: float, seconds: float, clocks, int_peaks=None) -> dict | None:
    """The dominant kernel against its own bound (the contract's roofline object is the HBM one).

    Peaks are the instruction rates measured in this process (``int_peaks``, all SMs, at the clock
    the probe ran); without them, the nominal 148 SMs x lanes/clk x SM clock.

    gap block: one conflict-free LDS.32 of a packed penalty word feeds two cells (two queries), so
    the algorithmic shared-memory traffic is 2 B/cell; the same two cells take one
    ``__viaddmin_s16x2``.  The bound is the LDS.32 rate (4 B per lane-load).
    alignment: DPX.  A DPX instruction updates one int16x2 cell pair.  Local mode needs 6 of them
    per pair (M, X, Y, H and the two gap extends) -- 3 per cell; global mode keeps the states
    raised by (i+j)*gap_extend, which folds each gap extend into its add-max, so 4 per pair -- 2
    per cell.  The bound is the measured ``__viaddmin_s16x2`` rate.
    levenshtein: ALU pipe.  The bit-vector step per text character is ten 64-bit logic, add and
    shift operations (the whole pattern, <= 64 symbols, in one word): 20 32-bit ALU lane-ops per
    (pair, query character), against the measured ALU-pipe rate (the IADD3 probe).
    """
    mhz = (clocks or {}).get("sm_mhz") or 1965.0
    sms = 148
    if w["kind"] in ("gapblock", "sparse"):
        lds, lds_clk = _peak_rate(int_peaks, "lds32")
        dpx, _ = _peak_rate(int_peaks, "viaddmin_s16x2")
        achieved = 2.0 * cells / seconds / 1e9
        if lds:
            peak, basis = 4.0 * lds / 1e9, (f"measured conflict-free LDS.32 rate, all SMs "
                                            f"({lds_clk:.1f} lane-loads/SM/clk)")
        else:
            peak, basis = sms * 128 * mhz * 1e6 / 1e9, f"148 SMs x 128 B/clk at {mhz:.0f} MHz"
        out = {"bound": "smem", "achieved": achieved, "peak": peak, "unit": "GB/s",
               "frac": achieved / peak, "work": "2 B of penalty per cell (one LDS.32 per 2 cells)",
               "peak_basis": basis}
        if dpx:
            a = cells / 2.0 / seconds
            out["dpx"] = {"op": "viaddmin_s16x2", "achieved": a / 1e9, "peak": dpx / 1e9,
                          "unit": "Glane-op/s", "frac": a / dpx, "work": "one per 2 cells"}
        return out
    if w["kind"] == "align":
        ops = 2.0 if w.get("mode") == "global" else 3.0
        achieved = ops * cells / seconds / 1e9
        dpx, dpx_clk = _peak_rate(int_peaks, "viaddmin_s16x2")
        if dpx:
            peak, basis = dpx / 1e9, (f"measured __viaddmin_s16x2 rate, all SMs "
                                      f"({dpx_clk:.1f} lanes/SM/clk)")
        else:
            peak, basis = sms * 64 * mhz * 1e6 / 1e9, f"148 SMs x 64 ALU lanes/clk at {mhz:.0f} MHz"
        return {"bound": "dpx", "achieved": achieved, "peak": peak, "unit": "Glane-op/s",
                "frac": achieved / peak,
                "work": f"{ops:.0f} DPX lane-ops per cell ({2 * ops:.0f} per int16x2 pair)",
                "peak_basis": basis}
    if w["kind"] == "levenshtein":
        steps = float(sum(map(len, w["queries"]))) * len(w["refs"])
        achieved = 20.0 * steps / seconds / 1e9
        alu, alu_clk = _peak_rate(int_peaks, "iadd3")
        if alu:
            peak, basis = alu / 1e9, (f"measured ALU-pipe rate (IADD3 probe), all SMs "
                                      f"({alu_clk:.1f} lanes/SM/clk)")
        else:
            peak, basis = sms * 64 * mhz * 1e6 / 1e9, f"148 SMs x 64 ALU lanes/clk at {mhz:.0f} MHz"
        return {"bound": "alu", "achieved": achieved, "peak": peak, "unit": "Glane-op/s",
                "frac": achieved / peak,
                "work": "20 ALU lane-ops per (pair, query character): one 64-bit bit-vector step",
                "peak_basis": basis}
    return None


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ----------------------------------------------------------------------------- reference ----
def _port_tables(name: str):
    """Penalty / similarity grid of a built-in matrix for the C port (only when the reference
    build is absent); the grids are plain Python data."""
    from seqtree_b200.matrix import SubstitutionMatrix
    return getattr(SubstitutionMatrix, name)()


def cpu_reference_call(w, threads: int):
    """(call(query_list) -> result, kind): the reference's own C++ when built, else the C port.
    Dense kinds return the int32 rows; sparse kinds return (row, ref) index arrays and scores of
    the cells <= the threshold."""
    import oracle
    if not isinstance(w["refs"], oracle.Prepacked):  # packed once, as a C++ caller holds them
        w["refs"] = oracle.Prepacked(w["refs"])
    if w["kind"] in ("sparse", "learned"):
        # The reference has no sparse form: its dense matrix over the sampled rows, thresholded.
        t = w["thresh"]
        if oracle.ref_available():
            def ref_sparse(q):
                d = oracle.ref_gapblock_matrix(q, w["refs"], matrix=w["matrix"], gap_open=8,
                                               gap_extend=1, threads=threads)
                return d, d <= t
            return ref_sparse, "reference"
        pen = _port_tables(w["matrix"]).penalty_grid

        def port_sparse(q):
            d = oracle.gapblock_matrix(q, w["refs"], pen, gap_open=8,
                                       threads=threads or os.cpu_count())
            return d, d <= t
        return port_sparse, "port"
    if w["kind"] == "gapblock":
        width = max(map(len, w["queries"] + w["refs"]))
        cube = w.setdefault("_cube", oracle.prior_cube(oracle.central_prior(21), width))
        if oracle.ref_available():
            return lambda q: oracle.ref_gapblock_matrix(q, w["refs"], matrix="blosum62",
                                                        gap_open=8, gap_extend=1, prior=cube,
                                                        prior_width=width, threads=threads), \
                "reference"
        pen = _port_tables("blosum62").penalty_grid
        return lambda q: oracle.gapblock_matrix(q, w["refs"], pen, gap_open=8, prior=cube,
                                                prior_width=width, threads=threads or os.cpu_count()), \
            "port"
    if w["kind"] in ("hamming", "levenshtein"):
        lev = w["kind"] == "levenshtein"
        if oracle.ref_available():
            return lambda q: oracle.ref_distance_matrix(q, w["refs"], lev, threads=threads), "reference"
        fn = oracle.levenshtein_matrix if lev else oracle.hamming_matrix
        return lambda q: fn(q, w["refs"], threads=threads or os.cpu_count()), "port"
    if oracle.ref_available():
        return lambda q: oracle.ref_align_matrix(q, w["refs"], "blosum62", mode=w["mode"],
                                                 dist=True, threads=threads), "reference"
    sim = _port_tables("blosum62").similarity_grid
    return lambda q: oracle.align_matrix(q, w["refs"], sim, mode=w["mode"], dist=True,
                                         threads=threads or os.cpu_count()), "port"


def spread_rows(n_total: int, n: int) -> np.ndarray:
    """n query rows evenly spaced over [0, n_total) (all of them when n >= n_total)."""
    if n >= n_total:
        return np.arange(n_total)
    return np.unique(np.linspace(0, n_total - 1, n).round().astype(np.int64))


def cpu_sample_rows(w, budget_s: float, threads: int, call=None) -> int:
    """Query rows such that one timed CPU call takes about budget_s seconds, rounded up to a
    multiple of the worker threads (the reference parallelises over query rows, so fewer rows
    than threads would leave cores idle)."""
    call = call or cpu_reference_call(w, threads)[0]
    cores = threads if threads > 0 else (os.cpu_count() or 1)
    n = min(len(w["queries"]), cores)
    t = time.perf_counter()
    call(w["queries"][:n])
    dt = max(time.perf_counter() - t, 1e-4)
    rows = int(n * budget_s / dt)
    rows = -(-max(rows, 1) // cores) * cores
    return max(1, min(len(w["queries"]), rows))


def run_cpu_baseline(w, budget_s=10.0, threads=0, gpu_rows=None):
    """The reference on evenly spaced query rows (about ``budget_s`` seconds of CPU work), and,
    with ``gpu_rows(rows) -> result`` given, the parity of the GPU result on those rows."""
    call, kind = cpu_reference_call(w, threads)
    n = cpu_sample_rows(w, budget_s, threads, call)
    if w["kind"] in ("sparse", "learned"):
        n = min(n, max(256, threads or os.cpu_count() or 1))  # dense rows over 1e6 refs: 4 MB each
    rows = spread_rows(len(w["queries"]), n)
    q = [w["queries"][int(i)] for i in rows]
    t = time.perf_counter()
    ref = call(q)
    dt = time.perf_counter() - t
    pairs = len(rows) * len(w["refs"])
    cores = threads if threads > 0 else (os.cpu_count() or 1)
    out = {"value": pairs / dt, "unit": "pairs/s", "cores": cores, "kind": kind,
           "sample": f"{len(rows)} of {len(w['queries'])} query rows, evenly spaced, x "
                     f"{len(w['refs'])} refs (rows are independent), one timed call"}
    if gpu_rows is not None:
        out["parity"] = parity(w, rows, ref, gpu_rows(rows), kind)
    return out


def parity(w, rows, ref, got, kind) -> dict:
    """Bit-exact comparison of GPU rows with the CPU checker's rows.  Dense kinds: ``got`` is the
    int32 rows.  Sparse kinds: ``got`` is a list of (ref_ids, scores) per row, which must equal the
    checker's thresholded dense row (refs ascending).  Learned: every GPU hit must be a checker
    hit with the same score, and the recall of those rows is reported."""
    checker = "reference C++ (oracle/_ref)" if kind == "reference" else "C port (oracle)"
    if w["kind"] in ("sparse", "learned"):
        dense, mask = ref
        exact, subset, found, want, nnz = True, True, 0, 0, 0
        for j, (ri, sc) in enumerate(got):
            cols = np.flatnonzero(mask[j]).astype(np.int32)
            want += cols.size
            nnz += ri.size
            if w["kind"] == "sparse":
                exact &= bool(np.array_equal(ri, cols) and np.array_equal(sc, dense[j, cols]))
            else:
                ok = bool(np.all(mask[j, ri]) and np.array_equal(sc, dense[j, ri])) if ri.size \
                    else True
                subset &= ok
                found += int(np.isin(ri, cols).sum())
        res = {"rows": int(len(rows)), "checker": checker, "checker_hits": int(want),
               "gpu_hits": int(nnz)}
        if w["kind"] == "sparse":
            res["exact"] = bool(exact)
        else:
            res.update(hits_exact=bool(subset), recall=found / want if want else 1.0)
        return res
    got = np.asarray(got)
    return {"rows": int(len(rows)), "cells": int(got.size), "exact": bool(np.array_equal(got, ref)),
            "checker": checker}


def main_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    line = reference_line(args, args.workload, world, float(
        os.environ.get("SEQTREE_B200_REF_STEP_S", "5")))
    if world == 1 and not args.no_suite and args.workload == "gapblock":
        line["workloads"] = {}
        for name in SUITE:
            try:
                line["workloads"][name] = reference_line(args, name, world, 0.25,
                                                         steps=min(args.steps, 5), warmup=1)
            except Exception as e:  # report and carry on with the next configuration
                line["workloads"][name] = {"impl": "reference", "error": str(e)}
    print(json.dumps(line), flush=True)
    return 0


def reference_line(args, name: str, world: int, step_s: float, steps: int | None = None,
                   warmup: int | None = None) -> dict:
    """The reference's own CPU implementation on the workload: each step a bounded sample of
    query rows (about ``step_s`` seconds, at least one row per host thread), with all host
    threads.  ``steps`` / ``warmup`` default to the command line's."""
    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    w = make_workload(name, 0, args.queries, args.refs)
    call, kind = cpu_reference_call(w, 0)
    rows = cpu_sample_rows(w, step_s, 0, call)
    q = w["queries"][:rows]
    for _ in range(warmup):
        call(q)
    times = []
    for _ in range(steps):
        t = time.perf_counter()
        call(q)
        times.append(time.perf_counter() - t)
    pairs = rows * len(w["refs"])
    v = pairs * len(times) / sum(times)
    cores = os.cpu_count() or 1
    return {"impl": "reference", "metric": w["metric"], "value": v, "unit": "pairs/s",
            "n_gpus": world, "steps": steps, "warmup": warmup,
            "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": line_config(w, world),
            "cpu_baseline": {"value": v, "unit": "pairs/s", "cores": cores, "kind": kind,
                             "sample": f"{rows} of {len(w['queries'])} query rows per step "
                                       f"(x {len(w['refs'])} refs)"},
            "e2e": {"value": v, "unit": "pairs/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


# ----------------------------------------------------------------------------- ours ---------
def measure_peaks() -> dict:
    """The instruction peaks (``st_measure_peak``) in this process, on one SM and on all SMs."""
    from seqtree_b200 import _lib
    return _lib.measure_peaks()


def main_ours(args):
    import torch

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    int_peaks = measure_peaks()
    if args.workload == "int_peak":
        line = peak_line(args, int_peaks, world)
    elif args.workload == "learned":
        line = measure_learned(args, world, rank, local, int_peaks)
    else:
        line = measure(args, args.workload, world, rank, local, int_peaks,
                       soak_s=args.soak_seconds)
    if line is not None and world == 1 and not args.no_suite and args.workload == "gapblock":
        line["workloads"] = {}
        for name in SUITE:
            try:
                if name == "learned":
                    sub = measure_learned(args, world, rank, local, int_peaks)
                else:
                    sub = measure(args, name, world, rank, local, int_peaks, soak_s=0.0)
            except Exception as e:  # report and carry on with the next configuration
                sub = {"metric": name, "error": f"{type(e).__name__}: {e}"}
            line["workloads"][name] = sub
            torch.cuda.empty_cache()
    if line is not None:
        line["int_peaks"] = {op: {"all_sms_lane_ops_per_s": v["all_sms"]["lane_ops_per_s"],
                                  "all_sms_per_sm_clk": v["all_sms"]["per_sm_clk"],
                                  "one_sm_per_clk": v["one_sm"]["per_sm_clk"]}
                             for op, v in int_peaks.items()}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def peak_line(args, int_peaks, world):
    alu = int_peaks["lop3"]["all_sms"]
    return {"metric": "integer ALU peak lane-ops/s (LOP3, all SMs)", "value": alu["lane_ops_per_s"],
            "unit": "lane-ops/s", "n_gpus": world, "steps": 3, "warmup": 1,
            "ms_per_step": alu["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic (register-only probe)",
            "config": {"workload": "instruction peak probes: 1,024-thread blocks, 8 accumulators "
                                   "per thread, 16,384 iterations; one SM and all SMs"},
            "probes": int_peaks}


def measure(args, name, world, rank, local, int_peaks, soak_s: float = 0.0):
    """One dense or sparse workload: device-resident steps (CUDA-graph replays where the step
    does not read back), end-to-end calls through the public API, the CPU reference on sampled
    rows and the parity of those rows.  Returns rank 0's line (None on other ranks)."""
    import torch

    import seqtree_b200 as stb
    from seqtree_b200 import _lib, device
    from seqtree_b200.gapblock import central_prior, prior_cube

    w = make_workload(name, rank, args.queries, args.refs)
    q, r = w["queries"], w["refs"]
    N, K = len(q), len(r)
    stream = torch.cuda.current_stream()
    out = None if w["kind"] == "sparse" else torch.empty((N, K), dtype=torch.int32, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device="cuda")
    B62 = stb.SubstitutionMatrix.blosum62()
    e2e_steps = args.e2e_steps if name == args.workload else min(args.e2e_steps, 3)

    cur = lambda: torch.cuda.current_stream().cuda_stream  # noqa: E731  (capture-aware)
    if w["kind"] == "gapblock":
        width = max(map(len, q + r))
        prior = central_prior(21)
        cube = np.asarray(prior_cube(prior, width), dtype=np.int32)
        qs, rs = device.SeqSet(q, "aa"), device.SeqSet(r, "aa")

        def step():
            device.gapblock_into(qs, rs, out.data_ptr(), cur(), matrix=B62,
                                 gap_open=8, gap_extend=1, prior=cube, prior_width=width)

        def e2e_call():
            return stb.gapblock.score_matrix(q, r, B62, gap_open=8, gap_extend=1,
                                             gap_prior=prior)
    elif w["kind"] == "sparse":
        from seqtree_b200.gapblock import score_sparse
        M = getattr(stb.SubstitutionMatrix, w["matrix"])()
        qs, rs = device.SeqSet(q, "aa"), device.SeqSet(r, "aa")
        hits = device.Hits()
        nnz_seen = []

        def step():
            nnz_seen.append(device.gapblock_sparse_into(qs, rs, hits, cur(), max_penalty=w["thresh"],
                                                        matrix=M, gap_open=8, gap_extend=1))

        def e2e_call():
            return score_sparse(q, r, w["thresh"], M, gap_open=8, gap_extend=1)
    elif w["kind"] in ("hamming", "levenshtein"):
        qs, rs = device.SeqSet(q, None), device.SeqSet(r, None)
        into = device.hamming_into if w["kind"] == "hamming" else device.levenshtein_into
        api = stb.distance.hamming_matrix if w["kind"] == "hamming" else stb.distance.levenshtein_matrix

        def step():
            into(qs, rs, out.data_ptr(), cur())

        def e2e_call():
            return api(q, r)
    else:
        qs, rs = device.SeqSet(q, "aa"), device.SeqSet(r, "aa")

        def step():
            device.align_into(qs, rs, out.data_ptr(), cur(), matrix=B62,
                              mode=w["mode"], gap_open=11, gap_extend=1, dist=True)

        def e2e_call():
            return stb.pairwise.dist_matrix(q, r, B62, mode=w["mode"])

    # warm-up (tuning, plans, workspace, module load), then capture one step in a CUDA graph so
    # the timed replays measure the device work alone (no host enqueue gaps inside the events)
    for _ in range(max(args.warmup, 1)):
        step()
    torch.cuda.synchronize()
    launches = _lib.last_launch_count()
    kernel_name = _lib.last_kernel_name()
    graph = None
    # The sparse step reads its hit count back to size the sort, so it is timed eagerly.
    if not args.no_graph and w["kind"] != "sparse":
        try:
            side = torch.cuda.Stream()
            side.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(side):
                step()
            torch.cuda.current_stream().wait_stream(side)
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph):
                step()
            torch.cuda.synchronize()
            run_step = graph.replay
        except Exception as e:  # not capturable on this path: time eager launches
            graph = None
            print(f"[bench] graph capture failed ({e}); timing eager launches", file=sys.stderr)
    if graph is None:
        run_step = step

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    sampler = ClockSampler(local)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    barrier()
    torch.cuda.synchronize()
    n0 = _lib.total_launch_count()
    with sampler:
        for i in range(args.steps):
            flush.zero_()  # evict the previous step's output from L2 (outside the events)
            ev[i][0].record(stream)
            run_step()
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        barrier()
        if graph is None:
            launches = (_lib.total_launch_count() - n0) // max(args.steps, 1)
        ms = [a.elapsed_time(b) for a, b in ev]
        # end-to-end through the public API on host lists (pinned result buffer)
        e2e_times = []
        for _ in range(e2e_steps):
            t = time.perf_counter()
            res = e2e_call()
            e2e_times.append(time.perf_counter() - t)
            del res
    total_ms = sum(ms)
    soak = None
    if soak_s > 0 and graph is not None:
        soak = run_soak(run_step, soak_s, local, total_ms / args.steps)
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    pairs_rank = N * K
    value = pairs_rank * world * args.steps / (total_ms / 1e3)
    e2e_s = statistics.median(e2e_times) if e2e_times else float("nan")
    in_bytes = sum(len(s) for s in q + r) + 8 * (N + K + 2)
    out_bytes_host = 4 * pairs_rank
    if w["kind"] == "sparse":
        out_bytes_host = 8 * (N + 1) + 8 * nnz_seen[-1]
    e2e = {"value": pairs_rank / e2e_s, "unit": "pairs/s", "h2d_bytes_per_step": in_bytes,
           "d2h_bytes_per_step": out_bytes_host, "seconds_per_step": e2e_s}
    if rank != 0:
        return None

    hbm, src = peaks()
    per_launch_s = (total_ms / args.steps) / 1e3
    out_bytes = 4.0 * pairs_rank if w["kind"] != "sparse" else float(out_bytes_host)
    in_dev_bytes = float(sum(len(s) for s in q + r))
    achieved = (out_bytes + in_dev_bytes) / per_launch_s / 1e9
    cells = cells_of(w)
    clocks = sampler.summary()
    line = {
        "metric": w["metric"], "value": value, "unit": "pairs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded, shapes and distributions of the named workload)",
        "config": line_config(w, world),
        "gcups": cells * world * args.steps / (total_ms / 1e3) / 1e9,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": TRAFFIC.get(w["kind"]),
                     "note": f"algorithmic bytes = 4 B/pair output + input residues; peak = "
                             f"{'measured copy bandwidth' if src == 'measured' else 'fallback 6.65 TB/s'} "
                             f"(of {src}); traffic = ncu dram read+write per launch (profiles/)"},
        "kernel_roofline": kernel_roofline(w, cells, per_launch_s, clocks, int_peaks),
        "e2e": e2e,
        "gpu_launches": int(launches) * args.steps,
        "kernel": kernel_name,
        "cuda_graph": graph is not None,
        "clocks": clocks,
        "tuning": [t for t in _lib.tuning_table().splitlines() if t],
    }
    if soak is not None:
        line["soak"] = soak
        # a timed region of ~1 ms gets at most one 200 ms sample: the soak's record (the same
        # step replayed for over a second right after it) stands in, the timed one kept beside
        if (not clocks or clocks.get("samples", 0) < 3) and soak.get("clocks"):
            if clocks:
                line["clocks_timed_region"] = clocks
            line["clocks"] = dict(soak["clocks"], source="soak: back-to-back replays of the "
                                                         "timed step, right after it")
    if w["kind"] == "sparse":
        line["nnz"] = nnz_seen[-1]
        line["roofline"]["note"] = ("algorithmic bytes = CSR output (8 B/hit + 8 B/row) + input "
                                    "residues; the scoring kernel is bound on chip (kernel_roofline)")

    def gpu_rows(rows):
        if w["kind"] == "sparse":
            return device.hits_rows(hits, rows)
        idx = torch.from_numpy(np.asarray(rows, np.int64)).cuda()
        return out.index_select(0, idx).cpu().numpy()

    if world == 1 and not args.no_cpu_baseline:
        try:
            budget = args.cpu_seconds if name == args.workload else min(args.cpu_seconds, 6.0)
            line["cpu_baseline"] = run_cpu_baseline(w, budget_s=budget, threads=0,
                                                    gpu_rows=gpu_rows)
        except Exception as e:  # the checker is absent: report, do not fail the run
            line["cpu_baseline"] = {"value": None, "error": str(e)}
    del out, flush
    return line


def run_soak(run_step, seconds: float, local: int, ms_per_step: float) -> dict:
    """Graph replays for about ``seconds`` (no L2 flush between them), with clocks sampled
    throughout: a clock record long enough to read, beside the short timed region."""
    import torch
    n = max(int(seconds * 1e3 / max(ms_per_step, 1e-3)), 1)
    sampler = ClockSampler(local)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    with sampler:
        a.record()
        for _ in range(n):
            run_step()
        b.record()
        torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    clocks = sampler.summary() or {}
    mhz = clocks.get("sm_mhz")
    return {"steps": n, "seconds": ms / 1e3, "ms_per_step": ms / n, "clocks": clocks,
            "ms_per_step_x_sm_mhz": (ms / n) * mhz if mhz else None,
            "note": "back-to-back graph replays, L2 warm; per-step time x median SM clock "
                    "normalises for the clock the steps ran at"}


def measure_learned(args, world, rank, local, int_peaks=None):
    """Learned proposal + exact rescore on 1M x 1M CDR3-like junctions.

    Setup (untimed): train the encoder on ``--train-pairs`` seeded pairs labelled by the exact
    kernel, embed the refs, calibrate on 4,000 held-out queries (seed 2): the threshold form's
    per-cell thresholds and fallback lengths (``--proposal range``, the default) or the top-256
    form's fallback lengths (``--proposal topk``).  A timed step re-embeds the refs and answers
    all queries: embed, propose, exact rescore, exhaustive fallback parts, CSR merge.  ``value``
    = nq * nr / step time (effective pairs/s).  Recall is measured on the first 2,000 workload queries against the exhaustive
    kernel; the exhaustive kernel's own pairs/s on 20,000 queries x all refs is reported beside.
    """
    import torch

    import seqtree_b200 as stb
    from seqtree_b200 import _lib, learned as Ln

    w = make_workload("learned", rank, args.queries, args.refs)
    M = stb.SubstitutionMatrix.blosum62()
    t0 = time.perf_counter()
    enc = Ln.Encoder(seed=0)
    if rank == 0:
        Ln.train(enc, args.train_pairs, seed=1, matrix=M, gap_open=8)
    params = enc.params()
    if world > 1:  # one trained model for every rank
        import torch.distributed as dist
        t = torch.from_numpy(params).cuda()
        dist.broadcast(t, 0)
        params = t.cpu().numpy()
        enc = Ln.Encoder(params)
    train_s = time.perf_counter() - t0
    idx = Ln.LearnedIndex(enc, w["r_codes"], w["r_lens"], matrix=M, gap_open=8, max_penalty=24,
                          k=256, proposal=args.proposal)
    cc, cl = W.cdr3_codes(2, 4000)
    cal = idx.calibrate(cc, cl, bound=0.99)
    qb = idx.queries(w["q_codes"], w["q_lens"])
    nq, nr = qb.count, idx.nr

    def step(phases=None):
        idx.embed_refs()
        if phases is not None:
            e = torch.cuda.Event(enable_timing=True)
            e.record()
            phases.setdefault("refs_embedded", []).append(e)
        return idx.search(qb, phases)

    for _ in range(max(args.warmup, 1)):
        res = step()
    torch.cuda.synchronize()
    del res
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device="cuda")
    sampler = ClockSampler(local)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    phases: dict = {}
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    last = None
    with sampler:
        n0 = _lib.total_launch_count()
        for i in range(args.steps):
            flush.zero_()
            ev[i][0].record()
            last = step(phases)
            ev[i][1].record()
        torch.cuda.synchronize()
        launches = (_lib.total_launch_count() - n0) / max(args.steps, 1)
        e2e_times, e2e_nnz = [], 0
        q_strings = w["queries"]
        e2e_steps = args.e2e_steps if args.workload == "learned" else min(args.e2e_steps, 3)
        for _ in range(e2e_steps):
            t = time.perf_counter()
            out = idx.search_strings(q_strings)
            e2e_times.append(time.perf_counter() - t)
            e2e_nnz = out.nnz
            del out
    ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = sum(ms)
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    # per-phase device time, averaged over the timed steps
    names = ["start", "refs_embedded", "embed", "propose", "rescore", "exhaustive", "merge"]
    have = [n for n in names if n in phases]
    phase_ms = {}
    for a, b in zip(have[:-1], have[1:]):
        phase_ms[f"{a}->{b}"] = statistics.mean(
            x.elapsed_time(y) for x, y in zip(phases[a], phases[b]))
    phase_ms["ref_embed"] = statistics.mean(
        x.elapsed_time(y) for x, y in zip((e[0] for e in ev), phases["refs_embedded"]))
    # recall on the first 2,000 workload queries; exhaustive kernel rate on 20,000
    ne = min(2000, nq)
    rec = idx.recall(w["q_codes"][:ne], w["q_lens"][:ne])
    nx = min(20000, nq)
    xq = idx.queries(w["q_codes"][:nx], w["q_lens"][:nx])
    xt = []
    for _ in range(3):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        idx.exhaustive(xq, w["q_codes"][:nx])
        b.record()
        torch.cuda.synchronize()
        xt.append(a.elapsed_time(b))
    exh_rate = nx * nr / (min(xt) / 1e3)
    value = nq * nr * world * args.steps / (total_ms / 1e3)
    if rank != 0:
        return None
    plans = None
    if not args.no_plans:
        other = "topk" if args.proposal == "range" else "range"
        plans = {"bound_0.99": learned_plans(w, M, (cc, cl), ne, 0.99, [
            ("fallback_only", None, 0, None, "topk"),
            ("untrained_encoder", Ln.Encoder(seed=0), 256, None, args.proposal),
            (f"trained_encoder_{other}", enc, 256, 1 if other == "topk" else None, other)])}
        plans["bound_0.99"][f"trained_encoder_{args.proposal}"] = {
            "ms_per_step": total_ms / args.steps, "effective_pairs_per_s": value / world,
            "recall": rec["recall"], "exhaustive_share": cal["exhaustive_share"],
            "query_fallback": cal["query_fallback"], "ref_fallback": cal["ref_fallback"],
            "the_timed_line": True}
        plans["bound_0.999"] = learned_plans(w, M, (cc, cl), ne, 0.999, [
            ("fallback_only", None, 0, None, "topk"),
            (f"trained_encoder_{args.proposal}", enc, 256, None, args.proposal)])
    e2e_s = statistics.median(e2e_times) if e2e_times else float("nan")
    prop_s = phase_ms.get("embed->propose", float("nan")) / 1e3
    n_lq, n_lr = len(qb.learn_rows), idx.n_learn
    if args.proposal == "range":  # the pairs the threshold form's tile ranges scan
        rg = qb.range_tiles(idx).view(-1, 2).cpu().numpy().astype(np.int64)
        rows = np.minimum(Ln.QUERY_TILE, n_lq - Ln.QUERY_TILE * np.arange(len(rg)))
        cols = np.minimum(rg[:, 1] * Ln.REF_TILE, n_lr) - np.minimum(rg[:, 0] * Ln.REF_TILE, n_lr)
        scanned = float((rows * np.maximum(cols, 0)).sum())
    else:
        scanned = float(n_lq) * n_lr
    flops = 2.0 * 64 * scanned
    achieved = flops / prop_s / 1e12 if prop_s > 0 else None
    peak, peak_src = FALLBACK_BF16_TFLOPS, "fallback"
    try:
        peak, peak_src = float(json.loads(PEAKS_FILE.read_text())["bf16_tflops"]), "measured"
    except Exception:
        pass
    kernel = "propose_range_kernel" if args.proposal == "range" else "propose_topk_kernel"
    clocks = sampler.summary()
    # The dominant kernel of the step is the exhaustive fallback's sparse gap-block kernel; its
    # phase is measured between the rescore and exhaustive marks.
    exh_s = phase_ms.get("rescore->exhaustive", float("nan")) / 1e3
    exh_pairs, exh_cells = fallback_cells(w["q_lens"], w["r_lens"], cal["query_fallback"],
                                          cal["ref_fallback"])
    nnz = int(last[0][-1].item()) if last is not None else 0
    residues = float(np.asarray(w["q_lens"], np.int64).sum() + np.asarray(w["r_lens"], np.int64).sum())
    hbm_peak, hbm_src = peaks()
    exh_bytes = 8.0 * nnz + 8.0 * (nq + 1) + residues
    exh_gbs = exh_bytes / exh_s / 1e9 if exh_s > 0 else None
    line = {
        "metric": w["metric"], "value": value, "unit": "pairs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16+int32",
        "data": "synthetic (seeded CDR3-like junctions, shapes and distributions of the named "
                "workload); encoder trained in setup on seeded pairs",
        "config": dict(line_config(w, world), train_pairs=args.train_pairs),
        "recall": rec["recall"], "recall_found": rec["found"], "recall_exact": rec["exact"],
        "recall_hits_all_exact": rec["subset_of_exact"],
        "recall_by_region": region_recall(rec["found_cells"], rec["exact_cells"]),
        "calibration": {k: v for k, v in cal.items()
                        if k not in ("cells_no_fallback", "candidate_cells", "levels")},
        "exhaustive_pairs_per_s": exh_rate, "speedup_vs_exhaustive": value / world / exh_rate,
        "phase_ms": phase_ms, "train_seconds": train_s,
        "plans": plans,
        "roofline": {"bound": "hbm", "achieved": exh_gbs, "peak": hbm_peak, "unit": "GB/s",
                     "frac": exh_gbs / hbm_peak if exh_gbs else None, "traffic": None,
                     "note": "dominant kernel: gapblock_fast_kernel<sparse>, the exhaustive "
                             "fallback's scoring (its phase time); algorithmic bytes = CSR rows "
                             f"(8 B/hit + 8 B/row) + input residues; peak = copy bandwidth (of "
                             f"{hbm_src}); the kernel is bound on chip (kernel_roofline)",
                     "pairs": exh_pairs},
        "kernel_roofline": kernel_roofline({"kind": "sparse"}, exh_cells, exh_s, clocks,
                                           int_peaks) if exh_s > 0 else None,
        "proposal_roofline": {"bound": "tensor", "achieved": achieved, "peak": peak,
                              "unit": "TFLOP/s", "frac": achieved / peak if achieved else None,
                              "note": f"{kernel}: 2*64 flops per scanned (learned query, learned "
                                      f"ref) pair / its phase time; peak = cuBLAS bf16 burst (of "
                                      f"{peak_src})",
                              "scanned_pairs": scanned},
        "e2e": {"value": nq * nr / e2e_s, "unit": "pairs/s",
                "h2d_bytes_per_step": int(sum(map(len, w["queries"])) + 8 * nq),
                "d2h_bytes_per_step": int(8 * (nq + 1) + 8 * e2e_nnz),
                "seconds_per_step": e2e_s},
        "gpu_launches": int(launches * args.steps),
        "kernel": "gapblock_fast_kernel<sparse> (exhaustive fallback)",
        "proposal_kernel": kernel,
        "proposal": args.proposal,
        "cuda_graph": False,
        "clocks": clocks,
    }
    ip, ri, sc = (x.cpu().numpy() for x in last)

    def gpu_rows(rows):
        return [(ri[ip[i]:ip[i + 1]], sc[ip[i]:ip[i + 1]]) for i in rows]

    if world == 1 and not args.no_cpu_baseline:
        try:
            budget = args.cpu_seconds if args.workload == "learned" else min(args.cpu_seconds, 6.0)
            line["cpu_baseline"] = run_cpu_baseline(w, budget_s=budget, threads=0,
                                                    gpu_rows=gpu_rows)
        except Exception as e:
            line["cpu_baseline"] = {"value": None, "error": str(e)}
    del last, flush
    return line


def region_recall(found_cells, exact_cells) -> dict:
    """Recall by (query length, ref length) region: a short query (8-10), a short ref (8-10)
    against a longer query, and both 11 or longer."""
    f, e = np.asarray(found_cells, np.float64), np.asarray(exact_cells, np.float64)
    regions = {"query_8_10": (slice(8, 11), slice(None)),
               "query_11plus_ref_8_10": (slice(11, None), slice(8, 11)),
               "both_11plus": (slice(11, None), slice(11, None))}
    out = {}
    for name, (a, b) in regions.items():
        ex = float(e[a, b].sum())
        out[name] = {"exact_hits": int(ex), "share_of_hits": ex / max(float(e.sum()), 1.0),
                     "recall": float(f[a, b].sum()) / ex if ex else 1.0}
    return out


def learned_plans(w, M, cal, rec_n: int, bound: float, plans, steps: int = 3) -> dict:
    """What the encoder earns: the same search, calibrated to the same recall ``bound`` on the
    same held-out batch, for each ``(name, encoder, k, band, proposal)`` of ``plans`` -- ``k = 0``
    is the method without the network (the calibrated exhaustive fallback alone); ``band`` limits
    each top-k query's proposals to refs within that many residues of its length; ``proposal`` is
    the top-k or the threshold form.  Each plan reports its step
    time over all queries (refs re-embedded, as in the timed steps), the effective pairs/s, the
    recall on the first ``rec_n`` workload queries and the share of pairs scored exhaustively."""
    import torch

    from seqtree_b200 import learned as Ln
    out = {}
    for name, enc, k, band, proposal in plans:
        idx = Ln.LearnedIndex(enc, w["r_codes"], w["r_lens"], matrix=M, gap_open=8,
                              max_penalty=24, k=k, band=band, proposal=proposal)
        cal_res = idx.calibrate(*cal, bound=bound)
        qb = idx.queries(w["q_codes"], w["q_lens"])
        idx.embed_refs()
        res = idx.search(qb)
        del res
        times = []
        for _ in range(steps):
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            idx.embed_refs()
            res = idx.search(qb)
            b.record()
            torch.cuda.synchronize()
            times.append(a.elapsed_time(b))
            del res
        rec = idx.recall(w["q_codes"][:rec_n], w["q_lens"][:rec_n])
        ms = statistics.median(times)
        out[name] = {"ms_per_step": ms, "effective_pairs_per_s": qb.count * idx.nr / (ms / 1e3),
                     "recall": rec["recall"], "exhaustive_share": cal_res["exhaustive_share"],
                     "recall_by_region": region_recall(rec["found_cells"], rec["exact_cells"]),
                     "query_fallback": cal_res["query_fallback"],
                     "ref_fallback": cal_res["ref_fallback"],
                     "candidates_per_query": cal_res.get("candidates_per_query")}
        del idx, qb
        torch.cuda.empty_cache()
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="gapblock",
                    choices=["gapblock", "hamming", "levenshtein", "nw", "sw", "sparse",
                             "sparse_structural", "learned", "int_peak"])
    ap.add_argument("--no-suite", action="store_true",
                    help="the named workload alone (no nested lines for the other configurations)")
    ap.add_argument("--train-pairs", type=int, default=10_000_000,
                    help="learned workload: encoder training pairs (setup, untimed)")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--soak-seconds", type=float, default=1.5,
                    help="graph replays after the timed steps, for the clock record")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--proposal", choices=["range", "topk"], default="range",
                    help="learned workload: threshold (range) or top-256 proposals")
    ap.add_argument("--no-plans", action="store_true",
                    help="learned workload: skip the without-network / untrained comparison")
    ap.add_argument("--no-graph", action="store_true", help="time eager launches instead")
    ap.add_argument("--queries", type=int, default=None,
                    help="use only the first N queries (smaller case for profiling captures)")
    ap.add_argument("--refs", type=int, default=None, help="use only the first N refs")
    args = ap.parse_args(argv)
    if args.impl == "reference":
        if args.workload == "int_peak":
            print(json.dumps({"impl": "reference", "unavailable": "instruction probes are GPU-only"}))
            return 0
        return main_reference(args)
    return main_ours(args)


if __name__ == "__main__":
    sys.exit(main())
