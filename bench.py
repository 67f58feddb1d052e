#!/usr/bin/env python
"""Benchmark of the all-vs-all scoring path on B200 (one JSON line on rank 0).

Default workload (the one the headline metric is quoted on): gap-block ``score_matrix``,
1,000 query x 10,000 reference CDR3-like junctions ('CASS' + uniform middle + 'F', length
uniform 10-20; numpy PCG64 seed 1 for queries, seed 0 for refs), BLOSUM62 penalties,
gap_open 8, gap_extend 1, central_prior(21); int32 output bit-identical to seqtree's C++.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload gapblock|hamming|
                    levenshtein|nw|sw|sparse|sparse_structural] [--impl ours|reference]

Other workloads: ``hamming`` / ``levenshtein`` (20,000 x 20,000 ACGT), ``nw`` / ``sw`` (4,096 x
4,096 proteins, distance matrix), ``sparse`` / ``sparse_structural`` (100,000 x 1,000,000
CDR3-like, thresholded at max_penalty 24 into CSR rows; the dense matrix would be 400 GB).

* ``value``: pairs/s with inputs resident in HBM (device sets) and the result written to HBM,
  device-timed with CUDA events on the launching stream; the L2 is flushed (a 256 MiB write)
  between timed steps.  N > 1 (torchrun): every rank scores its own query block (weak scaling,
  no data-path collective); value = all ranks' pairs / max over ranks of the device time.
* ``e2e``: the same metric through the public API (``seqtree_b200.gapblock.score_matrix`` on
  Python lists): packing, host->device copy, kernels and the device->host copy of the result.
* ``cpu_baseline``: the reference's own C++ (``oracle/_ref``) on the host cores, rank 0, N=1.
* ``--impl reference``: times that CPU implementation alone, on this workload.
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

AA20 = "ACDEFGHIKLMNPQRSTVWY"
PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0
FALLBACK_BF16_TFLOPS = 1590.0
# DRAM bytes (read + write) per launch of the dominant kernel on the named workload, from the ncu
# captures summarised in profiles/ (None until captured).
TRAFFIC: dict[str, float | None] = {
    "gapblock": 1.91e6,     # 1.89 MB read + 0.02 MB write (the result stays in L2)
    "hamming": 1.31e9,      # 262 MB per 4,000 rows, scaled to 20,000 rows
    "levenshtein": 1.03e9,  # 102.5 MB per 2,000 rows, scaled to 20,000 rows
    "align": 1.05e6,        # one row-bucket launch of the wavefront kernel
}


# ----------------------------------------------------------------------------- workloads ----
def cdr3(seed: int, n: int, lo: int = 10, hi: int = 20) -> list[str]:
    rng = np.random.default_rng(seed)
    lens = rng.integers(lo, hi + 1, size=n)
    mid = rng.integers(0, 20, size=int((lens - 5).sum()))
    letters = np.array(list(AA20))[mid]
    out, p = [], 0
    for L in lens:
        k = int(L) - 5
        out.append("CASS" + "".join(letters[p:p + k]) + "F")
        p += k
    return out


def uniform_strings(seed: int, n: int, lo: int, hi: int, alphabet: str) -> list[str]:
    rng = np.random.default_rng(seed)
    lens = rng.integers(lo, hi + 1, size=n)
    codes = rng.integers(0, len(alphabet), size=int(lens.sum()))
    letters = np.array(list(alphabet))[codes]
    out, p = [], 0
    for L in lens:
        out.append("".join(letters[p:p + int(L)]))
        p += int(L)
    return out


# Background amino-acid frequencies (Robinson & Robinson 1991), order ACDEFGHIKLMNPQRSTVWY.
BG_FREQ = np.array([7.805, 1.925, 5.364, 6.295, 3.856, 7.377, 2.199, 5.142, 5.744, 9.019, 2.243,
                    4.487, 5.203, 4.264, 5.129, 7.120, 5.841, 6.441, 1.330, 3.216])


def proteins(seed: int, n: int) -> list[str]:
    """Residues i.i.d. from background frequencies; length log-normal, median 180, sigma 0.5,
    clipped to 50-500."""
    rng = np.random.default_rng(seed)
    lens = np.clip(np.round(rng.lognormal(np.log(180), 0.5, size=n)), 50, 500).astype(int)
    p = BG_FREQ / BG_FREQ.sum()
    codes = rng.choice(20, size=int(lens.sum()), p=p)
    letters = np.array(list(AA20))[codes]
    out, o = [], 0
    for L in lens:
        out.append("".join(letters[o:o + int(L)]))
        o += int(L)
    return out


def make_workload(name: str, rank: int, nq: int | None = None, nr: int | None = None):
    """The named workload (queries, refs, kind, config, metric); nq / nr shrink it for
    profiling captures of the same kernels on a smaller case."""
    w = _make_workload(name, rank)
    if w.pop("_lazy_strings", False):  # code arrays first; strings for the CPU reference
        from seqtree_b200.learned import codes_to_strings
        if nq is not None:
            w["q_codes"], w["q_lens"] = w["q_codes"][:nq], w["q_lens"][:nq]
        if nr is not None:
            w["r_codes"], w["r_lens"] = w["r_codes"][:nr], w["r_lens"][:nr]
        w["queries"] = codes_to_strings(w["q_codes"], w["q_lens"])
        w["refs"] = codes_to_strings(w["r_codes"], w["r_lens"])
    if nq is not None or nr is not None:
        w["queries"] = w["queries"][:nq] if nq is not None else w["queries"]
        w["refs"] = w["refs"][:nr] if nr is not None else w["refs"]
        w["config"] = dict(w["config"], queries=len(w["queries"]), refs=len(w["refs"]),
                           workload="REDUCED " + w["config"]["workload"])
    return w


def cdr3_skewed(seed: int, n: int) -> list[str]:
    """CDR3-like junctions 'CASS' + uniform middle + 'F' with length 8-25, mode 14: P(L) is a
    Gaussian around 14 with sigma 2.5 below and 3.5 above (right-skewed, like TRB junctions)."""
    rng = np.random.default_rng(seed)
    L = np.arange(8, 26)
    sig = np.where(L < 14, 2.5, 3.5)
    p = np.exp(-0.5 * ((L - 14) / sig) ** 2)
    lens = rng.choice(L, size=n, p=p / p.sum())
    mids = rng.integers(0, 20, size=int((lens - 5).sum()), dtype=np.uint8)
    letters = np.frombuffer(AA20.encode(), np.uint8)[mids].tobytes().decode()
    out, o = [], 0
    for length in lens:
        k = int(length) - 5
        out.append("CASS" + letters[o:o + k] + "F")
        o += k
    return out


def _make_workload(name: str, rank: int):
    qseed = 1 + 1000 * rank  # rank 0 scores exactly the named workload
    if name in ("sparse", "sparse_structural"):
        mat = "blosum62" if name == "sparse" else "structural"
        return dict(kind="sparse", matrix=mat, thresh=24, queries=cdr3_skewed(qseed, 100000),
                    refs=cdr3_skewed(0, 1000000),
                    config={"workload": f"gapblock score_sparse 100000x1000000 CDR3-like (len 8-25, "
                                        f"mode 14), {mat}, gap_open 8, gap_extend 1, no prior, "
                                        "max_penalty 24, CSR (ref_id int32, score int32) output",
                            "queries": 100000, "refs": 1000000, "matrix": mat, "gap_open": 8,
                            "gap_extend": 1, "prior": None, "max_penalty": 24},
                    metric="gapblock thresholded sparse pairs/s")
    if name == "learned":
        from seqtree_b200.learned import cdr3_codes
        qc, ql = cdr3_codes(qseed, 1000000)
        rc, rl = cdr3_codes(0, 1000000)
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
        return dict(kind="gapblock", queries=cdr3(qseed, 1000), refs=cdr3(0, 10000),
                    config={"workload": "gapblock score_matrix 1000x10000 CDR3 junctions (len 10-20), "
                                        "BLOSUM62, gap_open 8, gap_extend 1, central_prior(21)",
                            "queries": 1000, "refs": 10000, "matrix": "BLOSUM62",
                            "gap_open": 8, "gap_extend": 1, "prior": "central_prior(21)"},
                    metric="gapblock score_matrix pairs/s")
    if name == "hamming":
        return dict(kind="hamming", queries=uniform_strings(qseed, 20000, 12, 12, "ACGT"),
                    refs=uniform_strings(0, 20000, 12, 12, "ACGT"),
                    config={"workload": "hamming_matrix 20000x20000 ACGT L=12", "queries": 20000,
                            "refs": 20000}, metric="hamming_matrix pairs/s")
    if name == "levenshtein":
        return dict(kind="levenshtein", queries=uniform_strings(qseed, 20000, 30, 60, "ACGT"),
                    refs=uniform_strings(0, 20000, 30, 60, "ACGT"),
                    config={"workload": "levenshtein_matrix 20000x20000 ACGT len 30-60",
                            "queries": 20000, "refs": 20000}, metric="levenshtein_matrix pairs/s")
    if name in ("nw", "sw"):
        mode = "global" if name == "nw" else "local"
        return dict(kind="align", mode=mode, queries=proteins(qseed, 4096), refs=proteins(0, 4096),
                    config={"workload": f"align_dist_matrix {mode} 4096x4096 proteins (log-normal "
                                        "median 180, 50-500), BLOSUM62, gap 11/1",
                            "queries": 4096, "refs": 4096, "mode": mode},
                    metric=f"align_dist_matrix ({mode}) pairs/s")
    raise SystemExit(f"unknown workload {name}")


def cells_of(w) -> float:
    """Algorithmic cells: gap block 2*min(m,n) (min(m,n) at d == 0); DP m*n; Hamming L."""
    lq = np.array([len(s) for s in w["queries"]], dtype=np.float64)
    lr = np.array([len(s) for s in w["refs"]], dtype=np.float64)
    if w["kind"] in ("gapblock", "sparse"):
        vq, cq = np.unique(lq, return_counts=True)
        vr, cr = np.unique(lr, return_counts=True)
        L = np.minimum(vq[:, None], vr[None, :])
        mult = np.where(vq[:, None] == vr[None, :], 1.0, 2.0)
        return float((cq[:, None] * cr[None, :] * L * mult).sum())
    if w["kind"] == "hamming":
        return float(lq.sum() * len(lr)) if len(lr) else 0.0
    return float(lq.sum() * lr.sum())


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


def kernel_roofline(w, cells: float, seconds: float, clocks) -> dict | None:
    """The dominant kernel's own bound (the contract's roofline object above is the HBM one).

    gap block: shared-memory bandwidth.  Every cell needs one 2-byte penalty; the kernel reads
    them as conflict-free 32-bit words, two cells (two queries) per word, so the algorithmic
    traffic is 2 B/cell against 128 B/clk/SM.
    alignment: ALU pipe.  A DPX instruction updates one int16x2 cell pair.  Local mode needs 6
    of them per pair (M, X, Y, H and the two gap extends) -- 3 per cell; global mode keeps the
    states raised by (i+j)*gap_extend, which folds each gap extend into its add-max, so 4 per
    pair -- 2 per cell -- against 64 lanes/clk/SM.
    levenshtein: ALU pipe.  The bit-vector step per text character is ten 64-bit logic, add and
    shift operations (the whole pattern, <= 64 symbols, in one word): 20 32-bit ALU lane-ops
    per (pair, query character) against 64 lanes/clk/SM.
    """
    mhz = (clocks or {}).get("sm_mhz") or 1965.0
    sms = 148
    if w["kind"] in ("gapblock", "sparse"):
        achieved = 2.0 * cells / seconds / 1e9
        peak = sms * 128 * mhz * 1e6 / 1e9
        return {"bound": "smem", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "work": "2 B of penalty per cell",
                "peak_basis": f"148 SMs x 128 B/clk at {mhz:.0f} MHz"}
    if w["kind"] == "align":
        ops = 2.0 if w.get("mode") == "global" else 3.0
        achieved = ops * cells / seconds / 1e9
        peak = sms * 64 * mhz * 1e6 / 1e9
        return {"bound": "alu", "achieved": achieved, "peak": peak, "unit": "Glane-op/s",
                "frac": achieved / peak,
                "work": f"{ops:.0f} DPX lane-ops per cell ({2 * ops:.0f} per int16x2 pair)",
                "peak_basis": f"148 SMs x 64 ALU lanes/clk at {mhz:.0f} MHz"}
    if w["kind"] == "levenshtein":
        steps = float(sum(map(len, w["queries"]))) * len(w["refs"])
        achieved = 20.0 * steps / seconds / 1e9
        peak = sms * 64 * mhz * 1e6 / 1e9
        return {"bound": "alu", "achieved": achieved, "peak": peak, "unit": "Glane-op/s",
                "frac": achieved / peak,
                "work": "20 ALU lane-ops per (pair, query character): one 64-bit bit-vector step",
                "peak_basis": f"148 SMs x 64 ALU lanes/clk at {mhz:.0f} MHz"}
    return None


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ----------------------------------------------------------------------------- reference ----
def cpu_reference_call(w, threads: int):
    import oracle
    if w["kind"] in ("sparse", "learned"):
        # The reference has no sparse form: its dense matrix over the sampled rows, thresholded.
        t = w["thresh"]
        if oracle.ref_available():
            def ref_sparse(q):
                d = oracle.ref_gapblock_matrix(q, w["refs"], matrix=w["matrix"], gap_open=8,
                                               gap_extend=1, threads=threads)
                return np.nonzero(d <= t)
            return ref_sparse, "reference"
        from seqtree_b200.matrix import SubstitutionMatrix
        pen = getattr(SubstitutionMatrix, w["matrix"])().penalty_grid

        def port_sparse(q):
            d = oracle.gapblock_matrix(q, w["refs"], pen, gap_open=8,
                                       threads=threads or os.cpu_count())
            return np.nonzero(d <= t)
        return port_sparse, "port"
    if w["kind"] == "gapblock":
        from seqtree_b200.gapblock import central_prior, prior_cube
        width = max(map(len, w["queries"] + w["refs"]))
        cube = w.setdefault("_cube", prior_cube(central_prior(21), width))
        if oracle.ref_available():
            return lambda q: oracle.ref_gapblock_matrix(q, w["refs"], matrix="blosum62",
                                                        gap_open=8, gap_extend=1, prior=cube,
                                                        prior_width=width, threads=threads), \
                "reference"
        from seqtree_b200.matrix import SubstitutionMatrix
        pen = SubstitutionMatrix.blosum62().penalty_grid
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
    from seqtree_b200.matrix import SubstitutionMatrix
    sim = SubstitutionMatrix.blosum62().similarity_grid
    return lambda q: oracle.align_matrix(q, w["refs"], sim, mode=w["mode"], dist=True,
                                         threads=threads or os.cpu_count()), "port"


def cpu_sample_rows(w, budget_s: float, threads: int) -> int:
    """Query rows such that one timed CPU call takes about budget_s seconds."""
    call, _ = cpu_reference_call(w, threads)
    n = min(len(w["queries"]), 8)
    t = time.perf_counter()
    call(w["queries"][:n])
    dt = max(time.perf_counter() - t, 1e-4)
    rows = int(n * budget_s / dt)
    return max(1, min(len(w["queries"]), rows))


def run_cpu_baseline(w, budget_s=10.0, threads=0, reps=1):
    call, kind = cpu_reference_call(w, threads)
    rows = cpu_sample_rows(w, budget_s / max(reps, 1), threads)
    q = w["queries"][:rows]
    times = []
    for _ in range(reps):
        t = time.perf_counter()
        call(q)
        times.append(time.perf_counter() - t)
    pairs = rows * len(w["refs"])
    cores = threads if threads > 0 else (os.cpu_count() or 1)
    return {"value": pairs / statistics.median(times), "unit": "pairs/s", "cores": cores,
            "kind": kind,
            "sample": f"{rows} of {len(w['queries'])} query rows x {len(w['refs'])} refs "
                      f"(rows are independent), median of {reps}"}


def main_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    w = make_workload(args.workload, 0, args.queries, args.refs)
    call, kind = cpu_reference_call(w, 0)
    # Each step is a bounded sample of the workload sized so the whole run stays in minutes.
    budget = float(os.environ.get("SEQTREE_B200_REF_STEP_S", "5"))
    rows = cpu_sample_rows(w, budget, 0)
    q = w["queries"][:rows]
    for _ in range(args.warmup):
        call(q)
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        call(q)
        times.append(time.perf_counter() - t)
    pairs = rows * len(w["refs"])
    v = pairs * len(times) / sum(times)
    cores = os.cpu_count() or 1
    line = {"impl": "reference", "metric": w["metric"], "value": v, "unit": "pairs/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": dict(w["config"], sample_rows=rows),
            "cpu_baseline": {"value": v, "unit": "pairs/s", "cores": cores, "kind": kind,
                             "sample": f"{rows} of {len(w['queries'])} query rows per step"},
            "e2e": {"value": v, "unit": "pairs/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------- ours ---------
def main_ours(args):
    import torch

    world, rank, local = dist_env()
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(local)
    import seqtree_b200 as stb
    from seqtree_b200 import _lib, device
    from seqtree_b200.gapblock import central_prior, prior_cube

    w = make_workload(args.workload, rank, args.queries, args.refs)
    q, r = w["queries"], w["refs"]
    N, K = len(q), len(r)
    stream = torch.cuda.current_stream()
    out = None if w["kind"] == "sparse" else torch.empty((N, K), dtype=torch.int32, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device="cuda")
    B62 = stb.SubstitutionMatrix.blosum62()

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

    # warm-up (plans, workspace, module load), then capture one step in a CUDA graph so the
    # timed replays measure the device work alone (no host enqueue gaps inside the events)
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
    with sampler:
        for i in range(args.steps):
            flush.zero_()  # evict the previous step's output from L2 (outside the events)
            ev[i][0].record(stream)
            run_step()
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        barrier()
        ms = [a.elapsed_time(b) for a, b in ev]
        # end-to-end through the public API on host lists (pinned result buffer)
        e2e_times, h2d = [], 0
        for _ in range(args.e2e_steps):
            t = time.perf_counter()
            res = e2e_call()
            e2e_times.append(time.perf_counter() - t)
            del res
    total_ms = sum(ms)
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
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return 0

    hbm, src = peaks()
    per_launch_s = (total_ms / args.steps) / 1e3
    out_bytes = 4.0 * pairs_rank if w["kind"] != "sparse" else float(out_bytes_host)
    in_dev_bytes = float(sum(len(s) for s in q + r))
    achieved = (out_bytes + in_dev_bytes) / per_launch_s / 1e9
    cells = cells_of(w)
    line = {
        "metric": w["metric"], "value": value, "unit": "pairs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded, shapes and distributions of the named workload)",
        "config": dict(w["config"], l2="flushed between timed steps (256 MiB write)",
                       parallelism=f"{world} independent query blocks" if world > 1 else "single GPU"),
        "gcups": cells * world * args.steps / (total_ms / 1e3) / 1e9,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": TRAFFIC.get(w["kind"]),
                     "note": f"algorithmic bytes = 4 B/pair output + input residues; peak = "
                             f"{'measured copy bandwidth' if src == 'measured' else 'fallback 6.65 TB/s'} "
                             f"(of {src}); traffic = ncu dram read+write per launch (profiles/)"},
        "kernel_roofline": kernel_roofline(w, cells, per_launch_s, sampler.summary()),
        "e2e": e2e,
        "gpu_launches": launches * args.steps,
        "kernel": kernel_name,
        "cuda_graph": graph is not None,
        "clocks": sampler.summary(),
        "tuning": [t for t in _lib.tuning_table().splitlines() if t],
    }
    if w["kind"] == "sparse":
        line["nnz"] = nnz_seen[-1]
        line["roofline"]["note"] = ("algorithmic bytes = CSR output (8 B/hit + 8 B/row) + input "
                                    "residues; the scoring kernel is bound on chip (kernel_roofline)")
    if world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = run_cpu_baseline(w, budget_s=args.cpu_seconds, threads=0)
        except Exception as e:  # the checker is absent: report, do not fail the run
            line["cpu_baseline"] = {"value": None, "error": str(e)}
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main_learned(args):
    """Learned proposal + exact rescore on 1M x 1M CDR3-like junctions.

    Setup (untimed): train the encoder on ``--train-pairs`` seeded pairs labelled by the exact
    kernel, embed the refs, calibrate the fallback lengths on 4,000 held-out queries (seed 2).
    A timed step re-embeds the refs and answers all queries: embed, propose top-256, exact
    rescore, exhaustive fallback parts, CSR merge.  ``value`` = nq * nr / step time (effective
    pairs/s).  Recall is measured on the first 2,000 workload queries against the exhaustive
    kernel; the exhaustive kernel's own pairs/s on 20,000 queries x all refs is reported beside.
    """
    import torch

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
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
                          k=256)
    cc, cl = Ln.cdr3_codes(2, 4000)
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
    with sampler:
        n0 = _lib.total_launch_count()
        for i in range(args.steps):
            flush.zero_()
            ev[i][0].record()
            res = step(phases)
            ev[i][1].record()
            del res
        torch.cuda.synchronize()
        launches = (_lib.total_launch_count() - n0) / max(args.steps, 1)
        e2e_times, e2e_nnz = [], 0
        q_strings = w["queries"]
        for _ in range(args.e2e_steps):
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
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return 0
    e2e_s = statistics.median(e2e_times) if e2e_times else float("nan")
    prop_s = phase_ms.get("embed->propose", float("nan")) / 1e3
    n_lq, n_lr = len(qb.learn_rows), idx.n_learn
    flops = 2.0 * 64 * n_lq * n_lr
    achieved = flops / prop_s / 1e12 if prop_s > 0 else None
    peak, peak_src = FALLBACK_BF16_TFLOPS, "fallback"
    try:
        peak, peak_src = float(json.loads(PEAKS_FILE.read_text())["bf16_tflops"]), "measured"
    except Exception:
        pass
    line = {
        "metric": w["metric"], "value": value, "unit": "pairs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16+int32",
        "data": "synthetic (seeded CDR3-like junctions, shapes and distributions of the named "
                "workload); encoder trained in setup on seeded pairs",
        "config": dict(w["config"], l2="flushed between timed steps (256 MiB write)",
                       train_pairs=args.train_pairs,
                       parallelism=f"{world} independent query blocks" if world > 1 else "single GPU"),
        "recall": rec["recall"], "recall_found": rec["found"], "recall_exact": rec["exact"],
        "recall_hits_all_exact": rec["subset_of_exact"],
        "calibration": {k: v for k, v in cal.items() if k != "cells_no_fallback"},
        "exhaustive_pairs_per_s": exh_rate, "speedup_vs_exhaustive": value / world / exh_rate,
        "phase_ms": phase_ms, "train_seconds": train_s,
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if achieved else None, "traffic": None,
                     "note": "propose_topk_kernel: 2*64 flops per (learned query, learned ref) "
                             f"pair / its phase time; peak = cuBLAS bf16 burst (of {peak_src})"},
        "e2e": {"value": nq * nr / e2e_s, "unit": "pairs/s",
                "h2d_bytes_per_step": int(sum(map(len, w["queries"])) + 8 * nq),
                "d2h_bytes_per_step": int(8 * (nq + 1) + 8 * e2e_nnz),
                "seconds_per_step": e2e_s},
        "gpu_launches": int(launches * args.steps),
        "kernel": "propose_topk_kernel",
        "cuda_graph": False,
        "clocks": sampler.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = run_cpu_baseline(w, budget_s=args.cpu_seconds, threads=0)
        except Exception as e:
            line["cpu_baseline"] = {"value": None, "error": str(e)}
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="gapblock",
                    choices=["gapblock", "hamming", "levenshtein", "nw", "sw", "sparse",
                             "sparse_structural", "learned"])
    ap.add_argument("--train-pairs", type=int, default=10_000_000,
                    help="learned workload: encoder training pairs (setup, untimed)")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-graph", action="store_true", help="time eager launches instead")
    ap.add_argument("--queries", type=int, default=None,
                    help="use only the first N queries (smaller case for profiling captures)")
    ap.add_argument("--refs", type=int, default=None, help="use only the first N refs")
    args = ap.parse_args(argv)
    if args.impl == "reference":
        return main_reference(args)
    if args.workload == "learned":
        return main_learned(args)
    return main_ours(args)


if __name__ == "__main__":
    sys.exit(main())
