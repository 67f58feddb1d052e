"""Host-side arithmetic of bench.py: the kernel rooflines, the peak fallback and the clock
sampler's parsing.  No device needed; nothing here times anything."""
from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("seqtree_bench", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    argv, sys.argv = sys.argv, ["bench.py"]
    try:
        spec.loader.exec_module(mod)
    finally:
        sys.argv = argv
    return mod


def test_kernel_rooflines(bench):
    clocks = {"sm_mhz": 1000.0}
    alu_peak = 148 * 64 * 1000.0 * 1e6 / 1e9
    # levenshtein: 20 ALU lane-ops per (pair, query character)
    w = {"kind": "levenshtein", "queries": ["A" * 40] * 10, "refs": ["C" * 50] * 30}
    r = bench.kernel_roofline(w, 0.0, 1e-3, clocks)
    assert r["bound"] == "alu" and r["peak"] == pytest.approx(alu_peak)
    assert r["achieved"] == pytest.approx(20.0 * 400 * 30 / 1e-3 / 1e9)
    # alignment: 2 DPX lane-ops per cell in global mode (raised states), 3 in local mode
    for mode, ops in (("global", 2.0), ("local", 3.0)):
        r = bench.kernel_roofline({"kind": "align", "mode": mode}, 1e9, 1.0, clocks)
        assert r["bound"] == "dpx"
        assert r["achieved"] == pytest.approx(ops) and r["frac"] == pytest.approx(ops / alu_peak)
    # gap block: 2 B of penalty per cell against 128 B/clk/SM of shared memory
    r = bench.kernel_roofline({"kind": "gapblock"}, 1e9, 1.0, clocks)
    assert r["bound"] == "smem" and r["peak"] == pytest.approx(148 * 128 * 1000.0 * 1e6 / 1e9)
    assert bench.kernel_roofline({"kind": "hamming"}, 1e9, 1.0, clocks) is None


def test_peak_fallback_is_labelled(bench, tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "PEAKS_FILE", tmp_path / "absent.json")
    assert bench.peaks() == (bench.FALLBACK_HBM_GBS, "fallback")
    f = tmp_path / "peaks.json"
    f.write_text('{"hbm_gbs": 7000.5}')
    monkeypatch.setattr(bench, "PEAKS_FILE", f)
    assert bench.peaks() == (7000.5, "measured")


def test_clock_sampler_parses_and_cleans_up(bench):
    s = bench.ClockSampler(0)
    s.path.write_text(
        "0, 1965, 1965, 700.0, 0x0, Not Active, Not Active, Not Active, Active\n"
        "0, 1800, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active\n"
        "0, 1900, 1965, 900.0, 0x0, Not Active, Not Active, Not Active, Not Active\n"
        "garbage line\n")
    s.proc = object()  # as if nvidia-smi had run and written the file
    got = s.summary()
    assert got == {"sm_mhz": 1900.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"],
                   "samples": 3}
    assert not s.path.exists() and s.summary() == got  # read once, then removed
    idle = bench.ClockSampler(0)  # never started: no summary, and its file is removed
    assert idle.summary() is None and not idle.path.exists()


def test_kernel_rooflines_use_measured_peaks(bench):
    def probe(rate, per_clk):
        return {"all_sms": {"lane_ops_per_s": rate, "per_sm_clk": per_clk},
                "one_sm": {"lane_ops_per_s": rate / 148, "per_sm_clk": per_clk}}
    peaks = {"lds32": probe(8e12, 27.5), "viaddmin_s16x2": probe(9e12, 31.0),
             "iadd3": probe(1.8e13, 62.0)}
    r = bench.kernel_roofline({"kind": "gapblock"}, 1e12, 1.0, None, peaks)
    assert r["peak"] == pytest.approx(4 * 8e12 / 1e9) and "measured" in r["peak_basis"]
    assert r["achieved"] == pytest.approx(2e3) and r["dpx"]["frac"] == pytest.approx(0.5e12 / 9e12)
    r = bench.kernel_roofline({"kind": "align", "mode": "local"}, 1e12, 1.0, None, peaks)
    assert r["peak"] == pytest.approx(9e3) and r["frac"] == pytest.approx(3e12 / 9e12)
    w = {"kind": "levenshtein", "queries": ["A" * 10] * 2, "refs": ["C"] * 5}
    r = bench.kernel_roofline(w, 0.0, 1.0, None, peaks)
    assert r["peak"] == pytest.approx(1.8e4) and r["achieved"] == pytest.approx(20 * 100 / 1e9)


def test_spread_rows_and_config_keys(bench):
    assert bench.spread_rows(5, 10).tolist() == [0, 1, 2, 3, 4]
    rows = bench.spread_rows(20000, 256)
    assert rows[0] == 0 and rows[-1] == 19999 and len(rows) == 256
    assert (rows[1:] > rows[:-1]).all()
    w = bench.make_workload("gapblock", 0)
    assert bench.line_config(w, 1) == bench.line_config(bench.make_workload("gapblock", 0), 1)
    assert set(bench.line_config(w, 2)) == set(w["config"]) | {"l2", "parallelism"}


def test_parity_dense_sparse_and_learned(bench):
    import numpy as np
    ref = np.arange(12, dtype=np.int32).reshape(3, 4)
    w = {"kind": "hamming"}
    assert bench.parity(w, [0, 1, 2], ref, ref.copy(), "reference")["exact"]
    bad = ref.copy()
    bad[1, 2] += 1
    assert not bench.parity(w, [0, 1, 2], ref, bad, "port")["exact"]
    dense = np.array([[3, 30, 1, 24], [50, 60, 70, 80]], np.int32)
    mask = dense <= 24
    good = [(np.array([0, 2, 3], np.int32), np.array([3, 1, 24], np.int32)),
            (np.zeros(0, np.int32), np.zeros(0, np.int32))]
    res = bench.parity({"kind": "sparse"}, [4, 9], (dense, mask), good, "reference")
    assert res["exact"] and res["checker_hits"] == 3 and res["gpu_hits"] == 3
    wrong = [(np.array([0, 2], np.int32), np.array([3, 1], np.int32)), good[1]]
    assert not bench.parity({"kind": "sparse"}, [4, 9], (dense, mask), wrong, "reference")["exact"]
    res = bench.parity({"kind": "learned"}, [4, 9], (dense, mask), wrong, "reference")
    assert res["hits_exact"] and res["recall"] == pytest.approx(2 / 3)
    lie = [(np.array([1], np.int32), np.array([30], np.int32)), good[1]]
    assert not bench.parity({"kind": "learned"}, [4, 9], (dense, mask), lie, "reference")["hits_exact"]


def test_reference_arm_does_not_load_the_library():
    """The reference arm builds its inputs and prior cube without this library's shared
    object: the process that times the reference's C++ never maps libseqtree_b200.so."""
    import subprocess
    code = (
        "import sys; sys.argv=['bench.py']; sys.path.insert(0, %r)\n"
        "import bench\n"
        "w = bench.make_workload('gapblock', 0, 4, 50)\n"
        "call, kind = bench.cpu_reference_call(w, 1)\n"
        "d = call(w['queries'])\n"
        "assert d.shape == (4, 50)\n"
        "maps = open('/proc/self/maps').read()\n"
        "assert 'libseqtree_b200' not in maps, 'library mapped'\n"
        "assert 'seqtree_b200._lib' not in sys.modules\n"
        "print('clean', kind)\n") % str(ROOT)
    res = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         timeout=300, cwd=str(ROOT))
    assert res.returncode == 0, res.stdout + res.stderr
    assert "clean" in res.stdout


def test_learned_fallback_cells(bench):
    """fallback_cells: the pairs and gap-block cells the learned search scores exhaustively --
    fallback-length queries against every ref, the other queries against fallback-length refs."""
    q = [8, 8, 12, 15]
    r = [8, 10, 12]
    pairs, cells = bench.fallback_cells(q, r, [8], [10])
    want_pairs = want_cells = 0.0
    for a in q:
        for b in r:
            if a == 8 or b == 10:
                want_pairs += 1
                want_cells += min(a, b) * (1 if a == b else 2)
    assert pairs == want_pairs and cells == want_cells
    assert bench.fallback_cells(q, r, [], []) == (0.0, 0.0)
