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
