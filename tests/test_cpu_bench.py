"""Pieces of bench.py's output contract that need no GPU: the roofline
denominators (measured file or the stated fallback), the mapped-read share,
the compact summary printed last, and the reference arm under torchrun
(ranks other than 0 exit 0 at once)."""
import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

import bench

ROOT = Path(__file__).resolve().parent.parent


def test_peaks_fall_back_and_say_so(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    pk, basis = bench.peaks()
    assert basis == "fallback"
    assert pk["hbm_gbs"] == 6650.0 and pk["bf16_tflops_sustained"] == 1400.0
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps(
        {"hbm_gbs": 6545.6, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1381.3}))
    pk, basis = bench.peaks()
    assert basis == "measured" and pk["bf16_tflops_sustained"] == 1381.3


def test_mapped_fraction_counts_overlapping_windows():
    # windows start every 15 bases (1-based starts); a read maps when one of
    # its top-k windows overlaps its true 150-base span
    col_start = np.array([1, 16, 31, 1001, 5001], np.int64)
    starts0 = np.array([0, 1000, 3000])          # 0-based true read starts
    locs = np.array([[1, 5], [5, 4], [1, 2]])    # 1-based columns
    frac = bench.mapped_fraction(locs, starts0, col_start)
    assert abs(frac - 2 / 3) < 1e-12


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2"],
                       capture_output=True, text=True, timeout=120, env=env, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""


def test_summary_carries_every_leg_and_tolerates_missing_ones():
    line = {"value": 42550.1, "e2e": {"value": 42410.2},
            "roofline": {"achieved": 2925.3, "frac": 1.0569, "tensor_pipe": {"est_active_frac": 0.8042}},
            "encoder": {"achieved_gbs": 510.2, "alone_gbs": 1193.0, "peak_gbs": 6547.8}}
    out = bench.summary(line)
    assert out["headline_reads_s"] == 42550.0 and out["tensor_pipe_est"] == 0.804
    assert "C4_serving" not in out and "C2_precision" not in out
    line["serving"] = {"serving": {"reads_per_s": 205595.3, "p50_s": 1.5805, "p99_s": 2.228, "tflops": 2777.2,
                                   "tensor_pipe_est": 0.70222},
                       "serving_vs_plain": 5.409, "plain_fused_kernel": {"reads_per_s": 156342.0},
                       "top20_recall_vs_plain_reference": 1.0, "untied_misses": 0, "reads": 967725}
    sv = bench.summary(line)["C4_serving"]
    assert sv["tensor_pipe_est"] == 0.702 and sv["tflops"] == 2777.0 and sv["vs_plain_fused_kernel"] == 1.32
    del line["serving"]["serving"]["tensor_pipe_est"]  # no clock samples: reported as null
    assert bench.summary(line)["C4_serving"]["tensor_pipe_est"] is None
    assert list(bench.summary(line))[-1] == "C4_serving"
