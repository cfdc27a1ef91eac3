"""The bench's host-side bookkeeping (no GPU): the byte model behind the roofline record, the
per-kernel event sums, the reference full-scan cotangent and the default command line."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent.parent))

import bench  # noqa: E402


def test_algorithmic_bytes_per_sample_follow_the_kernels_reads_and_writes():
    # FP32 storage: eight 4-byte corners read; the volume scatter writes 32 bytes of increments
    assert bench.algorithmic_bytes("forward", 4) == 32
    assert bench.algorithmic_bytes("forward_moments", 4) == 32
    assert bench.algorithmic_bytes("vjp_volume", 4) == 32
    assert bench.algorithmic_bytes("vjp", 4) == 64
    assert bench.algorithmic_bytes("vjp_pose", 2) == 16  # BF16 corners
    assert bench.algorithmic_bytes("fold", 4) == 0  # not a sampling launch


class _Event:
    def __init__(self, t: float) -> None:
        self.t = t

    def elapsed_time(self, end: "_Event") -> float:
        return end.t - self.t


def test_kernel_times_and_as_built_bytes_from_a_launch_log():
    realised = np.array([10, 20, 30, 40], dtype=np.int64)  # per view
    log = [("forward_moments", 0, 4, _Event(0.0), _Event(5.0)),
           ("vjp_volume", 0, 2, _Event(5.0), _Event(7.0)),
           ("vjp_volume", 2, 2, _Event(7.0), _Event(10.0)),
           ("fold", 0, 4, _Event(10.0), _Event(10.5))]
    times, samples = bench.kernel_times(log, realised)
    assert times == {"forward_moments": [5.0], "vjp_volume": [2.0, 3.0], "fold": [0.5]}
    assert samples == {"forward_moments": [100], "vjp_volume": [30, 70], "fold": [100]}
    # one step: 100 samples x 32 B (forward) + 100 x 32 B (scatter); the fold adds nothing
    assert bench.as_built_bytes(samples, 4, steps=1) == 6400
    assert bench.as_built_bytes(samples, 4, steps=2) == 3200


@pytest.mark.parametrize("views", [[0, 45, 90, 135, 180, 225, 270, 315], [0, 1, 2]])
def test_reference_cotangent_is_the_l1_normalised_full_scan_formula(views):
    total, rows, cols = 360, 6, 5
    cot = bench.reference_cotangent(views, rows, cols, total)
    assert cot.shape == (len(views), rows, cols) and cot.dtype == np.float32
    assert np.all(cot > 0)
    assert abs(float(np.abs(cot.astype(np.float64)).sum()) - 1.0) < 1e-6
    # the formula at one pixel, before the normalisation
    k, r, c = 1, 2, 3
    theta = 2 * np.pi * views[k] / total
    rr, cc = 2 * (r + 0.5) / rows - 1, 2 * (c + 0.5) / cols - 1
    raw = 1 + 0.2 * np.sin(theta) + 0.1 * np.cos(2 * theta) + 0.15 * rr + 0.1 * cc + 0.05 * np.sin(theta) * cc
    ratio = float(cot[k, r, c]) / float(cot[0, 0, 0])
    theta0 = 2 * np.pi * views[0] / total
    r0, c0 = 2 * 0.5 / rows - 1, 2 * 0.5 / cols - 1
    raw0 = 1 + 0.2 * np.sin(theta0) + 0.1 * np.cos(2 * theta0) + 0.15 * r0 + 0.1 * c0 + 0.05 * np.sin(theta0) * c0
    assert ratio == pytest.approx(raw / raw0, rel=1e-6)


def test_default_command_line_is_the_headline_run(monkeypatch):
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    args = bench.parse()
    assert (args.gpus, args.views, args.size, args.detector, args.samples) == (1, 360, 256, 512, 1024)
    assert args.storage == "float32" and args.mode == "iteration" and args.impl == "dpt_b200"
    assert args.warmup >= 3
