"""bench.py pieces that run on host cores (CPU).

The reference arm (`bench.py --impl reference`) times the reference's own CPU
build on the bench's operator and must print one JSON line with the GPU arm's
metric and direction, a config and unit naming the size it actually ran (n = 32:
the reference needs hours at n = 128), the number of steps it actually timed, a
cpu_baseline describing the run and an e2e entry without host-device traffic.
The serving arrivals are a seeded Poisson process whose mix the workload
description states.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import bench

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not os.path.exists(bench.REF_PROBE),
                    reason="reference CPU build absent (make -C oracle)")
def test_reference_arm_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "0"],
                         capture_output=True, text=True, timeout=600, check=True).stdout
    line = json.loads(out.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC
    n = bench.REF_N
    assert line["unit"] == f"factor+solve steps/s at n={n}" and line["higher_is_better"] is True
    cfg = line["config"]
    for k, v in bench.workload_config(n, 1e-6, 1).items():
        assert cfg[k] == v
    assert f"n={n} " in cfg["workload"]
    assert line["steps"] == 1 and line["requested_steps"] == 1
    assert line["value"] > 0 and line["ms_per_step"] == pytest.approx(1e3 / line["value"])
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == line["value"]
    assert "not scaled" in cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"],
                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    # the reference's own per-level times, every level of the n = 32 factorization
    assert [lv["level"] for lv in line["per_level_s"]] == [0, 1, 2, 3]


def test_serving_schedule_is_seeded_poisson_with_the_stated_mix():
    a = bench.serving_schedule(400, 8.0)
    b = bench.serving_schedule(400, 8.0)
    assert a == b
    arr = np.array([x[0] for x in a])
    assert np.all(np.diff(arr) >= 0)
    assert 400 / arr[-1] == pytest.approx(8.0, rel=0.15)  # mean rate
    n_factor = sum(1 for x in a if x[1] == "factor")
    assert 0.22 < n_factor / 400 < 0.38  # 30% factorizations


def test_bench_field_has_the_stated_correlation_length():
    """The bench's coefficient field a = exp(g): g has standard deviation 1 and
    correlation exp(-d^2 / (2 l^2)) with l = 1/16 of the unit cube."""
    from hifde3d_b200 import synth

    N = 63
    NC = N + 1
    assert bench.GRF_CORRELATION == 1.0 / 16
    vals = {1: [], 2: [], 4: []}
    for seed in range(3):
        ax, _, _ = synth.face_coefficients_grf(N, seed, bench.GRF_ELL_PARAM, 1.0)
        g = np.log(ax)
        for q in vals:
            vals[q].append(np.mean(g * np.roll(g, -q, axis=0)) / np.mean(g * g))
    ell = bench.GRF_CORRELATION
    for q, v in vals.items():
        d = q / NC
        assert np.mean(v) == pytest.approx(np.exp(-d * d / (2 * ell * ell)), abs=0.04)
