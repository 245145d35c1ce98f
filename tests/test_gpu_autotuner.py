"""The autotuner's reference interface on the GPU (GPUSimulators/Autotuner.py:
48-222): benchmark(simulator), get_peak_performance(simulator) and
run_benchmark(simulator, arguments)."""

import os

import numpy as np
import pytest

import finitevolumegpu_b200 as fv
from finitevolumegpu_b200.Autotuner import Autotuner, TILE_CONFIGS

pytestmark = pytest.mark.gpu


def test_peak_performance_and_cached_benchmark(tmp_path):
    cache = str(tmp_path / "tuning.json")
    tuner = Autotuner(nx=256, ny=256, cache_file=cache)
    peak = tuner.get_peak_performance(fv.KP07_dimsplit.KP07_dimsplit)
    assert set(peak) == {"block_width", "block_height", "megacells"}
    assert peak["block_width"] in (28, 60, 124) and peak["block_height"] in (28, 60)
    assert peak["megacells"] > 100.0  # a 256^2 step takes tens of microseconds
    mtime = os.path.getmtime(cache)
    tuner.benchmark(fv.KP07_dimsplit.KP07_dimsplit)  # cached: nothing to do
    assert os.path.getmtime(cache) == mtime
    assert len(Autotuner(cache_file=cache)._load()["NVIDIA B200"]["KP07_dimsplit"]["4^8"]["all"]) == \
        TILE_CONFIGS["KP07_dimsplit"]


def test_run_benchmark_with_reference_arguments(ctx):
    h, hu, hv, dx, dy, dt = Autotuner.gen_test_data(nx=512, ny=512, g=9.81)
    arguments = {"context": ctx, "h0": h, "hu0": hu, "hv0": hv, "nx": 512, "ny": 512, "dx": dx, "dy": dy,
                 "dt": 0.9 * dt, "g": 9.81, "block_width": 16, "block_height": 16}
    megacells = Autotuner.run_benchmark(fv.KP07_dimsplit.KP07_dimsplit, arguments)
    assert np.isfinite(megacells) and megacells > 0.0
    # a case that cannot be built gives NaN, as in the reference
    bad = dict(arguments, nx=-1)
    assert np.isnan(Autotuner.run_benchmark(fv.KP07_dimsplit.KP07_dimsplit, bad))
