"""Tile-shape autotuner: the counterpart of GPUSimulators/Autotuner.py.

The reference sweeps CUDA block widths and heights 8..31 on a 2048^2 cosine
bump, times ten launches with CUDA events and caches the fastest
configuration per host in an .npz file (GPUSimulators/Autotuner.py:35-142).
(As shipped it calls a method the simulators no longer have, so it cannot
run; see GPUSimulators/Autotuner.py:192,197.)

Here the tunable parameter is the tile configuration of each scheme's stage
kernel (tile width/height and threads per CTA, the entries of libfvgpu's
kernel table).  ``benchmark()`` times every configuration of a scheme on the
GPU with fv_sim_advance's CUDA-event timing and stores the fastest one per
(device name, scheme, size class) in a JSON cache; ``get_tile()`` is what the
simulators consult at construction.
"""

from __future__ import annotations

import json
import logging
import os
import time

import numpy as np

# Number of tile configurations per scheme in libfvgpu's kernel table.
TILE_CONFIGS = {
    "KP07_dimsplit": 4,
    "HLL2": 3,
    "WAF": 3,
    "FORCE": 3,
    "HLL": 4,
    "EE2D_KP07_dimsplit": 4,
    "LxF": 4,
    "KP07": 4,
}
# Tile configurations of the batched (persistent) kernels per scheme.
BATCH_TILE_CONFIGS = {
    "KP07_dimsplit": 4,
    "HLL": 4,
    "EE2D_KP07_dimsplit": 3,
    "HLL2": 3,
    "WAF": 3,
    "FORCE": 3,
}

DEFAULT_CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "autotuning_data.json")


def size_class(nx: int, ny: int) -> str:
    """Grids are grouped by cell count into powers of four (64^2, 128^2, ...)."""
    cells = max(1, int(nx) * int(ny))
    k = int(round(np.log(cells) / np.log(4.0)))
    return "4^%d" % k


class Autotuner(object):
    def __init__(self, cache_file=None):
        self.logger = logging.getLogger(__name__)
        self.cache_file = cache_file or os.environ.get("FVGPU_AUTOTUNE_CACHE", DEFAULT_CACHE)
        self._cache = None

    def _load(self):
        if self._cache is None:
            self._cache = {}
            if os.path.isfile(self.cache_file):
                try:
                    with open(self.cache_file) as f:
                        self._cache = json.load(f)
                except (OSError, ValueError):
                    self.logger.warning("ignoring unreadable autotuner cache %s", self.cache_file)
        return self._cache

    def get_tile(self, scheme, nx, ny, device_name="NVIDIA B200"):
        """Tile configuration index for a simulation, or -1 for the scheme default."""
        entry = self._load().get(device_name, {}).get(scheme, {})
        best = entry.get(size_class(nx, ny))
        if best is None and entry:
            # nearest size class that was tuned
            k = int(size_class(nx, ny).split("^")[1])
            keys = sorted(entry, key=lambda s: abs(int(s.split("^")[1]) - k))
            best = entry[keys[0]]
        return int(best["tile"]) if best is not None else -1

    def get_batch_tile(self, scheme, device_name="NVIDIA B200"):
        """Tile configuration of the batched kernel, or -1 for the default."""
        best = self._load().get(device_name, {}).get("batch:" + scheme)
        return int(best["tile"]) if best is not None else -1

    def benchmark_batch(self, context, scheme, scenarios, steps=40):
        """Time every batched-kernel tile configuration on a list of scenarios
        (variables, nx, ny, dx, dy) and record the fastest.  Returns {tile: ms per step}."""
        from .batch import Batch

        results = {}
        for tile in range(BATCH_TILE_CONFIGS[scheme]):
            b = Batch(context, scheme, tile=tile, max_instances=len(scenarios) + 1,
                      g=0.0 if scheme == "EE2D_KP07_dimsplit" else 9.81)
            for (q, nx, ny, dx, dy) in scenarios:
                b.add(q, nx, ny, dx, dy, 1e30)
            b.run(4)
            b.sync()
            b.run(steps)
            b.sync()
            results[tile] = b.info()["last_run_ms"] / steps
            del b
        best = min(results, key=results.get)
        cache = self._load()
        cache.setdefault(context.device_name, {})["batch:" + scheme] = {
            "tile": best, "ms_per_step": results[best], "all": {str(k): v for k, v in results.items()},
            "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime())}
        with open(self.cache_file, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
        return results

    def benchmark(self, context, scheme, nx, ny, steps=20, warmup=5):
        """Time every tile configuration of `scheme` on an nx x ny dam break and
        record the fastest.  Returns {tile: ms_per_step}."""
        from . import SCHEMES

        cls = SCHEMES[scheme]
        rng = np.random.default_rng(0)
        y, x = np.mgrid[0:ny, 0:nx]
        r = np.hypot(x - nx / 2.0, y - ny / 2.0)
        h = np.where(r < 0.2 * min(nx, ny), 1.0, 0.1).astype(np.float32)
        z = np.zeros_like(h)
        results = {}
        for tile in range(TILE_CONFIGS[scheme]):
            self._forced_tile = tile
            ctx_tuner = context.autotuner
            context.autotuner = _Fixed(tile)
            try:
                if scheme == "EE2D_KP07_dimsplit":
                    E = (2.5 / 0.4 + 0.0 * h).astype(np.float32)
                    sim = cls(context, h + 1.0, z, z, E, nx, ny, 1.0 / nx, 1.0 / ny, 0.0, 1.4)
                else:
                    sim = cls(context, h, z, z, nx, ny, 1.0, 1.0, 9.81)
                sim.advance(warmup)
                sim.advance(steps)
                results[tile] = sim.last_advance_ms()
                del sim
            finally:
                context.autotuner = ctx_tuner
        best = min(results, key=results.get)
        cache = self._load()
        cache.setdefault(context.device_name, {}).setdefault(scheme, {})[size_class(nx, ny)] = {
            "tile": best,
            "ms_per_step": results[best],
            "all": {str(k): v for k, v in results.items()},
            "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()),
        }
        with open(self.cache_file, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
        return results


class _Fixed(object):
    """Autotuner stand-in that forces one tile configuration."""

    def __init__(self, tile):
        self.tile = tile

    def get_tile(self, scheme, nx, ny, device_name=None):
        return self.tile
