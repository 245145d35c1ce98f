"""Tile-shape autotuner: the counterpart of GPUSimulators/Autotuner.py.

The reference sweeps CUDA block widths and heights 8..31 on a 2048^2 cosine
bump, times ten launches with CUDA events and caches the fastest
configuration per host in an .npz file (GPUSimulators/Autotuner.py:35-142).
(As shipped it calls a method the simulators no longer have, so it cannot
run; see GPUSimulators/Autotuner.py:192,197.)

Here the tunable parameter is the tile configuration of each scheme's stage
kernel (tile width/height and threads per CTA, the entries of libfvgpu's
kernel table).  ``benchmark_tiles()`` times every configuration of a scheme
on the GPU with fv_sim_advance's CUDA-event timing and stores the fastest one
per (device name, scheme, size class) in a JSON cache; ``get_tile()`` is what
the simulators consult at construction.

The reference's own interface is kept beside it and works: ``Autotuner(nx,
ny, block_widths, block_heights)``, ``benchmark(simulator, force)``,
``get_peak_performance(simulator)`` (the fastest tile's width and height as
``block_width``/``block_height`` and its megacells per second), and the static
``run_benchmark``, ``gen_test_data`` and ``sanity_check``.  Block ranges are
accepted and ignored: the tile shapes are the library's own.
"""

from __future__ import annotations

import json
import logging
import os
import time

import numpy as np

# Number of tile configurations per scheme in libfvgpu's kernel table.
TILE_CONFIGS = {
    "KP07_dimsplit": 11,
    "HLL2": 11,
    "WAF": 11,
    "FORCE": 4,
    "HLL": 4,
    "EE2D_KP07_dimsplit": 10,
    "LxF": 4,
    "KP07": 4,
}
# Tile configurations of the batched kernels per scheme.
BATCH_TILE_CONFIGS = {
    "LxF": 2,
    "KP07": 2,
    "KP07_dimsplit": 7,
    "HLL": 4,
    "EE2D_KP07_dimsplit": 4,
    "HLL2": 4,
    "WAF": 4,
    "FORCE": 3,
}

DEFAULT_CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "autotuning_data.json")


def size_class(nx: int, ny: int) -> str:
    """Grids are grouped by cell count into powers of four (64^2, 128^2, ...)."""
    cells = max(1, int(nx) * int(ny))
    k = int(round(np.log(cells) / np.log(4.0)))
    return "4^%d" % k


class Autotuner(object):
    def __init__(self, nx=2048, ny=2048, block_widths=range(8, 32, 1), block_heights=range(8, 32, 1),
                 cache_file=None):
        self.logger = logging.getLogger(__name__)
        self.cache_file = cache_file or os.environ.get("FVGPU_AUTOTUNE_CACHE", DEFAULT_CACHE)
        self._cache = None
        self.nx, self.ny = int(nx), int(ny)
        self.block_widths, self.block_heights = block_widths, block_heights
        self.performance = {}
        self._context = None

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

    def benchmark_tiles(self, context, scheme, nx, ny, steps=20, warmup=5):
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


    # -- the reference's interface (GPUSimulators/Autotuner.py:35-287)

    def _ctx(self):
        if self._context is None:
            from .CudaContext import CudaContext

            self._context = CudaContext(autotuning=False)
        return self._context

    def benchmark(self, simulator, force=False):
        """Benchmark the scheme of simulator class `simulator` on an nx x ny grid
        and cache its fastest tile, unless already cached (or `force`)
        (GPUSimulators/Autotuner.py:48-98)."""
        key = simulator.__name__
        ctx = self._ctx()
        cached = self._load().get(ctx.device_name, {}).get(key, {}).get(size_class(self.nx, self.ny))
        if cached is not None and not force:
            self.logger.info("%s already benchmarked - skipping", key)
            return
        self.benchmark_tiles(ctx, key, self.nx, self.ny)
        self.performance.pop(key, None)

    def get_peak_performance(self, simulator):
        """{"block_width", "block_height", "megacells"} of the fastest tile for
        `simulator` at nx x ny, benchmarking first if needed
        (GPUSimulators/Autotuner.py:104-146)."""
        key = simulator.__name__
        if key in self.performance:
            return self.performance[key]
        ctx = self._ctx()
        entry = self._load().get(ctx.device_name, {}).get(key, {}).get(size_class(self.nx, self.ny))
        if entry is None:
            self.benchmark(simulator)
            entry = self._load()[ctx.device_name][key][size_class(self.nx, self.ny)]
        from . import SCHEMES

        cls = SCHEMES[key]
        tuner, ctx.autotuner = ctx.autotuner, _Fixed(int(entry["tile"]))
        try:  # the tile's shape, from a small simulator built with it
            q = [np.ones((8, 8), np.float32), np.zeros((8, 8), np.float32), np.zeros((8, 8), np.float32)]
            if key == "EE2D_KP07_dimsplit":
                sim = cls(ctx, *q, np.full((8, 8), 6.25, np.float32), 8, 8, 1.0, 1.0, 0.0, 1.4)
            else:
                sim = cls(ctx, *q, 8, 8, 1.0, 1.0, 9.81)
            info = sim.tile_info()
            del sim
        finally:
            ctx.autotuner = tuner
        self.performance[key] = {"block_width": info["tile_w"], "block_height": info["tile_h"],
                                 "megacells": self.nx * self.ny / (float(entry["ms_per_step"]) * 1e-3) / 1e6}
        return self.performance[key]

    @staticmethod
    def run_benchmark(simulator, arguments, timesteps=10, warmup_timesteps=2):
        """Megacells per second of `simulator(**arguments)` stepping with the
        arguments' dt, or NaN if it cannot be built or its state leaves the
        sanity bounds (GPUSimulators/Autotuner.py:175-222).  The reference steps
        with a method its simulators no longer have; here step() is used."""
        args = dict(arguments)
        dt = args.pop("dt", None)
        try:
            sim = simulator(**args)
        except Exception:
            logging.getLogger(__name__).debug("Failed creating %s with arguments %s", simulator.__name__, args)
            return np.nan
        if dt is None:
            dt = sim.computeDt() * sim.cfl_scale
        for _ in range(warmup_timesteps):
            sim.step(dt)
        sim.synchronize()
        t0 = time.perf_counter()
        for _ in range(timesteps):
            sim.step(dt)
        sim.synchronize()
        elapsed = time.perf_counter() - t0
        megacells = (sim.nx * sim.ny * timesteps / 1e6) / elapsed
        h, hu, hv = sim.download()[:3]
        sane = (Autotuner.sanity_check(h, 0.3, 0.7) and Autotuner.sanity_check(hu, -0.2, 0.2)
                and Autotuner.sanity_check(hv, -0.2, 0.2))
        return megacells if sane else np.nan

    @staticmethod
    def gen_test_data(nx, ny, g):
        """The reference's benchmark case: a smooth raised-cosine bump of depth
        and momentum on a 100 x 100 domain, with the time step of Courant
        number 0.7 for its largest expected wave speed
        (GPUSimulators/Autotuner.py:226-265).  Returns (h, hu, hv, dx, dy, dt)."""
        width = height = 100.0
        dx, dy = width / float(nx), height / float(ny)
        size = width / 5.0
        x = (dx * (np.arange(0, nx, dtype=np.float32) + 0.5) - dx * nx / 2.0) / size
        y = (dy * (np.arange(0, ny, dtype=np.float32) + 0.5) - dy * ny / 2.0) / size
        xv, yv = np.meshgrid(x, y, sparse=False, indexing="xy")
        r = np.minimum(1.0, np.sqrt(xv ** 2 + yv ** 2))
        bump = 0.1 * 0.5 * (1.0 + np.cos(np.pi * r))
        h = 0.5 + bump
        hu = bump
        hv = bump.copy()
        dt = 0.7 * min(dx, dy) / (0.1 * np.sqrt(2.0) + np.sqrt(g * 0.6))
        return h, hu, hv, dx, dy, dt

    @staticmethod
    def sanity_check(variable, bound_min, bound_max):
        """False if `variable` has a NaN or leaves [bound_min, bound_max]."""
        maxval, minval = np.amax(variable), np.amin(variable)
        return not (np.isnan(maxval) or np.isnan(minval) or maxval > bound_max or minval < bound_min)


class _Fixed(object):
    """Autotuner stand-in that forces one tile configuration."""

    def __init__(self, tile):
        self.tile = tile

    def get_tile(self, scheme, nx, ny, device_name=None):
        return self.tile
