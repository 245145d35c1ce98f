"""Benchmark of the GPUSimulators time-step path on B200.

Workload: KP07_dimsplit shallow water on a 4096 x 4096 FP32 grid, circular dam
break (h = 1 inside a seeded radius R ~ U(0.1, 0.3) * width, 0.1 outside,
hu = hv = 0, g = 9.81, reflective walls), stepped with simulate()'s CFL
schedule (dt recomputed every 100 steps).  One bench step is one full time
step (two stage-kernel launches).  The state (2 x 201 MB) is larger than L2,
so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mine|reference]

N > 1 (launched with torch.distributed.run) runs one independent replica per
GPU (the path does not shard: weak scaling, no collective on the data path).
``--impl reference`` times the reference algorithm on the host CPU (the CPU
restatement of the reference kernels; the reference itself has no CPU path),
on rank 0 only.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time
import traceback

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX = NY = 4096  # may be overridden by --size (profiling captures use a smaller grid)
SCHEME = "KP07_dimsplit"
BYTES_PER_CELL_SUBSTEP = 24  # 3 FP32 variables read + written per stage launch
SUBSTEPS = 2
# Algorithmic floating-point operations per cell and stage launch (averaged
# over the launches of a step) of each scheme as the reference formulates it:
# +, -, *, /, sqrt, min, max counted once each ("flops"), of which divisions and
# square roots ("mufu").  Counted by running the CPU restatement with an
# operation-counting number type (oracle.oracle.ops_per_cell_substep);
# tests/test_flop_count.py checks these figures against that count.
ALG_OPS_PER_CELL_LAUNCH = {
    "LxF": {"flops": 123.0, "mufu": 21.0},
    "FORCE": {"flops": 184.0, "mufu": 30.0},
    "HLL": {"flops": 164.0, "mufu": 38.0},
    "HLL2": {"flops": 484.0, "mufu": 56.0},
    "WAF": {"flops": 506.0, "mufu": 88.0},
    "KP07": {"flops": 474.0, "mufu": 39.0},
    "KP07_dimsplit": {"flops": 450.0, "mufu": 46.0},
    "EE2D_KP07_dimsplit": {"flops": 585.0, "mufu": 51.0},
}
# FP32 FLOP per cell and stage launch that this library's kernels execute
# (FMA = 2), measured with ncu's sass op counters on a 3072^2 dam break
# (profiles/flop_crosscheck_3072.md): each cell is reconstructed once per
# sweep and each face flux computed once, so the kernels need half the
# reference formulation's operations.  Packing two lines per instruction
# (f32x2) does the same operations in fewer instructions.
EXECUTED_FLOP_PER_CELL_LAUNCH = {"LxF": 66.0, "FORCE": 118.0, "HLL": 130.0, "HLL2": 233.0, "WAF": 354.0,
                                 "KP07": 172.0, "KP07_dimsplit": 215.0, "EE2D_KP07_dimsplit": 321.0}
# The same counts as FP32 pipe operations (fadd + fmul + ffma per cell and
# launch, one FMA-pipe lane slot each): an add or a multiply occupies a lane
# as long as an FMA does, so these, not the FLOPs, set the FP32 pipe's floor.
FP32_PIPE_OPS_PER_CELL_LAUNCH = {"LxF": 54.0, "FORCE": 95.0, "HLL": 105.0, "HLL2": 171.0, "WAF": 308.0,
                                 "KP07": 138.0, "KP07_dimsplit": 159.0, "EE2D_KP07_dimsplit": 235.0}
FP32_LANES_PER_SM = 128  # FP32 FMA lanes per Blackwell SM
PROFILE_JSON = os.path.join(ROOT, "profiles", "kp07_dimsplit_stage_4096.json")


def dam_break_4096(seed=0):
    rng = np.random.default_rng(seed)
    R = rng.uniform(0.1, 0.3) * NX
    y, x = np.mgrid[0:NY, 0:NX] + 0.5
    r = np.hypot(x - NX / 2.0, y - NY / 2.0)
    h = np.where(r < R, 1.0, 0.1).astype(np.float32)
    z = np.zeros_like(h)
    return h, z, z.copy(), float(R)


class ClockSampler:
    """Samples SM clock and throttle reasons through NVML during the timed region."""

    REASONS = {
        0x0000000000000004: "sw_power_cap",
        0x0000000000000008: "hw_slowdown",
        0x0000000000000020: "sw_thermal_slowdown",
        0x0000000000000040: "hw_thermal_slowdown",
        0x0000000000000080: "hw_power_brake_slowdown",
    }

    def __init__(self, device_index=0, period=0.005):
        self.period = period
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self._stop = threading.Event()
        self._ok = False
        try:
            import pynvml

            pynvml.nvmlInit()
            self._nv = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
            self._ok = True
        except Exception:
            self._ok = False

    def _run(self):
        nv = self._nv
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
                fn = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                    nv.nvmlDeviceGetCurrentClocksThrottleReasons
                mask = fn(self._h)
                for bit, name in self.REASONS.items():
                    if mask & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(self.period)

    def __enter__(self):
        if self._ok:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        if self._ok:
            self._stop.set()
            self._t.join()

    def summary(self):
        if not self._ok or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unavailable"]}
        return {"sm_mhz": float(statistics.median(self.samples)), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0}, "fallback"


def load_profile():
    try:
        with open(PROFILE_JSON) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def aux_leg(fn, *args, **kwargs):
    """Runs one of the measurements beside the headline (batched, served, CPU
    baseline).  A failure is reported in its place in the JSON line, with the
    traceback on stderr, instead of taking the headline measurement with it."""
    try:
        return fn(*args, **kwargs)
    except Exception as e:
        traceback.print_exc()
        return {"error": "%s: %s" % (type(e).__name__, e)}


def cpu_baseline_leg(steps=3):
    """FP64 CPU oracle on the host cores: a bounded sample of the workload."""
    from oracle.oracle import OracleSim

    h, hu, hv, _ = dam_break_4096()
    cores = len(os.sched_getaffinity(0))
    sim = OracleSim(SCHEME, [h, hu, hv], NX, NY, 1.0, 1.0, 9.81, dtype=np.float64, nthreads=cores)
    dt = sim.computeDt() * 0.9
    t0 = time.perf_counter()
    for _ in range(steps):
        sim.step(dt)
    el = time.perf_counter() - t0
    return {"value": NX * NY * steps / el, "unit": "cell-updates/s", "cores": cores, "kind": "port",
            "sample": "%d steps of the full 4096x4096 grid, FP64 C restatement (OpenMP, %d threads)" % (steps, cores)}


def run_reference(args, rank, world, budget_s=120.0):
    """The reference algorithm on the host CPU (FP32 oracle), rank 0 only.

    Each step is one KP07_dimsplit time step of the full 4096 x 4096 grid when
    the --steps/--warmup run of that fits in about `budget_s` seconds of host
    time; otherwise of the widest centred stripe that does (measured on one
    calibration step of the full grid), and config.workload says which."""
    if rank != 0:
        return None
    from oracle.oracle import OracleSim

    cores = len(os.sched_getaffinity(0))
    h, hu, hv, _ = dam_break_4096()

    def make(rows):
        r0 = NY // 2 - rows // 2
        q = [a[r0:r0 + rows].copy() for a in (h, hu, hv)]
        return OracleSim(SCHEME, q, NX, rows, 1.0, 1.0, 9.81, dtype=np.float32, nthreads=cores)

    sim = make(NY)
    dt = sim.computeDt() * 0.9
    t0 = time.perf_counter()
    sim.step(dt)  # calibration (and first warm-up) step of the full grid
    full_s = time.perf_counter() - t0
    n = max(1, args.steps + args.warmup - 1)
    rows = NY
    if n * full_s > budget_s:
        rows = max(64, min(NY, int(NY * budget_s / (n * full_s)) // 8 * 8))
        sim = make(rows)
    for _ in range(args.warmup - 1):
        sim.step(dt)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sim.step(dt)
    el = time.perf_counter() - t0
    v = NX * rows * args.steps / el
    what = "the full 4096x4096 grid" if rows == NY else "a centred 4096x%d stripe of the 4096x4096 grid" % rows
    sample = "each step: one KP07_dimsplit time step of %s (dam break), FP32 C restatement, %d threads" % (what, cores)
    return {
        "metric": "cell-updates/s", "value": v, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
        "config": {"workload": "KP07_dimsplit circular dam break, CPU: %s per step" % what,
                   "scheme": SCHEME, "nx": NX, "ny": rows, "parallelism": "host threads"},
        "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def reference_kernels_leg(my_ms_per_step, steps=40, warmup=5):
    """The reference's own KP07_dimsplit kernel (its CUDA source compiled
    unmodified for sm_100a) on the same 4096 x 4096 dam break on this GPU,
    at the fastest of its default block and the other built block shapes:
    CUDA events around `steps` steps of fixed dt (its kernel launches and
    buffer swaps), against this library's ms per step."""
    from oracle import ref_kernels

    h, hu, hv, _ = dam_break_4096()
    per_block = {}
    for block in [None] + list(ref_kernels.BLOCKS):
        if not ref_kernels.available(SCHEME, block):
            continue
        ref = ref_kernels.RefKernelSim(SCHEME, [h, hu, hv], NX, NY, 1.0, 1.0, 9.81, block=block)
        dt = np.float32(ref.computeDt() * np.float32(0.9))
        ref.time_steps(warmup, dt)
        per_block["%dx%d" % (ref.bw, ref.bh)] = ref.time_steps(steps, dt)
        ref.close()
    best = min(per_block, key=per_block.get)
    ms = per_block[best]
    return {"what": "reference KP07DimsplitKernel, CUDA source compiled unmodified for sm_100a, same input and GPU",
            "ms_per_step": ms, "block": best, "ms_per_step_by_block": per_block,
            "cell_updates_per_s": NX * NY / (ms * 1e-3), "speedup_of_this_library": ms / my_ms_per_step}


# The initial-state generators below feed the served leg's client threads (one
# state per request, made just before its admission), so they are written to
# cost little per cell: the served rate would otherwise measure the load
# generator.  Each gives the same bits as the plain full-grid formula in its
# docstring (tests/test_bench_logic.py compares them).

# Beyond this many cells from its centre a bump's exp(-r^2 / 800) is below
# 2^-65, so 1 + A * exp(...) rounds to exactly 1.0 in FP64.
BUMP_REACH = 200.0


def bump_ic(nx, ny, rng):
    """Gaussian bump: h = 1 + A exp(-r^2/(2 sigma^2)), A ~ U(0.1, 0.5), centre ~ U(0.3, 0.7) x domain, sigma = 20 cells.
    Full-grid formula: h = float32(1.0 + A * exp(-((x - cx)^2 + (y - cy)^2) / (2 * 20^2))) with x, y the FP32
    cell centres; evaluated only within BUMP_REACH cells of the centre, 1.0 elsewhere."""
    A = rng.uniform(0.1, 0.5)
    cx, cy = rng.uniform(0.3, 0.7) * nx, rng.uniform(0.3, 0.7) * ny
    x = np.arange(nx, dtype=np.float32) + 0.5
    y = np.arange(ny, dtype=np.float32) + 0.5
    x0, x1 = np.searchsorted(x, cx - BUMP_REACH), np.searchsorted(x, cx + BUMP_REACH, side="right")
    y0, y1 = np.searchsorted(y, cy - BUMP_REACH), np.searchsorted(y, cy + BUMP_REACH, side="right")
    h = np.ones((ny, nx), np.float32)
    xs, ys = x[x0:x1], y[y0:y1]
    h[y0:y1, x0:x1] = 1.0 + A * np.exp(-((xs[None, :] - cx) ** 2 + (ys[:, None] - cy) ** 2) / (2 * 20.0 ** 2))
    z = np.zeros((ny, nx), np.float32)
    return [h, z, z.copy()]


def dam_ic(nx, ny, rng):
    """Circular dam break: h = 1 inside R ~ U(0.1, 0.3) x width of the centre, 0.1 outside.
    Full-grid formula: h = where(x^2 + y^2 < R^2, 1.0, 0.1) in FP32, x, y the FP32 offsets of the cell
    centres from the domain centre."""
    R = rng.uniform(0.1, 0.3) * nx
    x = np.arange(nx, dtype=np.float32) + 0.5 - nx / 2.0
    y = np.arange(ny, dtype=np.float32) + 0.5 - ny / 2.0
    h = np.where(x[None, :] ** 2 + y[:, None] ** 2 < R * R, np.float32(1.0), np.float32(0.1))
    z = np.zeros((ny, nx), np.float32)
    return [h, z, z.copy()]


def kh_ic(nx, ny, rng, gamma=1.4):
    """Kelvin-Helmholtz: rho = 2, u = +0.5 in the middle half band, rho = 1, u = -0.5 outside, p = 2.5,
    v = 0.01 sin(4 pi x + phi) with seeded phase.  Full-grid formula, in FP64 then rounded to FP32:
    (rho, rho u, rho v, E) with E = p / (gamma - 1) + 0.5 rho (u^2 + v^2).  Every row of the band (and every
    row outside it) is the same, so the two distinct rows are computed and repeated."""
    phi = rng.uniform(0, 2 * np.pi)
    yy = (np.arange(ny, dtype=np.float32) + 0.5) / ny
    xx = (np.arange(nx, dtype=np.float32) + 0.5) / nx
    band = ((yy >= 0.25) & (yy < 0.75))[:, None]
    v = 0.01 * np.sin(4 * np.pi * xx[None, :] + phi)
    rows = []
    for r0, u0 in ((2.0, 0.5), (1.0, -0.5)):
        rho = np.full((1, nx), r0)
        u = np.full((1, nx), u0)
        E = 2.5 / (gamma - 1.0) + 0.5 * rho * (u ** 2 + v ** 2)
        rows.append([a.astype(np.float32) for a in (rho, rho * u, rho * v, E)])
    return [np.where(band, a, b) for a, b in zip(rows[0], rows[1])]


def run_batched(ctx, n_inst=512, seed=4, check=8):
    """Config 4: 512 KP07_dimsplit simulations, sides log-uniform in [64, 1024], bump or dam break,
    t_end ~ U(5, 50): one batch (one batched launch per substep, CUDA graphs) vs the plain simulators one after another."""
    from finitevolumegpu_b200 import KP07_dimsplit
    from finitevolumegpu_b200.batch import Batch

    rng = np.random.default_rng(seed)
    cases = []
    for i in range(n_inst):
        nx = int(round(np.exp(rng.uniform(np.log(64), np.log(1024)))))
        ny = int(round(np.exp(rng.uniform(np.log(64), np.log(1024)))))
        q = bump_ic(nx, ny, rng) if rng.random() < 0.5 else dam_ic(nx, ny, rng)
        cases.append((q, nx, ny, float(rng.uniform(5.0, 50.0))))
    # Warm-up: one untimed admission of the whole workload grows the device
    # memory pool and the pinned staging ring once, as a long-running service
    # would have them; the plain path below runs with the same warm pool.
    import torch

    w = Batch(ctx, "KP07_dimsplit", max_instances=n_inst)
    for (q, nx, ny, t_end) in cases:
        w.add(q, nx, ny, 1.0, 1.0, t_end)
    w.sync()
    del w
    # batched: admit all, run to completion, download all
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    b = Batch(ctx, "KP07_dimsplit", max_instances=n_inst)
    slots = [b.add(q, nx, ny, 1.0, 1.0, t_end) for (q, nx, ny, t_end) in cases]
    t_add = time.perf_counter()
    dev_ms = 0.0
    steps = 0
    while True:
        b.sync()
        dev_ms += b.info()["last_run_ms"] if steps else 0.0
        if all(b.status(s)["done"] for s in slots):
            break
        b.run(16)
        steps += 16
    t_run = time.perf_counter()
    batched_out = b.download_many(slots)
    nts = [b.status(s)["nt"] for s in slots]
    t1 = time.perf_counter()
    info = b.info()
    del b
    total = sum(nx * ny * nt for (q, nx, ny, t_end), nt in zip(cases, nts))
    # plain: one simulator after the other
    t2 = time.perf_counter()
    max_diff = 0.0
    plain_nts = []
    for i, (q, nx, ny, t_end) in enumerate(cases):
        sim = KP07_dimsplit.KP07_dimsplit(ctx, q[0], q[1], q[2], nx, ny, 1.0, 1.0, 9.81)
        sim.simulate(t_end)
        out = sim.download()
        plain_nts.append(sim.simSteps())
        for a, w in zip(out, batched_out[i]):
            d = float(np.max(np.abs(a - w)))
            max_diff = max(max_diff, d)
        del sim
    t3 = time.perf_counter()
    # FP64 oracle on a sample stratified by grid size: the simulations sorted
    # by cell count are split into `check` strata, the largest grids among
    # them, and each stratum contributes its simulation with the earliest t_end
    # (which bounds the oracle's host time)
    l1 = 0.0
    from oracle.oracle import OracleSim

    order = sorted(range(n_inst), key=lambda i: cases[i][1] * cases[i][2])
    sample = [min(part, key=lambda i: cases[i][3]) for part in np.array_split(order, check)]
    checked = []
    for i in sample:
        q, nx, ny, t_end = cases[i]
        o = OracleSim("KP07_dimsplit", q, nx, ny, 1.0, 1.0, 9.81, dtype=np.float64)
        o.simulate(t_end)
        e = max(float(np.sum(np.abs(a - w)) / max(np.sum(np.abs(w)), 1e-30))
                for a, w in zip(batched_out[i], o.download()))
        l1 = max(l1, e)
        checked.append({"nx": nx, "ny": ny, "steps": o.simSteps(), "rel_l1": e})
    return {
        "workload": "512 KP07_dimsplit simulations, sides log-uniform [64,1024] (seed %d), bump or dam break, "
                    "t_end ~ U(5,50), each with its own CFL dt" % seed,
        "cell_updates": total,
        "batched_cell_updates_per_s": total / (t1 - t0),
        "batched_device_cell_updates_per_s": total / (dev_ms / 1e3) if dev_ms else None,
        "plain_cell_updates_per_s": total / (t3 - t2),
        "speedup_vs_plain": (t3 - t2) / (t1 - t0),
        "batched_s": {"admit": t_add - t0, "run": t_run - t_add, "download": t1 - t_run, "total": t1 - t0},
        "plain_s": t3 - t2,
        "steps_identical": nts == plain_nts,
        "max_abs_diff_batched_vs_plain": max_diff,
        "max_rel_l1_vs_fp64_oracle": l1,
        "oracle_checked": checked,
        "tile": {k: info[k] for k in ("tile_w", "tile_h", "threads", "grid")},
    }


class ICFeed(object):
    """The clients' side of the served stream: initial states generated on
    `threads` host threads ahead of their requests' admission (requests are
    numbered in arrival order), at most `ahead` requests past the latest one
    taken, so that the server's own threads only upload them."""

    def __init__(self, make, count, threads=4, ahead=48):
        import concurrent.futures

        self.make = make
        self.cv = threading.Condition()
        self.taken = -1  # highest request index taken so far
        self.pool = concurrent.futures.ThreadPoolExecutor(threads, thread_name_prefix="ic-feed")
        self.futures = {}
        self.ahead = ahead
        self.stop = False
        self.feeder = threading.Thread(target=self._feed, args=(count,), daemon=True)
        self.feeder.start()

    def _feed(self, count):
        for i in range(count):
            with self.cv:
                while not self.stop and i > self.taken + self.ahead:
                    self.cv.wait(0.1)
                if self.stop:
                    return
                self.futures[i] = self.pool.submit(self.make, i)
                self.cv.notify_all()

    def get(self, i):
        with self.cv:
            while i not in self.futures and i > self.taken and not self.stop:
                self.taken = max(self.taken, i - self.ahead)  # let the feeder reach i
                self.cv.notify_all()
                self.cv.wait(0.1)
            fut = self.futures.pop(i, None)
            self.taken = max(self.taken, i)
            self.cv.notify_all()
        # a retried admission (the GPU was full) takes its state a second time
        return fut.result() if fut is not None else self.make(i)

    def close(self):
        with self.cv:
            self.stop = True
            self.cv.notify_all()
        self.feeder.join()
        self.pool.shutdown(wait=True)


def run_served(ctx, n_req=10000, rates=(300.0, 600.0, 900.0, 1200.0), seed=5, plain_sample=200, warmup_req=64):
    """Config 5: scenario requests with Poisson arrivals, scheme uniform over {KP07_dimsplit, HLL, EE2D},
    sides log-uniform [128, 2048], t_end ~ U(1, 20), served with continuous batching under a 120 GB budget.
    The same scenarios are served at each arrival rate of the sweep (the last one saturates the server).
    Top-level figures: the highest rate the server sustained (it completed requests at no less than 95 % of
    the arrival rate, so its queue did not grow) with its p50/p99 latency; `capacity` is the rate of highest
    throughput (past it, arrivals only queue).
    Initial states are made from per-request seeds by client threads just ahead of admission, and each
    result is reduced on the server's return threads to per-variable sums of its bit patterns (the
    first `plain_sample` keep their arrays), so host memory stays bounded; the checksums must agree
    across the rates (each result is independent of what else was on the GPU).  A short warm-up serve first pays
    the one-time costs (memory pool and pinned staging growth)."""
    from finitevolumegpu_b200 import SCHEMES, BoundaryCondition
    from finitevolumegpu_b200.server import Request, Server

    rng = np.random.default_rng(seed)
    schemes = ["KP07_dimsplit", "HLL", "EE2D_KP07_dimsplit"]
    periodic = BoundaryCondition(BoundaryCondition.getTypes(0x02020202))
    specs = []
    for i in range(n_req):
        s = schemes[int(rng.integers(0, 3))]
        nx = int(round(np.exp(rng.uniform(np.log(128), np.log(2048)))))
        ny = int(round(np.exp(rng.uniform(np.log(128), np.log(2048)))))
        kind = "kh" if s == "EE2D_KP07_dimsplit" else ("bump" if rng.random() < 0.5 else "dam")
        specs.append((s, nx, ny, kind, float(rng.uniform(1.0, 20.0)), int(rng.integers(0, 2 ** 31))))
    gaps = np.random.default_rng(seed + 1).exponential(1.0, n_req)

    def make_ic(i):
        s, nx, ny, kind, _, icseed = specs[i]
        r = np.random.default_rng(icseed)
        # unit cells; the Euler requests are the Kelvin-Helmholtz family scaled to the grid
        return {"kh": kh_ic, "bump": bump_ic, "dam": dam_ic}[kind](nx, ny, r)

    def checksum(state):
        # per variable, the wrapping sum of its bits read as 64-bit words (and
        # the last 32-bit word of an odd count): any single changed bit shows
        out = []
        for a in state:
            w = a.reshape(-1).view(np.uint32)
            even = w.size & ~1
            out.append((int(w[:even].view(np.uint64).sum()), int(w[even:].sum())))
        return tuple(out)

    def keep(req, state):  # state lives in the return thread's reused buffer
        if req.rid < plain_sample:
            return [a.copy() for a in state]
        return checksum(state)

    def serve(rate, count=n_req):
        t = np.cumsum(gaps[:count]) / rate
        feed = ICFeed(make_ic, count)
        try:
            reqs = [Request(i, s, (lambda i=i: feed.get(i)), nx, ny, 1.0, 1.0, te, arrival=float(t[i]),
                            boundary_conditions=periodic if s == "EE2D_KP07_dimsplit" else None)
                    for i, (s, nx, ny, _, te, _) in enumerate(specs[:count])]
            return Server(ctx, budget_bytes=120e9, chunk_steps=8).serve(reqs, result_fn=keep)
        finally:
            feed.close()

    serve(1e9, warmup_req)
    sweep, sums, results = [], [], None
    for rate in rates:
        results, st = serve(rate)
        st["arrival_rate_per_s"] = rate
        sweep.append(st)
        sums.append({r.rid: (r.state if r.rid >= plain_sample else checksum(r.state))
                     for r in results if r.status == "done"})
    # top-level figures: the highest rate the server sustained (requests done
    # per second of its run >= 95 % of the arrival rate); every rate is in the
    # sweep, and `capacity` is the one of highest throughput
    def sustained(st):
        return st["requests"] / st["elapsed_s"] >= 0.95 * st["arrival_rate_per_s"]

    cap = max(sweep, key=lambda st: st["cell_updates_per_s"])
    ok = [st for st in sweep if sustained(st)]
    stats = dict(max(ok, key=lambda st: st["arrival_rate_per_s"]) if ok else cap)
    stats["sustained"] = bool(ok)
    # plain one-at-a-time path on a sample of the same requests
    by_id = {r.rid: r for r in results}
    t0 = time.perf_counter()
    cells = 0
    same = True
    for i in range(min(plain_sample, n_req)):
        s, nx, ny, _, te, _ = specs[i]
        q = make_ic(i)
        cls = SCHEMES[s]
        if s == "EE2D_KP07_dimsplit":
            sim = cls(ctx, *q, nx, ny, 1.0, 1.0, 0.0, 1.4, boundary_conditions=periodic)
        else:
            sim = cls(ctx, *q, nx, ny, 1.0, 1.0, 9.81)
        sim.simulate(te)
        out = sim.download()
        cells += nx * ny * sim.simSteps()
        same = same and by_id[i].status == "done" and all(np.array_equal(a, w) for a, w in zip(out, by_id[i].state))
        del sim
    plain_rate = cells / (time.perf_counter() - t0)
    stats.update({
        "workload": "%d requests, Poisson arrivals (seed %d) swept over %s per s, schemes KP07_dimsplit/HLL/EE2D, "
                    "sides log-uniform [128,2048], t_end ~ U(1,20), 120 GB budget; top-level figures at the "
                    "highest sustained rate, capacity at the rate of highest throughput"
                    % (n_req, seed, "/".join("%.0f" % r for r in rates)),
        "sweep": [{k: v for k, v in st.items() if k in ("arrival_rate_per_s", "requests", "rejected", "failed",
                                                        "cell_updates_per_s", "p50_latency_s", "p99_latency_s",
                                                        "mean_latency_s", "elapsed_s", "host_seconds")}
                  for st in sweep],
        "plain_one_at_a_time_cell_updates_per_s": plain_rate,
        "plain_sample_requests": min(plain_sample, n_req),
        "speedup_vs_plain": stats["cell_updates_per_s"] / plain_rate,
        "capacity": {"arrival_rate_per_s": cap["arrival_rate_per_s"],
                     "requests_per_s": cap["requests"] / cap["elapsed_s"],
                     "cell_updates_per_s": cap["cell_updates_per_s"],
                     "speedup_vs_plain": cap["cell_updates_per_s"] / plain_rate,
                     "p50_latency_s": cap["p50_latency_s"], "p99_latency_s": cap["p99_latency_s"]},
        "results_identical_to_plain": same,
        "results_identical_across_rates": all(d == sums[0] for d in sums[1:]) and len(sums[0]) == n_req,
    })
    return stats


# Algorithmic HBM bytes per cell per stage launch, averaged over the launches of
# one step: state read + written (3 or 4 FP32 variables); KP07's second RK
# stage also reads u^n, so its two launches average (24 + 36) / 2.
BYTES_PER_CELL_LAUNCH = {"LxF": 24, "FORCE": 24, "HLL": 24, "HLL2": 24, "WAF": 24, "KP07": 30,
                         "KP07_dimsplit": 24, "EE2D_KP07_dimsplit": 32}


def make_scheme_sim(ctx, scheme, seed):
    """The benchmark workload of one scheme: a seeded circular dam break on NX x NY (SWE), or the
    Kelvin-Helmholtz problem on NX x NX/2 with periodic boundaries (Euler)."""
    from finitevolumegpu_b200 import SCHEMES, BoundaryCondition

    if scheme == "EE2D_KP07_dimsplit":
        nx, ny = NX, NX // 2
        q = kh_ic(nx, ny, np.random.default_rng(seed))
        bc = BoundaryCondition(BoundaryCondition.getTypes(0x02020202))
        sim = SCHEMES[scheme](ctx, q[0], q[1], q[2], q[3], nx, ny, 1.0 / nx, 1.0 / ny, 0.0, 1.4,
                              boundary_conditions=bc)
        return sim, nx, ny, q, "Kelvin-Helmholtz %dx%d, periodic" % (nx, ny)
    h, hu, hv, R = dam_break_4096(seed=seed)
    sim = SCHEMES[scheme](ctx, h, hu, hv, NX, NY, 1.0, 1.0, 9.81)
    return sim, NX, NY, [h, hu, hv], "circular dam break %dx%d (R=%.0f cells), reflective walls" % (NX, NY, R)


def rooflines(scheme, cells, launch_s, pk, pk_kind, props, prof=None):
    """HBM and FP32 rooflines of one stage launch of `scheme` over `cells`
    cells taking `launch_s` seconds on average.

    HBM: the algorithmic bytes (BYTES_PER_CELL_LAUNCH) against the measured
    copy bandwidth.  FP32, against the nominal FP32 peak (an FMA is 2
    operations): the FLOP this kernel executes (its own formulation) and, for
    comparison, the reference formulation's algorithmic count; and the floor
    set by its FP32 pipe operations.  The binding roofline is the longer of
    the HBM and FP32 lower-bound times."""
    prof = prof or {}
    alg_bytes = BYTES_PER_CELL_LAUNCH[scheme] * cells
    achieved = alg_bytes / launch_s / 1e9
    roof = {"bound": "hbm", "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / pk["hbm_gbs"], "traffic": prof.get("dram_bytes_per_launch"), "peak_kind": pk_kind,
            "algorithmic_bytes_per_launch": alg_bytes}
    sm_max_mhz = float(pk.get("sm_max_mhz") or 1965.0)
    fp32_peak = props.multi_processor_count * FP32_LANES_PER_SM * 2 * sm_max_mhz * 1e6 / 1e12
    ops = ALG_OPS_PER_CELL_LAUNCH[scheme]
    ref_flop = ops["flops"] * cells
    own = EXECUTED_FLOP_PER_CELL_LAUNCH.get(scheme)
    own_flop = own * cells if own else None
    roof_fp32 = {"bound": "fp32", "peak": fp32_peak, "unit": "TFLOP/s",
                 "peak_kind": "nominal: %d SMs x %d FP32 lanes x 2 x %.0f MHz" % (
                     props.multi_processor_count, FP32_LANES_PER_SM, sm_max_mhz),
                 "reference_formulation_flop_per_cell_launch": ops["flops"],
                 "reference_formulation_achieved": ref_flop / launch_s / 1e12,
                 "reference_formulation_frac": ref_flop / launch_s / 1e12 / fp32_peak,
                 "mufu_per_cell_launch_reference_formulation": ops["mufu"]}
    if own_flop:
        roof_fp32.update({"achieved": own_flop / launch_s / 1e12, "frac": own_flop / launch_s / 1e12 / fp32_peak,
                          "flop_per_cell_launch": own,
                          "flop_source": "FP32 FLOP this kernel executes per cell-substep (ncu sass op counters)"})
    if prof.get("executed_inst_per_cell_substep"):
        roof_fp32["executed_inst_per_cell_launch"] = prof["executed_inst_per_cell_substep"]
    t_hbm = alg_bytes / (pk["hbm_gbs"] * 1e9)
    t_fp32 = (own_flop or ref_flop) / (fp32_peak * 1e12)
    pipe_ops = FP32_PIPE_OPS_PER_CELL_LAUNCH.get(scheme)
    if pipe_ops:
        # FP32 lanes x clock: the pipe's operation rate (half the FLOP peak)
        t_pipe = pipe_ops * cells / (fp32_peak * 1e12 / 2.0)
        roof_fp32["pipe"] = {"fp32_ops_per_cell_launch": pipe_ops, "floor_us_per_launch": t_pipe * 1e6,
                             "frac": t_pipe / launch_s,
                             "what": "fadd + fmul + ffma lane operations (ncu sass counters) on 128 FP32 lanes "
                                     "per SM at the maximum SM clock"}
        t_fp32 = max(t_fp32, t_pipe)
    if t_fp32 > t_hbm:
        roof["binding"] = "fp32_pipe" if pipe_ops else ("fp32_flop" if own_flop else "fp32_flop_reference_formulation")
    else:
        roof["binding"] = "hbm"
    roof["frac_of_binding"] = max(t_hbm, t_fp32) / launch_s
    return roof, roof_fp32


ALL_SCHEMES = ("LxF", "FORCE", "HLL", "HLL2", "WAF", "KP07", "KP07_dimsplit", "EE2D_KP07_dimsplit")


def schemes_leg(ctx, steps=200, warmup=5, ref_steps=40):
    """Every scheme on its benchmark workload (the seven shallow-water schemes
    on the 4096 x 4096 dam break, Euler on the 4096 x 2048 Kelvin-Helmholtz
    problem): device ms per step over `steps` steps of simulate()'s dt
    schedule (CUDA events), HBM and FP32 rooflines of the stage kernel, and
    the reference's own kernel of the scheme (CUDA source compiled unmodified
    for sm_100a) on the same input and GPU at the fastest of its built block
    shapes, `ref_steps` steps of fixed dt."""
    import torch

    from oracle import ref_kernels

    pk, pk_kind = peaks()
    props = torch.cuda.get_device_properties(ctx.device_id)
    out = {}
    for scheme in ALL_SCHEMES:
        sim, nx, ny, q, desc = make_scheme_sim(ctx, scheme, 0)
        sim.advance(warmup)
        sim.advance(steps)
        ms = sim.last_advance_ms()
        info = sim.tile_info()
        del sim
        torch.cuda.synchronize(ctx.device_id)
        cells = nx * ny
        roof, roof_fp32 = rooflines(scheme, cells, ms * 1e-3 / info["launches_per_step"], pk, pk_kind, props)
        row = {"workload": desc, "ms_per_step": ms, "cell_updates_per_s": cells / (ms * 1e-3),
               "launches_per_step": info["launches_per_step"],
               "tile": "%dx%d, %d threads" % (info["tile_w"], info["tile_h"], info["threads"]),
               "hbm_gbs": roof["achieved"], "hbm_frac": roof["frac"], "binding": roof["binding"],
               "frac_of_binding": roof["frac_of_binding"]}
        if "pipe" in roof_fp32:
            row["fp32_pipe_floor_us_per_launch"] = roof_fp32["pipe"]["floor_us_per_launch"]
        per_block = {}
        kw = {"gamma": 1.4, "bc": 0x02020202} if scheme == "EE2D_KP07_dimsplit" else {}
        dx, dy, g = (1.0 / nx, 1.0 / ny, 0.0) if scheme == "EE2D_KP07_dimsplit" else (1.0, 1.0, 9.81)
        for block in [None] + list(ref_kernels.BLOCKS):
            if not ref_kernels.available(scheme, block):
                continue
            ref = ref_kernels.RefKernelSim(scheme, q, nx, ny, dx, dy, g, block=block, **kw)
            dt = np.float32(ref.computeDt() * np.float32(0.9))
            ref.time_steps(warmup, dt)
            per_block["%dx%d" % (ref.bw, ref.bh)] = ref.time_steps(ref_steps, dt)
            ref.close()
        if per_block:
            best = min(per_block, key=per_block.get)
            row["reference_kernels_gpu"] = {"ms_per_step": per_block[best], "block": best,
                                            "speedup_of_this_library": per_block[best] / ms}
        out[scheme] = row
    return {"what": "each scheme on its benchmark workload, %d steps (simulate()'s dt schedule), device time; "
                    "reference kernels: their CUDA source compiled unmodified for sm_100a, same input and GPU, "
                    "fastest built block, %d steps of fixed dt" % (steps, ref_steps),
            "schemes": out}


def run_mine(args, rank, world, local_rank):
    import torch

    from finitevolumegpu_b200 import CudaContext, SCHEMES, _lib

    dist = world > 1
    ctx = CudaContext.CudaContext(device=local_rank, autotuning=True)
    if args.tile is not None:  # one tile configuration instead of the autotuner's choice (profiling)
        from finitevolumegpu_b200.Autotuner import _Fixed

        ctx.autotuner = _Fixed(args.tile)
    scheme = args.scheme
    sim, nx, ny, q0, desc = make_scheme_sim(ctx, scheme, rank)
    sim.advance(args.warmup)
    info = sim.tile_info()

    def barrier():
        if dist:
            torch.distributed.barrier()
        torch.cuda.synchronize(local_rank)

    clocks = ClockSampler(local_rank)
    barrier()
    t0 = time.perf_counter()
    with clocks:
        sim.advance(args.steps)  # CUDA events on the simulation stream around the K steps
        barrier()
    wall = time.perf_counter() - t0
    dev_ms_per_step = sim.last_advance_ms()
    T = dev_ms_per_step * args.steps / 1e3
    if dist:
        t = torch.tensor([T], dtype=torch.float64, device="cuda:%d" % local_rank)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        T = float(t.item())
    cells = nx * ny
    value = world * cells * args.steps / T
    launches = args.steps * info["launches_per_step"]

    # roofline of the dominant kernel (the stage kernel)
    pk, pk_kind = peaks()
    launch_s = T / launches
    prof = load_profile() if scheme == SCHEME and NX == 4096 else {}
    roof, roof_fp32 = rooflines(scheme, cells, launch_s, pk, pk_kind, torch.cuda.get_device_properties(local_rank),
                                prof)
    roof["kernel"] = "%s stage kernel, tile %dx%d, %d threads" % (scheme, info["tile_w"], info["tile_h"],
                                                                   info["threads"])

    result = None
    if rank == 0:
        result = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": T / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "%s %s, simulate() dt schedule, cfl_scale 0.9" % (scheme, desc),
                       "scheme": scheme, "nx": nx, "ny": ny, "parallelism": "replicas" if world > 1 else "single",
                       "tile": info,
                       "l2": "state %.0f MB (two buffers) > 126 MB L2; no flush" % (
                           2 * (4 if scheme == "EE2D_KP07_dimsplit" else 3) * cells * 4 / 1e6)},
            "roofline": roof,
            "roofline_fp32": roof_fp32,
            "gpu_launches": launches,
            "clocks": clocks.summary(),
            "wall_s_timed_region": wall,
        }
    # end-to-end through the public API: pinned upload, K steps, download
    e2e = None
    # The timed simulator's device memory goes back to the stream-ordered pool,
    # where the end-to-end simulator below finds it, as a later simulation of
    # a running application would.
    del sim
    torch.cuda.synchronize(local_rank)
    if not args.no_e2e and scheme == SCHEME:
        # every rank runs its replica end to end; the time is the max over ranks
        h, hu, hv = q0
        nbytes = cells * 4
        L = _lib.lib()
        bufs = []
        import ctypes

        def pinned(shape):
            p = ctypes.c_void_p()
            _lib.check(L.fv_host_alloc(ctypes.byref(p), nbytes))
            bufs.append(p)
            arr = np.ctypeslib.as_array((ctypes.c_float * (cells)).from_address(p.value)).reshape(shape)
            return arr

        hin = [pinned((NY, NX)) for _ in range(3)]
        for a, b in zip(hin, (h, hu, hv)):
            a[:] = b
        hout = [pinned((NY, NX)) for _ in range(3)]
        barrier()
        t0 = time.perf_counter()
        s2 = SCHEMES[SCHEME](ctx, hin[0], hin[1], hin[2], NX, NY, 1.0, 1.0, 9.81)
        t_create = time.perf_counter()
        s2.advance(args.steps)
        s2.synchronize()
        t_steps = time.perf_counter()
        for v in range(3):
            s2._download_var(v, hout[v])
        e2e_s = time.perf_counter() - t0
        split = {"create": t_create - t0, "steps": t_steps - t_create, "download": t0 + e2e_s - t_steps}
        if dist:
            t = torch.tensor([e2e_s], dtype=torch.float64, device="cuda:%d" % local_rank)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            e2e_s = float(t.item())
        del s2
        for p in bufs:
            L.fv_host_free(p)
        e2e = {"value": world * cells * args.steps / e2e_s, "unit": "cell-updates/s",
               "h2d_bytes_per_step": 3 * nbytes / args.steps, "d2h_bytes_per_step": 3 * nbytes / args.steps,
               "what": "constructor with pinned host upload + %d steps + download of the final state" % args.steps,
               "seconds": split}
        if result is not None:
            result["e2e"] = e2e
    if rank == 0 and world == 1 and not args.no_batched and scheme == SCHEME:
        result["batched"] = aux_leg(run_batched, ctx)
    if rank == 0 and world == 1 and not args.no_served and scheme == SCHEME:
        result["served"] = aux_leg(run_served, ctx, n_req=args.served_requests,
                                   rates=tuple(float(r) for r in args.served_rates.split(",")))
    if rank == 0 and world == 1 and not args.no_cpu_baseline and scheme == SCHEME:
        result["cpu_baseline"] = aux_leg(cpu_baseline_leg)
    if rank == 0 and world == 1 and not args.no_reference_kernels and scheme == SCHEME and NX == 4096:
        result["reference_kernels_gpu"] = aux_leg(reference_kernels_leg, dev_ms_per_step)
    if rank == 0 and world == 1 and not args.no_schemes and scheme == SCHEME and NX == 4096:
        result["schemes"] = aux_leg(schemes_leg, ctx)
    return result


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="mine", choices=["mine", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the 512-simulation batched workload")
    ap.add_argument("--no-served", action="store_true", help="skip the served request stream")
    ap.add_argument("--no-reference-kernels", action="store_true",
                    help="skip timing the reference's own kernel on the same GPU")
    ap.add_argument("--no-schemes", action="store_true",
                    help="skip the per-scheme leg (every scheme on its benchmark workload, with the reference kernels)")
    ap.add_argument("--served-requests", type=int, default=10000)
    ap.add_argument("--served-rates", default="300,600,900,1200",
                    help="Poisson arrival rates (requests/s) of the served sweep, comma separated; the top-level "
                         "figures are those of the highest rate the server sustained, `capacity` those of the "
                         "rate with the highest throughput")
    ap.add_argument("--size", type=int, default=4096, help="grid side (the benchmark workload is 4096)")
    ap.add_argument("--scheme", default=SCHEME, help="scheme of the single-simulation timing (default KP07_dimsplit)")
    ap.add_argument("--tile", type=int, default=None,
                    help="tile configuration of the timed simulation (index into the scheme's kernel table; "
                         "default: the autotuner's)")
    args = ap.parse_args()
    global NX, NY
    NX = NY = args.size
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        res = run_reference(args, rank, world)
        if res is not None:
            print(json.dumps(res), flush=True)
        return
    if world > 1:
        import datetime

        import torch

        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    res = run_mine(args, rank, world, local_rank)
    if res is not None:
        print(json.dumps(res), flush=True)
    if world > 1:
        import torch

        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
