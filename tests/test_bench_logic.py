"""bench.py's host logic on the CPU: a failing side measurement does not cost
the headline line, and the reference arm (the CPU restatement of the
reference algorithm) keeps the benchmark contract under torchrun: rank 0 alone
prints one JSON line, every rank exits 0."""

import json
import os
import subprocess
import sys

from conftest import ROOT

import bench
from stripe_helpers import free_port


def test_aux_leg_reports_failures():
    def failing(n, scale=1):
        raise RuntimeError("leg %d failed" % (n * scale))

    assert bench.aux_leg(failing, 2, scale=3) == {"error": "RuntimeError: leg 6 failed"}
    assert bench.aux_leg(lambda a, b=0: {"v": a + b}, 2, b=5) == {"v": 7}


def test_reference_arm_under_torchrun():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(free_port()), "bench.py", "--impl", "reference", "--gpus", "2",
           "--steps", "1", "--warmup", "0"]
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600,
                         env=dict(os.environ, OMP_NUM_THREADS="4"))
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [line for line in out.stdout.splitlines() if line.startswith("{")]
    assert len(lines) == 1, out.stdout
    res = json.loads(lines[0])
    assert res["impl"] == "reference" and res["n_gpus"] == 2 and res["steps"] == 1
    assert res["metric"] == "cell-updates/s" and res["higher_is_better"] is True and res["value"] > 0
    assert res["cpu_baseline"]["value"] == res["value"] and res["cpu_baseline"]["kind"] == "port"
    assert res["e2e"] == {"value": res["value"], "unit": res["unit"], "h2d_bytes_per_step": 0,
                          "d2h_bytes_per_step": 0}


def test_bench_legs_and_initial_states():
    """Every leg the GPU arm runs is defined, and the seeded initial states
    have the requested shapes (bench.py's host side, no GPU)."""
    import numpy as np

    for name in ("run_mine", "run_reference", "run_batched", "run_served", "cpu_baseline_leg",
                 "reference_kernels_leg", "schemes_leg", "rooflines", "make_scheme_sim", "ICFeed"):
        assert callable(getattr(bench, name)), name
    rng = np.random.default_rng(0)
    for make, nv in ((bench.bump_ic, 3), (bench.dam_ic, 3), (bench.kh_ic, 4)):
        q = make(37, 21, rng)
        assert len(q) == nv and all(a.shape == (21, 37) and a.dtype == np.float32 for a in q)
        assert np.all(q[0] > 0)


def test_initial_states_match_their_full_grid_formulas():
    """The served leg's initial-state generators take shortcuts (a bump is
    evaluated only near its centre, the Kelvin-Helmholtz rows are computed
    once); they must give the bits of the plain full-grid formulas."""
    import numpy as np

    def bump(nx, ny, rng):
        A = rng.uniform(0.1, 0.5)
        cx, cy = rng.uniform(0.3, 0.7) * nx, rng.uniform(0.3, 0.7) * ny
        x = np.arange(nx, dtype=np.float32) + 0.5
        y = np.arange(ny, dtype=np.float32) + 0.5
        h = 1.0 + A * np.exp(-((x[None, :] - cx) ** 2 + (y[:, None] - cy) ** 2) / (2 * 20.0 ** 2))
        return [h.astype(np.float32)]

    def dam(nx, ny, rng):
        R = rng.uniform(0.1, 0.3) * nx
        x = np.arange(nx, dtype=np.float32) + 0.5 - nx / 2.0
        y = np.arange(ny, dtype=np.float32) + 0.5 - ny / 2.0
        return [np.where(x[None, :] ** 2 + y[:, None] ** 2 < R * R, 1.0, 0.1).astype(np.float32)]

    def kh(nx, ny, rng, gamma=1.4):
        phi = rng.uniform(0, 2 * np.pi)
        yy = (np.arange(ny, dtype=np.float32) + 0.5) / ny
        xx = (np.arange(nx, dtype=np.float32) + 0.5) / nx
        band = ((yy >= 0.25) & (yy < 0.75))[:, None]
        rho = np.where(band, 2.0, 1.0) * np.ones((1, nx))
        u = np.where(band, 0.5, -0.5) * np.ones((1, nx))
        v = 0.01 * np.sin(4 * np.pi * xx[None, :] + phi) * np.ones((ny, 1))
        E = 2.5 / (gamma - 1.0) + 0.5 * rho * (u ** 2 + v ** 2)
        return [a.astype(np.float32) for a in (rho, rho * u, rho * v, E)]

    for nx, ny in ((128, 128), (2048, 2048), (700, 300), (129, 2047), (1500, 131), (3, 5), (900, 64)):
        for seed in range(4):
            for fast, plain in ((bench.bump_ic, bump), (bench.dam_ic, dam), (bench.kh_ic, kh)):
                got = fast(nx, ny, np.random.default_rng(seed))
                want = plain(nx, ny, np.random.default_rng(seed))
                for a, b in zip(got, want):
                    assert a.dtype == np.float32 and a.shape == (ny, nx)
                    assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (fast.__name__, nx, ny, seed)
                if fast is not bench.kh_ic:
                    assert not np.any(got[1]) and not np.any(got[2])


def test_ic_feed_serves_requests_in_order_with_skips_and_retries():
    made = []

    def make(i):
        made.append(i)
        return i * 10

    feed = bench.ICFeed(make, 100, threads=3, ahead=4)
    try:
        got = [feed.get(i) for i in range(100) if i % 7 != 3]  # some requests are never admitted
        assert got == [i * 10 for i in range(100) if i % 7 != 3]
        assert feed.get(17) == 170  # a retried admission regenerates its state
    finally:
        feed.close()


def test_rooflines_of_every_scheme():
    """rooflines(): algorithmic bytes over the launch time against the
    measured HBM peak, and the binding floor (the longer of the HBM and the
    FP32-pipe lower bounds) over the launch time, for every scheme."""
    import types

    props = types.SimpleNamespace(multi_processor_count=148)
    pk = {"hbm_gbs": 6500.0, "sm_max_mhz": 1965.0}
    cells = 4096 * 4096
    for scheme in bench.ALL_SCHEMES:
        launch_s = 200e-6
        roof, fp32 = bench.rooflines(scheme, cells, launch_s, pk, "measured", props)
        alg = bench.BYTES_PER_CELL_LAUNCH[scheme] * cells
        assert roof["algorithmic_bytes_per_launch"] == alg
        assert abs(roof["achieved"] - alg / launch_s / 1e9) < 1e-6 * roof["achieved"]
        assert abs(roof["frac"] - roof["achieved"] / 6500.0) < 1e-12
        t_hbm = alg / 6500e9
        t_pipe = bench.FP32_PIPE_OPS_PER_CELL_LAUNCH[scheme] * cells / (148 * 128 * 1965e6)
        assert abs(fp32["pipe"]["floor_us_per_launch"] - t_pipe * 1e6) < 1e-9 * t_pipe * 1e6
        assert roof["binding"] == ("fp32_pipe" if t_pipe > t_hbm else "hbm"), scheme
        assert abs(roof["frac_of_binding"] - max(t_hbm, t_pipe) / launch_s) < 1e-12
    # the headline kernel binds on its FP32 pipe operations (71.6 us against 62 us of HBM traffic)
    roof, _ = bench.rooflines("KP07_dimsplit", cells, 155e-6, {"hbm_gbs": 6500.0}, "measured", props)
    assert roof["binding"] == "fp32_pipe"
