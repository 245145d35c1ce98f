"""Snapshot output (runSimulation / DataDumper counterparts), host logic on the CPU."""

import numpy as np
import pytest

from finitevolumegpu_b200.Common import DataDumper, quantize, runSimulation


def test_quantize_is_netcdf4_least_significant_digit():
    # 3 digits -> bits = ceil(log2(1000)) = 10, multiples of 1/1024
    x = np.array([0.1234567, -2.5000001, 1.0, 1e-4, 3.14159], dtype=np.float32)
    q = quantize(x, 3)
    assert np.array_equal(q, (np.around(x.astype(np.float64) * 1024) / 1024).astype(np.float32))
    assert np.all(np.abs(q - x) <= 0.5 / 1024 + 1e-7)
    assert q[0] == np.float32(126 / 1024)


def test_datadumper_never_overwrites(tmp_path):
    path = str(tmp_path / "sub" / "run.nc")
    names = []
    for _ in range(3):
        with DataDumper(path, mode="w") as d:
            d.ncfile.createDimension("x", 2)
            names.append(d.filename)
    assert names[0].endswith("run.nc") and names[1].endswith("run_0000.nc") and names[2].endswith("run_0001.nc")


class FakeSim(object):
    """Deterministic stand-in with the simulator methods runSimulation uses."""

    def __init__(self, nx, ny, dx=1.0, dy=1.0, **kw):
        self.nx, self.ny, self.dx, self.dy = nx, ny, dx, dy
        self.t, self.nt = 0.0, 0

    def simulate(self, t, dt=None):
        self.t += t
        self.nt += 7

    def download(self, variables=None):
        y, x = np.mgrid[0:self.ny, 0:self.nx]
        fields = [np.sin(0.1 * x + self.t) + y * 1e-3, np.cos(0.2 * y - self.t), x * self.t]
        return [fields[i].astype(np.float32) for i in (variables if variables is not None else range(3))]

    def check(self):
        pass

    def getExtent(self):
        return [0, self.nx * self.dx, 0, self.ny * self.dy]

    def simSteps(self):
        return self.nt

    def simTime(self):
        return self.t


def test_run_simulation_writes_quantised_frames(tmp_path):
    from scipy.io import netcdf_file

    times = np.array([0.0, 0.5, 1.25])
    fname, timing, mpi = runSimulation(FakeSim, {"nx": 12, "ny": 9, "dx": 1.0, "dy": 1.0}, str(tmp_path / "o.nc"),
                                       times, ["h", None, "hv"])
    assert mpi is None and set(timing) == {"start", "end"}
    for stage in ("t_sim_init", "t_nc_write", "t_full_step"):
        assert timing["end"][stage] - timing["start"][stage] >= 0.0
    ref = FakeSim(12, 9)
    with netcdf_file(fname, "r", mmap=False) as f:
        assert np.allclose(f.variables["time"][:], times)
        assert f.variables["x"][:].shape == (12,) and "hu" not in f.variables
        assert b"nx" in f.sim_args
        for k, t in enumerate(times):
            ref.t = t
            h, hv = ref.download([0, 2])
            assert np.array_equal(f.variables["h"][k], quantize(h, 3))
            assert np.array_equal(f.variables["hv"][k], quantize(hv, 3))


def test_timer_records_and_logs(caplog):
    import logging
    import time

    from finitevolumegpu_b200.Common import Timer

    with caplog.at_level(logging.DEBUG, logger="finitevolumegpu_b200.Common"):
        with Timer("block") as t:
            time.sleep(0.02)
            assert t.elapsed() > 0.0
    assert 0.015 < t.secs < 2.0 and abs(t.msecs - 1000.0 * t.secs) < 1e-9
    assert any(r.getMessage().startswith("block: ") and r.getMessage().endswith(" ms") for r in caplog.records)


def test_progress_printer(monkeypatch):
    import finitevolumegpu_b200.Common as common

    clock = {"t": 100.0}
    monkeypatch.setattr(common.time, "time", lambda: clock["t"])
    p = common.ProgressPrinter(100, print_every=5)
    clock["t"] = 103.0
    assert p.getPrintString(10) is None            # before print_every seconds
    clock["t"] = 110.0
    line = p.getPrintString(50)                    # 10 s for 50 units: 0.2 s each, 50 left
    assert line == "0% [" + "#" * 15 + "=" * 15 + "] 100%. Total: 20s, elapsed: 10s, remaining: 10s"
    clock["t"] = 112.0
    assert p.getPrintString(60) is None            # the next line is due 5 s after the last
    clock["t"] = 116.0
    assert p.getPrintString(50) is None            # no progress since the last line
    assert common.ProgressPrinter.timeString(3725.9) == "1h 2m 5s"
    assert common.ProgressPrinter.timeString(0.2) == "1s"
    assert common.ProgressPrinter.timeString(120) == "2m"
    assert common.ProgressPrinter.progressBar(0, 10, width=4) == "0% [====] 100%"
    assert common.ProgressPrinter.progressBar(10, 10, width=4) == "0% [####] 100%"


def test_git_helpers():
    import re
    import subprocess

    from finitevolumegpu_b200.Common import getGitHash, getGitStatus, safeCall

    try:
        h = getGitHash()
    except (OSError, subprocess.CalledProcessError):
        pytest.skip("package not in a git checkout")
    assert re.fullmatch(r"[0-9a-f]{40}\n", h)
    assert isinstance(getGitStatus(), str)
    with pytest.raises(subprocess.CalledProcessError):
        safeCall(["git", "rev-parse", "--verify", "no-such-ref-here"])
