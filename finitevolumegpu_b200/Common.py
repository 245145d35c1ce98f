"""Simulation runs with snapshot output, and checkpoint/resume: the counterparts of
``runSimulation`` and ``DataDumper`` in GPUSimulators/Common.py.

``runSimulation`` (GPUSimulators/Common.py:86-208) constructs a simulator,
advances it to each of the requested save times with ``simulate`` and stores
the chosen variables at those times in a NetCDF file with ``time``, ``x`` and
``y`` coordinates plus the run's metadata.  The reference writes netCDF4 with
zlib compression and ``least_significant_digit=3``; this environment has no
netCDF4 library, so the file here is NetCDF3 (written by SciPy, readable by
any NetCDF reader) without compression, and the values are quantised the way
netCDF4 quantises for ``least_significant_digit``: rounded to a multiple of
2**-ceil(log2(10**digits)), so a reader sees the same numbers as in the
reference's files.

``DataDumper`` (GPUSimulators/Common.py:361-434) opens such a file, creating
the directory and, for writing, a fresh file name (``name_0000.nc``, …) rather
than overwriting an existing file.

The module's small host helpers keep the reference's names and behaviour:
``Timer`` (a logged ``with`` block timer), ``ProgressPrinter`` (the progress
line ``runSimulation`` logs), ``safeCall``, ``getGitHash`` and
``getGitStatus``.

``save_checkpoint`` / ``load_checkpoint`` have no reference counterpart: they
store a simulator's state with its time-stepping state (t, nt, dt and the last
CFL minimum) so that a run continued from the checkpoint takes exactly the
steps the uninterrupted run takes.  Ghost cells are not stored: they are
rebuilt from the boundary conditions (Dirichlet ghost values start from zero).
"""

from __future__ import annotations

import inspect
import json
import logging
import os
import subprocess
import time

import numpy as np


def quantize(data, least_significant_digit):
    """netCDF4's lossy quantisation for ``least_significant_digit``: values are
    rounded to the nearest multiple of 2**-bits, bits = ceil(log2(10**digits))."""
    bits = int(np.ceil(np.log2(10.0 ** least_significant_digit)))
    scale = 2.0 ** bits
    return (np.around(scale * np.asarray(data, dtype=np.float64)) / scale).astype(np.float32)


def safeCall(cmd):
    """Output of `cmd` (a list) run in this package's directory, stderr merged
    into it; a failing command is logged and its CalledProcessError re-raised
    (GPUSimulators/Common.py:48-66)."""
    try:
        return subprocess.check_output(cmd, stderr=subprocess.STDOUT, cwd=os.path.dirname(os.path.abspath(__file__)),
                                       universal_newlines=True, shell=False)
    except subprocess.CalledProcessError as e:
        logging.getLogger(__name__).error("Git failed, \nReturn code: %s\nOutput: %s", e.returncode, e.output)
        raise


def getGitHash():
    """Commit hash of the checkout holding this package (Common.py:68-69)."""
    return safeCall(["git", "rev-parse", "HEAD"])


def getGitStatus():
    """Changed tracked files of that checkout (Common.py:71-72)."""
    return safeCall(["git", "status", "--porcelain", "-uno"])


def _git(args):
    """Like safeCall, but quietly "" where git or a checkout is missing: run
    metadata must not stop (or log errors for) a simulation that runs from a
    copy of the package."""
    try:
        return subprocess.check_output(["git"] + args, stderr=subprocess.STDOUT,
                                       cwd=os.path.dirname(os.path.abspath(__file__))).decode().strip()
    except (OSError, subprocess.CalledProcessError):
        return ""


class Timer(object):
    """Wall time of a ``with`` block, logged at `log_level` on exit as
    "<tag>: <ms> ms"; ``secs`` and ``msecs`` hold it afterwards and
    ``elapsed()`` reads it while the block runs (Common.py:215-238)."""

    def __init__(self, tag, log_level=logging.DEBUG):
        self.tag = tag
        self.log_level = log_level
        self.logger = logging.getLogger(__name__)

    def __enter__(self):
        self.start = time.time()
        return self

    def __exit__(self, *args):
        self.end = time.time()
        self.secs = self.end - self.start
        self.msecs = self.secs * 1000.0
        self.logger.log(self.log_level, "%s: %f ms", self.tag, self.msecs)

    def elapsed(self):
        return time.time() - self.start


class ProgressPrinter(object):
    """Progress line for a loop over `total_steps` units (Common.py:436-496).

    ``getPrintString(step)`` returns None until `print_every` seconds have
    passed since the last line, then a bar with the elapsed, remaining and
    total time.  The remaining time extrapolates the time per unit, smoothed
    over the lines printed so far (the newest interval weighs 0.8)."""

    def __init__(self, total_steps, print_every=5):
        self.logger = logging.getLogger(__name__)
        self.start = time.time()
        self.total_steps = total_steps
        self.print_every = print_every
        self.next_print_time = print_every
        self.last_step = 0
        self.secs_per_iter = None

    def getPrintString(self, step):
        elapsed = time.time() - self.start
        if elapsed <= self.next_print_time:
            return None
        done = step - self.last_step
        if done == 0:
            return None
        interval = elapsed - (self.next_print_time - self.print_every)
        rate = interval / done
        self.secs_per_iter = rate if not self.secs_per_iter else 0.2 * self.secs_per_iter + 0.8 * rate
        self.last_step = step
        self.next_print_time = elapsed + self.print_every
        remaining = (self.total_steps - step) * self.secs_per_iter
        return "{:s}. Total: {:s}, elapsed: {:s}, remaining: {:s}".format(
            ProgressPrinter.progressBar(step, self.total_steps), ProgressPrinter.timeString(elapsed + remaining),
            ProgressPrinter.timeString(elapsed), ProgressPrinter.timeString(remaining))

    @staticmethod
    def timeString(seconds):
        """Whole seconds (at least 1) as "1h 2m 3s", zero fields left out."""
        s = int(max(seconds, 1))
        h, s = divmod(s, 3600)
        m, s = divmod(s, 60)
        return " ".join("%d%s" % (v, unit) for v, unit in ((h, "h"), (m, "m"), (s, "s")) if v)

    @staticmethod
    def progressBar(step, total_steps, width=30):
        """"0% [####======] 100%" with `width` cells, '#' for the done fraction."""
        filled = int(np.round(width * step / total_steps))
        return "0% [" + "#" * filled + "=" * (width - filled) + "] 100%"


def toJson(in_dict):
    """JSON of a dictionary, arrays as lists and anything else unserialisable as its string."""
    out = {}
    for key, value in in_dict.items():
        if isinstance(value, np.ndarray):
            out[key] = value.tolist()
        else:
            try:
                json.dumps(value)
                out[key] = value
            except TypeError:
                out[key] = str(value)
    return json.dumps(out)


class DataDumper(object):
    """A NetCDF file for the duration of a ``with`` block::

        with DataDumper("out.nc", mode="w") as data:
            data.ncfile.createDimension(...)
    """

    def __init__(self, filename, *args, **kwargs):
        self.logger = logging.getLogger(__name__)
        filename = os.path.abspath(filename)
        dirname = os.path.dirname(filename)
        if dirname and not os.path.isdir(dirname):
            os.makedirs(dirname)
        mode = args[0] if args else kwargs.get("mode", "r")
        if any(c in mode for c in "wa+"):
            i = 0
            stem, ext = os.path.splitext(filename)
            while os.path.isfile(filename):
                filename = "{:s}_{:04d}{:s}".format(stem, i, ext)
                i += 1
        self.filename = filename
        self.mode = mode
        self.ncfile = None

    def __enter__(self):
        from scipy.io import netcdf_file

        self.ncfile = netcdf_file(self.filename, self.mode[0], version=2)
        return self

    def __exit__(self, *args):
        self.ncfile.close()


def runSimulation(simulator, simulator_args, outfile, save_times, save_var_names=(), dt=None,
                  least_significant_digit=3):
    """Run `simulator(**simulator_args)` and store `save_var_names` at each of
    `save_times` (None entries skip that variable) in a new NetCDF file.

    Returns (file name, host timings, the simulator's profiling_data_mpi) as
    the reference does (GPUSimulators/Common.py:98-105, :208).  The timings are
    {"start": {stage: s}, "end": {stage: s}} with end - start the time spent in
    each stage ("t_sim_init", "t_nc_write", "t_full_step"): host clock stamps
    added up before and after each visit, as the reference adds them.  The
    third value is None for a simulator without MPI profiling."""
    logger = logging.getLogger(__name__)
    save_times = np.asarray(save_times, dtype=np.float64)
    assert len(save_times) > 0, "Need to specify which times to save"
    stages = ("t_sim_init", "t_nc_write", "t_full_step")
    timing = {"start": {k: 0.0 for k in stages}, "end": {k: 0.0 for k in stages}}
    timing["start"]["t_sim_init"] = time.time()
    with Timer("construct") as t:
        sim = simulator(**simulator_args)
    logger.info("Constructed in %s seconds", t.secs)
    with DataDumper(outfile, mode="w") as outdata:
        nc = outdata.ncfile
        nc.created = time.ctime(time.time())
        nc.git_hash = _git(["rev-parse", "HEAD"])
        nc.git_status = _git(["status", "--porcelain", "-uno"])
        nc.simulator = str(simulator)
        # the initial fields are too large for attributes
        nc.sim_args = toJson({k: v for k, v in simulator_args.items() if not isinstance(v, np.ndarray)})
        nx, ny = int(simulator_args["nx"]), int(simulator_args["ny"])
        nc.createDimension("time", len(save_times))
        nc.createDimension("x", nx)
        nc.createDimension("y", ny)
        ncvars = {"time": nc.createVariable("time", "f", ("time",)), "x": nc.createVariable("x", "f", ("x",)),
                  "y": nc.createVariable("y", "f", ("y",))}
        ncvars["time"][:] = save_times
        extent = sim.getExtent()
        ncvars["x"][:] = np.linspace(extent[0], extent[1], nx)
        ncvars["y"][:] = np.linspace(extent[2], extent[3], ny)
        download_vars = [i for i, name in enumerate(save_var_names) if name is not None]
        names = [save_var_names[i] for i in download_vars]
        for name in names:
            ncvars[name] = nc.createVariable(name, "f", ("time", "y", "x"))
            ncvars[name].least_significant_digit = least_significant_digit
        t_steps = np.empty_like(save_times)
        t_steps[0] = save_times[0]
        t_steps[1:] = save_times[1:] - save_times[:-1]
        timing["end"]["t_sim_init"] = time.time()
        progress = ProgressPrinter(save_times[-1], print_every=10)
        for k in range(len(save_times)):
            try:
                sim.check()
            except AssertionError as e:
                logger.error("Error after %d steps (t=%f): %s", sim.simSteps(), sim.simTime(), str(e))
                return outdata.filename, timing, getattr(sim, "profiling_data_mpi", None)
            timing["start"]["t_full_step"] += time.time()
            if t_steps[k] > 0.0:
                sim.simulate(t_steps[k], dt)
            timing["end"]["t_full_step"] += time.time()
            timing["start"]["t_nc_write"] += time.time()
            values = sim.download(download_vars)
            for i, name in enumerate(names):
                ncvars[name][k, :, :] = quantize(values[i], least_significant_digit)
            timing["end"]["t_nc_write"] += time.time()
            line = progress.getPrintString(save_times[k])
            if line:
                logger.debug(line)
        logger.debug("Simulated to t=%f in %d steps", sim.simTime(), sim.simSteps())
        return outdata.filename, timing, getattr(sim, "profiling_data_mpi", None)


# Constructor keyword arguments of each scheme beyond (context, fields, nx, ny, dx, dy, g).
_SCHEME_KWARGS = ("theta", "cfl_scale", "order")


def save_checkpoint(sim, path):
    """Store a simulator's state and time-stepping state in an .npz file; returns the path."""
    t, nt, dt, cfl_min = sim.get_control()
    meta = {
        "scheme": type(sim).__name__,
        "nx": int(sim.nx), "ny": int(sim.ny), "dx": float(sim.dx), "dy": float(sim.dy),
        "g": float(getattr(sim, "g", 0.0)), "gamma": float(getattr(sim, "gamma", 1.4)),
        "theta": float(getattr(sim, "theta", 1.3)), "order": int(getattr(sim, "order", 2)),
        "cfl_scale": float(sim.cfl_scale), "boundary_conditions": int(sim.boundary_conditions),
        "t": float(t), "nt": int(nt), "dt": float(dt), "cfl_min": float(cfl_min),
    }
    state = sim.download()
    np.savez(path, meta=json.dumps(meta), **{"var%d" % i: a for i, a in enumerate(state)})
    return path if path.endswith(".npz") else path + ".npz"


def load_checkpoint(context, path):
    """A simulator rebuilt from `save_checkpoint`'s file, ready to continue."""
    from . import SCHEMES
    from .Simulator import BoundaryCondition

    with np.load(path) as f:
        meta = json.loads(str(f["meta"]))
        state = [f["var%d" % i] for i in range(sum(1 for k in f.files if k.startswith("var")))]
    cls = SCHEMES[meta["scheme"]]
    accepted = inspect.signature(cls.__init__).parameters
    kwargs = {k: meta[k] for k in _SCHEME_KWARGS if k in accepted}
    kwargs["boundary_conditions"] = BoundaryCondition(BoundaryCondition.getTypes(meta["boundary_conditions"]))
    pos = [meta["nx"], meta["ny"], meta["dx"], meta["dy"], meta["g"]]
    if "gamma" in accepted:
        pos.append(meta["gamma"])
    sim = cls(context, *state, *pos, **kwargs)
    sim.set_control(meta["t"], meta["nt"], meta["dt"], meta["cfl_min"])
    return sim
