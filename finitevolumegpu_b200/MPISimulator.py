"""Row-stripe domain decomposition: the counterpart of GPUSimulators/MPISimulator.py.

The reference splits one domain into north-south stripes, one MPI rank (and
GPU) per stripe (``MPIGrid.getGrid`` keeps ``grid[0] = 1``,
GPUSimulators/MPISimulator.py:137-143).  Each rank runs an ordinary simulator
on its stripe whose internal north/south edges are Dirichlet, i.e. whose ghost
rows hold whatever was last stored there (MPISimulator.py:239-258); after every
substep the ranks exchange two rows with each neighbour, so those ghost rows
hold the neighbour's edge rows (``full_exchange``, :371-480), and the time step
is the minimum over all ranks (``computeDt``, :349-355).

Here the same scheme runs on top of the sm_100a simulators:

* ``StripeGrid`` is the ``MPIGrid`` counterpart over a ``torch.distributed``
  process group (NCCL between GPUs, gloo on CPU).
* ``MPISimulator(sim, grid)`` wraps a local simulator like the reference class.
  The halo rows are zero-copy views of the simulator's device buffers
  (``BaseSimulator.halo_views``) and the sends and receives are issued on the
  simulator's own CUDA stream, so they are ordered with the stage kernels
  without host synchronisation.  Each message is one variable's two full
  storage rows (ghost columns included), 2 x pitch floats.
* ``StripedSimulator`` runs all stripes of a domain in one process (on one
  GPU or several), exchanging the rows with device copies ordered by CUDA
  events.

East and west edges are not exchanged: every stripe spans the whole width, so
its own boundary handling (periodic wrap or reflective mirror along x,
including the corner cells of the exchanged ghost rows) gives the cells the
reference's self-exchange along x gives.  With the same per-cell arithmetic in
every tile, a decomposed run reproduces the single-domain run bit for bit.

Any local simulator with this interface can be decomposed: ``nx, ny, dx, dy,
cfl_scale, num_substeps``, ``substep(dt, step_number)``, ``computeDt()``,
``download()``, ``synchronize()``, ``getBoundaryConditions()`` /
``setBoundaryConditions(bc)``, ``halo_views()`` and ``comm_stream()``.
"""

from __future__ import annotations

import logging
import time

import numpy as np

from .Simulator import BoundaryCondition

GOING_NORTH = 0  # tag of rows sent to the northern neighbour (they fill its south ghost rows)
GOING_SOUTH = 1  # tag of rows sent to the southern neighbour (they fill its north ghost rows)


def stripe_rows(ny, n):
    """Split ny rows into n stripes, south to north: a list of (first row, rows);
    sizes differ by at most one row."""
    ny, n = int(ny), int(n)
    assert 1 <= n <= ny, "cannot split %d rows into %d stripes" % (ny, n)
    base, extra = divmod(ny, n)
    out, y = [], 0
    for j in range(n):
        rows = base + (1 if j < extra else 0)
        out.append((y, rows))
        y += rows
    return out


def stripe_boundaries(boundary_conditions, j, n):
    """Boundary conditions of stripe j of n and whether it has a southern and a
    northern neighbour (MPISimulator.py:239-258): internal edges become
    Dirichlet, the domain's south (north) edge keeps its condition unless it is
    periodic, in which case the first and last stripes are neighbours."""
    bc = boundary_conditions
    T = BoundaryCondition.Type
    has_south = not (j == 0 and bc.south != T.Periodic)
    has_north = not (j == n - 1 and bc.north != T.Periodic)
    new = BoundaryCondition({
        "north": T.Dirichlet if has_north else bc.north,
        "south": T.Dirichlet if has_south else bc.south,
        "east": bc.east,
        "west": bc.west,
    })
    return new, has_south, has_north


class StripeGrid(object):
    """North-south stripes over a torch.distributed process group: the
    counterpart of MPIGrid (GPUSimulators/MPISimulator.py:34-203) with its
    vertical-only partitioning."""

    def __init__(self, group=None, device=None):
        import torch.distributed as dist

        assert dist.is_initialized(), "torch.distributed must be initialised"
        self.group = group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)
        self.grid = np.array([1, self.size])
        self.backend = dist.get_backend(group)
        if device is None:
            import torch

            device = torch.device("cuda", torch.cuda.current_device()) if self.backend == "nccl" else torch.device("cpu")
        self.device = device

    def getCoordinate(self, rank=None):
        rank = self.rank if rank is None else rank
        return 0, rank

    def getRank(self, i, j):
        return j

    def getNorth(self):
        return (self.rank + 1) % self.size

    def getSouth(self):
        return (self.rank + self.size - 1) % self.size

    def getEast(self):
        return self.rank

    def getWest(self):
        return self.rank

    def getLocalRank(self):
        import os

        return int(os.environ.get("LOCAL_RANK", self.rank))

    def exchange(self, sends, recvs):
        """Point-to-point messages: sends and recvs are lists of (peer, tensor,
        tag), posted in list order; returns once all have completed on the
        current stream."""
        import torch.distributed as dist

        ops = [dist.P2POp(dist.isend, t, self._global(p), self.group, tag) for p, t, tag in sends]
        ops += [dist.P2POp(dist.irecv, t, self._global(p), self.group, tag) for p, t, tag in recvs]
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()

    def allreduce_min(self, value):
        import torch
        import torch.distributed as dist

        t = torch.tensor([float(value)], dtype=torch.float32, device=self.device)
        dist.all_reduce(t, op=dist.ReduceOp.MIN, group=self.group)
        return np.float32(t.item())

    def gather(self, data, root=0):
        """Stripes of all ranks stacked on `root` (None elsewhere)."""
        import torch.distributed as dist

        out = [None] * self.size if self.rank == root else None
        dist.gather_object(np.asarray(data), out, dst=self._global(root), group=self.group)
        return out

    def _global(self, rank):
        import torch.distributed as dist

        return rank if self.group is None else dist.get_global_rank(self.group, rank)


def _exchange_plan(views, north, south):
    """Sends and receives of one halo exchange in an order every rank shares:
    both sends, then the receive from the south, then from the north, so the
    k-th message between two ranks is matched by position even when the
    northern and southern neighbours are the same rank."""
    sends, recvs = [], []
    nv = len(views["north_send"])
    if north is not None:
        sends += [(north, views["north_send"][v], GOING_NORTH) for v in range(nv)]
    if south is not None:
        sends += [(south, views["south_send"][v], GOING_SOUTH) for v in range(nv)]
    if south is not None:
        recvs += [(south, views["south_ghost"][v], GOING_NORTH) for v in range(nv)]
    if north is not None:
        recvs += [(north, views["north_ghost"][v], GOING_SOUTH) for v in range(nv)]
    return sends, recvs


class HaloProfile(object):
    """The reference's ``profiling_data_mpi`` (GPUSimulators/MPISimulator.py:210-221):
    {"start": {stage: s}, "end": {stage: s}, "n_time_steps": n}, read by its
    drivers as end - start per stage (mpiTesting.py:171-177).

    The reference adds host time stamps; here each stage's duration is timed
    with CUDA events on the stream the stage runs on (host clock for
    host-memory simulators) and added to "end", "start" staying 0, so
    end - start is the same total.  Stages: "t_mpi_step" (the stage kernels of
    a substep), "t_mpi_halo_exchange" (a whole exchange) and
    "t_mpi_halo_exchange_sendreceive" (its point-to-point messages).  The
    exchange moves rows between device buffers directly, with no host staging,
    so "t_mpi_halo_exchange_download" and "..._upload" stay 0.
    "n_time_steps" counts substeps, as the reference's does (:338).  Event
    pairs are read back lazily, when the dictionary is read."""

    STAGES = ("t_mpi_halo_exchange", "t_mpi_halo_exchange_download", "t_mpi_halo_exchange_upload",
              "t_mpi_halo_exchange_sendreceive", "t_mpi_step")
    MAX_PENDING = 512  # event pairs kept before the oldest are read back

    def __init__(self):
        self.data = {"start": {k: 0 for k in self.STAGES}, "end": {k: 0 for k in self.STAGES}, "n_time_steps": 0}
        self._pending = []  # (stage, start event, end event)
        self._free = []

    def _event(self):
        if self._free:
            return self._free.pop()
        import torch

        return torch.cuda.Event(enable_timing=True)

    def begin(self, stream):
        """A token marking the start of a stage on `stream` (None: host clock)."""
        if stream is None:
            return time.perf_counter()
        ev = self._event()
        ev.record(stream)
        return ev

    def end(self, stage, token, stream):
        if stream is None:
            self.data["end"][stage] += time.perf_counter() - token
            return
        ev = self._event()
        ev.record(stream)
        self._pending.append((stage, token, ev))
        if len(self._pending) > self.MAX_PENDING:
            self._resolve(len(self._pending) // 2)

    def _resolve(self, n=None):
        n = len(self._pending) if n is None else n
        done, self._pending = self._pending[:n], self._pending[n:]
        for stage, e0, e1 in done:
            e1.synchronize()
            self.data["end"][stage] += e0.elapsed_time(e1) / 1000.0
            self._free += [e0, e1]

    def read(self):
        self._resolve()
        return self.data


class MPISimulator(object):
    """One stripe of a decomposed simulation (GPUSimulators/MPISimulator.py:205-480).

    ``sim`` is this rank's simulator on its stripe (nx x ny_local cells, its
    own initial state), ``grid`` a ``StripeGrid``.  Time stepping follows
    BaseSimulator.simulate/step (GPUSimulators/Simulator.py:176-228), with the
    time step reduced over all ranks."""

    def __init__(self, sim, grid, overlap=True):
        self.logger = logging.getLogger(__name__)
        self.sim = sim
        self.grid = grid
        self._profile = HaloProfile()
        # exchange the edge rows while the interior of the stripe is computed
        # (MPISimulator.py:318-331); needs at least three tile rows
        self.overlap = False
        if overlap and hasattr(sim, "substep_rows"):
            # The exchange sends rows 0, 1 (tile row 0) and ny-2, ny-1, which lie
            # in tile rows from (ny - 2) // H on: those are the edge bands.
            rows, h = sim.tile_rows(), sim.tile_info()["tile_h"]
            self._bottom = (int(sim.ny) - 2) // h
            self.overlap = self._bottom >= 2 and rows >= 3
        self._xstream = None
        self.context = getattr(sim, "context", None)
        self.nx, self.ny, self.dx, self.dy = sim.nx, sim.ny, sim.dx, sim.dy
        self.cfl_scale = sim.cfl_scale
        self.num_substeps = sim.num_substeps
        self.t, self.nt = 0.0, 0
        self.dt = None
        bc = sim.getBoundaryConditions()
        self.boundary_conditions = bc
        _, j = grid.getCoordinate()
        new_bc, has_south, has_north = stripe_boundaries(bc, j, grid.grid[1])
        self.north = grid.getNorth() if has_north else None
        self.south = grid.getSouth() if has_south else None
        self.east = self.west = None
        sim.setBoundaryConditions(new_bc)
        self.full_exchange()
        sim.synchronize()

    # -- Simulator.py:176-217
    def simulate(self, t, dt=None):
        t_end = self.t + t
        update_dt = dt is None
        if not update_dt:
            self.dt = np.float32(dt)
        while self.t < t_end:
            if update_dt and (self.nt % 100 == 0):
                self.dt = np.float32(self.computeDt() * np.float32(self.cfl_scale))
            current_dt = np.float32(min(self.dt, t_end - self.t))
            if current_dt <= 0.0:
                break
            self.step(current_dt)
        return self.t, self.nt

    # -- Simulator.py:220-228
    def step(self, dt):
        for i in range(self.num_substeps):
            self.substep(dt, i)
        self.t = float(self.t) + float(np.float32(dt))
        self.nt += 1

    @property
    def profiling_data_mpi(self):
        """Accumulated stage times and substep count (see HaloProfile)."""
        return self._profile.read()

    def substep(self, dt, step_number):
        prof = self._profile
        prof.data["n_time_steps"] += 1
        if not self.overlap:
            stream = self.sim.comm_stream()
            tok = prof.begin(stream)
            self.sim.substep(dt, step_number)
            prof.end("t_mpi_step", tok, stream)
            self.full_exchange()
            return
        # The tile rows at the stripe's edges first; their rows go to the
        # neighbours on a second stream while the interior rows are computed,
        # and the next substep waits for both.
        sim = self.sim
        rows = sim.tile_rows()
        stream = sim.comm_stream()
        bottom = self._bottom
        tok = prof.begin(stream)
        if stream is None:
            # A host-memory simulator: each call has completed when it returns,
            # so the same band order runs without streams or events.
            sim.substep_rows(dt, step_number, 0, 1)
            sim.substep_rows(dt, step_number, bottom, rows - bottom)
            self.full_exchange(views=sim.halo_views(pending=True))
            sim.substep_rows(dt, step_number, 1, bottom - 1, last=True)
            prof.end("t_mpi_step", tok, stream)
            return
        import torch

        if self._xstream is None:
            self._xstream = torch.cuda.Stream(device=stream.device)
        sim.substep_rows(dt, step_number, 0, 1)
        sim.substep_rows(dt, step_number, bottom, rows - bottom)
        edges_done = torch.cuda.Event()
        edges_done.record(stream)
        self._xstream.wait_event(edges_done)
        self.full_exchange(views=sim.halo_views(pending=True), stream=self._xstream)
        exchanged = torch.cuda.Event()
        exchanged.record(self._xstream)
        sim.substep_rows(dt, step_number, 1, bottom - 1, last=True)
        prof.end("t_mpi_step", tok, stream)  # the stage kernels of all bands
        stream.wait_event(exchanged)

    def computeDt(self):
        return self.grid.allreduce_min(np.float32(self.sim.computeDt()))

    def full_exchange(self, views=None, stream=None):
        views = self.sim.halo_views() if views is None else views
        me = self.grid.rank
        sends, recvs = _exchange_plan(views, self.north, self.south)
        stream = self.sim.comm_stream() if stream is None else stream
        ctx = _stream_context(stream)
        prof = getattr(self, "_profile", None)
        with ctx:
            t_all = prof.begin(stream) if prof else None
            # a stripe that is its own neighbour (periodic, one rank) copies locally
            nv = len(views["north_send"])
            if self.south == me:
                for v in range(nv):
                    views["south_ghost"][v].copy_(views["north_send"][v])
            if self.north == me:
                for v in range(nv):
                    views["north_ghost"][v].copy_(views["south_send"][v])
            t_msg = prof.begin(stream) if prof else None
            with _nvtx("fv halo exchange"):
                self.grid.exchange([s for s in sends if s[0] != me], [r for r in recvs if r[0] != me])
            if prof:
                prof.end("t_mpi_halo_exchange_sendreceive", t_msg, stream)
                prof.end("t_mpi_halo_exchange", t_all, stream)

    def download(self, variables=None):
        return self.sim.download(variables) if variables is not None else self.sim.download()

    def getOutput(self):
        return self.sim.getOutput()

    def synchronize(self):
        self.sim.synchronize()

    def check(self):
        return self.sim.check()

    def simTime(self):
        return self.t

    def simSteps(self):
        return self.nt

    def getBoundaryConditions(self):
        return self.boundary_conditions

    def getExtent(self):
        """[x0, x1, y0, y1] of this rank's stripe (MPISimulator.py:357-369)."""
        width = self.nx * self.dx
        height = self.ny * self.dy
        i, j = self.grid.getCoordinate()
        x0, y0 = i * width, j * height
        return [x0, x0 + width, y0, y0 + height]


def _nvtx(name):
    """An NVTX range on a profiler's timeline (a no-op without CUDA)."""
    import contextlib

    try:
        import torch

        if torch.cuda.is_available():
            return torch.cuda.nvtx.range(name)
    except Exception:
        pass
    return contextlib.nullcontext()


def _stream_context(stream):
    if stream is None:
        import contextlib

        return contextlib.nullcontext()
    import torch

    return torch.cuda.stream(stream)


class StripedSimulator(object):
    """All stripes of one domain in one process (``sims`` ordered south to
    north, each holding its stripe's initial state): halo rows move by device
    copies ordered with CUDA events between the stripes' streams (or plain
    copies for host-memory simulators).  Results equal a single-domain run."""

    def __init__(self, sims, boundary_conditions=None):
        assert len(sims) >= 1
        self.sims = list(sims)
        s0 = self.sims[0]
        assert all(s.nx == s0.nx for s in self.sims), "stripes must have the same width"
        self.nx = s0.nx
        self.ny = sum(int(s.ny) for s in self.sims)
        self.dx, self.dy = s0.dx, s0.dy
        self.cfl_scale = s0.cfl_scale
        self.num_substeps = s0.num_substeps
        self.t, self.nt, self.dt = 0.0, 0, None
        bc = boundary_conditions or s0.getBoundaryConditions()
        self.boundary_conditions = bc
        n = len(self.sims)
        self.neighbours = []
        for j, s in enumerate(self.sims):
            new_bc, has_south, has_north = stripe_boundaries(bc, j, n)
            s.setBoundaryConditions(new_bc)
            self.neighbours.append(((j + n - 1) % n if has_south else None, (j + 1) % n if has_north else None))
        self.full_exchange()
        for s in self.sims:
            s.synchronize()

    def simulate(self, t, dt=None):
        t_end = self.t + t
        update_dt = dt is None
        if not update_dt:
            self.dt = np.float32(dt)
        while self.t < t_end:
            if update_dt and (self.nt % 100 == 0):
                self.dt = np.float32(self.computeDt() * np.float32(self.cfl_scale))
            current_dt = np.float32(min(self.dt, t_end - self.t))
            if current_dt <= 0.0:
                break
            self.step(current_dt)
        return self.t, self.nt

    def step(self, dt):
        for i in range(self.num_substeps):
            self.substep(dt, i)
        self.t = float(self.t) + float(np.float32(dt))
        self.nt += 1

    def substep(self, dt, step_number):
        for s in self.sims:
            s.substep(dt, step_number)
        self.full_exchange()

    def computeDt(self):
        return np.float32(min(np.float32(s.computeDt()) for s in self.sims))

    def full_exchange(self):
        views = [s.halo_views() for s in self.sims]
        streams = [s.comm_stream() for s in self.sims]
        events = None
        if streams[0] is not None:
            import torch

            events = []
            for st in streams:
                ev = torch.cuda.Event()
                ev.record(st)
                events.append(ev)
        for j, (south, north) in enumerate(self.neighbours):
            dst = views[j]
            pairs = []
            if south is not None:
                pairs.append((south, "south_ghost", "north_send"))
            if north is not None:
                pairs.append((north, "north_ghost", "south_send"))
            with _stream_context(streams[j]):
                for peer, ghost, send in pairs:
                    if events is not None:
                        streams[j].wait_event(events[peer])
                    for v in range(len(dst[ghost])):
                        dst[ghost][v].copy_(views[peer][send][v])

    def download(self):
        parts = [s.download() for s in self.sims]
        return [np.concatenate([p[v] for p in parts], axis=0) for v in range(len(parts[0]))]

    def synchronize(self):
        for s in self.sims:
            s.synchronize()

    def simTime(self):
        return self.t

    def simSteps(self):
        return self.nt
