"""Test helpers for the row-stripe decomposition on the CPU.

``OracleStripe`` gives the CPU oracle the local-simulator interface that
``MPISimulator`` and ``StripedSimulator`` drive (halo rows as torch views of its
host arrays, no stream), so the decomposition logic and its message plan can
be checked against a single-domain oracle run with gloo ranks, without a GPU.
"""

import os
import socket

import numpy as np

from oracle.oracle import DIMSPLIT_HALF_DT, OracleSim


class OracleStripe(OracleSim):
    """OracleSim with the local-simulator interface of the stripe drivers."""

    def getBoundaryConditions(self):
        from finitevolumegpu_b200.Simulator import BoundaryCondition

        return BoundaryCondition(BoundaryCondition.getTypes(self.bc))

    def setBoundaryConditions(self, bc):
        self.bc = int(bc.asCodedInt())

    def halo_views(self, pending=False):
        """Views of the current state's edge and ghost rows; with pending=True
        of the buffer a substep in progress writes (BandedOracleStripe)."""
        import torch

        g, ny = self.gc, self.ny
        bufs = self.u1 if pending else self.u0

        def rows(a, r0):
            return torch.from_numpy(a[r0:r0 + g].reshape(-1))

        return {"south_ghost": [rows(a, 0) for a in bufs], "south_send": [rows(a, g) for a in bufs],
                "north_send": [rows(a, ny) for a in bufs], "north_ghost": [rows(a, ny + g) for a in bufs]}

    def comm_stream(self):
        return None

    def synchronize(self):
        pass

    def check(self):
        for a in self.u0:
            assert np.all(np.isfinite(a[self.gc:self.gc + self.ny, self.gc:self.gc + self.nx])), "NaN in state"


class BandedOracleStripe(OracleStripe):
    """OracleStripe that also runs a substep in bands of tile rows, as the GPU
    simulators' substep_rows does, so MPISimulator takes its overlapped
    schedule (edge bands, exchange into the pending buffer, interior band).
    A band writes only its rows of the output buffer: the full substep is
    computed into a copy of that buffer and the band's rows are copied back
    (the oracle, like the kernels, writes interior cells only).  The buffers
    swap after the band marked last, whose CFL is the full grid's."""

    TILE_H = 4

    def tile_rows(self):
        return -(-self.ny // self.TILE_H)

    def tile_info(self):
        return {"tile_h": self.TILE_H}

    def substep_rows(self, dt, step_number, row0, nrows, last=False):
        T = self.dtype.type
        dt = T(dt)
        kdt = T(dt * T(0.5)) if self.scheme in DIMSPLIT_HALF_DT else dt
        out = self.u1
        self.u1 = [a.copy() for a in out]
        cfl = self._launch(kdt, int(step_number))
        full, self.u1 = self.u1, out
        y0 = self.gc + row0 * self.TILE_H
        y1 = self.gc + min((row0 + nrows) * self.TILE_H, self.ny)
        for a, f in zip(out, full):
            a[y0:y1] = f[y0:y1]
        if last:
            if self.scheme != "WAF":
                self.cfl = cfl
            self.u0, self.u1 = self.u1, self.u0


def global_state(scheme, nx, ny, seed=0):
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:ny, 0:nx] + 0.5
    if scheme == "EE2D_KP07_dimsplit":
        band = (y >= 0.25 * ny) & (y < 0.75 * ny)
        rho = np.where(band, 2.0, 1.0)
        u = np.where(band, 0.5, -0.5)
        v = 0.01 * np.sin(4 * np.pi * x / nx + rng.uniform(0, 6.28))
        q = [rho, rho * u, rho * v, 2.5 / 0.4 + 0.5 * rho * (u * u + v * v)]
        return [a.astype(np.float32) for a in q], 1.0 / nx, 1.0 / ny, 0.0
    cx, cy = rng.uniform(0.3, 0.7) * nx, rng.uniform(0.3, 0.7) * ny
    h = 1.0 + 0.4 * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * (min(nx, ny) / 6.0) ** 2))
    h = np.where(np.hypot(x - 0.7 * nx, y - 0.3 * ny) < 0.1 * min(nx, ny), 1.6, h)  # a small dam as well
    z = np.zeros_like(h)
    return [h.astype(np.float32), z.astype(np.float32), z.astype(np.float32)], 1.0, 1.0, 9.81


def free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def gloo_worker(rank, world, port, scheme, nx, ny, bc, t_end, out_path, banded=False):
    """One rank of a gloo run: simulate this rank's stripe and gather to rank 0
    (banded: with the overlapped schedule of banded substeps)."""
    import datetime

    import torch.distributed as dist

    from finitevolumegpu_b200.MPISimulator import MPISimulator, StripeGrid, stripe_rows

    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        q, dx, dy, g = global_state(scheme, nx, ny)
        y0, rows = stripe_rows(ny, world)[rank]
        local = [a[y0:y0 + rows] for a in q]
        cls = BandedOracleStripe if banded else OracleStripe
        sim = cls(scheme, local, nx, rows, dx, dy, g, cfl_scale=0.45, bc=bc)
        mpi = MPISimulator(sim, StripeGrid())
        if mpi.overlap != banded:
            raise RuntimeError("overlapped schedule %s, expected %s" % (mpi.overlap, banded))
        mpi.simulate(t_end)
        parts = mpi.grid.gather(np.stack(mpi.download()))
        if rank == 0:
            full = np.concatenate(parts, axis=1)
            np.savez(out_path, state=full, nt=mpi.simSteps(), t=mpi.simTime())
    finally:
        dist.destroy_process_group()


def run_gloo(world, scheme, nx, ny, bc, t_end, out_path, banded=False):
    import torch.multiprocessing as mp

    os.environ.setdefault("GLOO_SOCKET_IFNAME", "lo")
    mp.start_processes(gloo_worker, args=(world, free_port(), scheme, nx, ny, bc, t_end, out_path, banded),
                       nprocs=world, join=True, start_method="spawn")
    return np.load(out_path)


def profiling_worker(rank, world, port, out_path):
    """One rank of a gloo run of Common.runSimulation over an MPISimulator,
    with the reference driver's profile aggregation (mpiTesting.py:171-177)
    applied to the returned dictionaries on rank 0."""
    import datetime
    import json

    import torch.distributed as dist

    from finitevolumegpu_b200.Common import runSimulation
    from finitevolumegpu_b200.MPISimulator import MPISimulator, StripeGrid, stripe_rows

    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        nx, ny = 40, 24
        q, dx, dy, g = global_state("KP07_dimsplit", nx, ny)
        y0, rows = stripe_rows(ny, world)[rank]
        grid = StripeGrid()

        def gen_sim(nx, ny, dx, dy, g, h0, hu0, hv0):
            sim = BandedOracleStripe("KP07_dimsplit", [h0, hu0, hv0], nx, ny, dx, dy, g, cfl_scale=0.45,
                                     bc=0x03030303)
            return MPISimulator(sim, grid)

        args = {"nx": nx, "ny": rows, "dx": dx, "dy": dy, "g": g,
                "h0": q[0][y0:y0 + rows], "hu0": q[1][y0:y0 + rows], "hv0": q[2][y0:y0 + rows]}
        outfile, sim_runner_profiling_data, sim_profiling_data = runSimulation(
            gen_sim, args, out_path + ".%d.nc" % rank, [0.0, 1.0, 2.0], ["h", "hu", "hv"])
        profiling_data = {}
        for stage in sim_runner_profiling_data["start"].keys():
            profiling_data[stage] = sim_runner_profiling_data["end"][stage] - sim_runner_profiling_data["start"][stage]
        for stage in sim_profiling_data["start"].keys():
            profiling_data[stage] = sim_profiling_data["end"][stage] - sim_profiling_data["start"][stage]
        profiling_data["n_time_steps"] = sim_profiling_data["n_time_steps"]
        if rank == 0:
            with open(out_path, "w") as f:
                json.dump(profiling_data, f)
    finally:
        dist.destroy_process_group()


def run_profiling_gloo(world, out_path):
    import json

    import torch.multiprocessing as mp

    os.environ.setdefault("GLOO_SOCKET_IFNAME", "lo")
    mp.start_processes(profiling_worker, args=(world, free_port(), out_path), nprocs=world, join=True,
                       start_method="spawn")
    with open(out_path) as f:
        return json.load(f)
