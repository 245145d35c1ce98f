"""Row-stripe decomposition on the GPU: decomposed runs equal single-domain runs.

StripedSimulator runs 2-4 stripes of one domain on this GPU, each an ordinary
simulator with Dirichlet internal edges, exchanging two rows per substep by
device copies on the stripes' streams; MPISimulator runs one NCCL rank whose
periodic north/south neighbour is itself.  The stage kernels compute each
cell identically whatever tile it falls in, and the global time step is the
minimum of the stripes' CFL minima, so the assembled state must equal the
single-domain simulate() bit for bit, with the same step count.
"""

import datetime
import os

import numpy as np
import pytest

from stripe_helpers import free_port, global_state

import finitevolumegpu_b200 as fv
from finitevolumegpu_b200.MPISimulator import MPISimulator, StripedSimulator, StripeGrid, stripe_rows

pytestmark = pytest.mark.gpu

REFLECTIVE = 0x03030303
PERIODIC = 0x02020202
MIXED = 0x02020303


def make(ctx, scheme, q, nx, ny, dx, dy, g, bc):
    cls = fv.SCHEMES[scheme]
    b = fv.BoundaryCondition(fv.BoundaryCondition.getTypes(bc))
    if scheme == "EE2D_KP07_dimsplit":
        return cls(ctx, *q, nx, ny, dx, dy, g, 1.4, boundary_conditions=b, cfl_scale=0.45)
    return cls(ctx, *q, nx, ny, dx, dy, g, boundary_conditions=b, cfl_scale=0.45)


def t_end_for(scheme):
    return 0.03 if scheme == "EE2D_KP07_dimsplit" else 4.0


@pytest.mark.parametrize("scheme,bc,n", [
    ("KP07_dimsplit", REFLECTIVE, 2),
    ("KP07_dimsplit", PERIODIC, 3),
    ("KP07_dimsplit", MIXED, 1),
    ("HLL", REFLECTIVE, 4),
    ("HLL2", MIXED, 2),
    ("KP07", PERIODIC, 3),
    ("EE2D_KP07_dimsplit", PERIODIC, 2),
])
def test_striped_equals_single_domain(ctx, scheme, bc, n):
    nx, ny = 200, 251
    q, dx, dy, g = global_state(scheme, nx, ny, seed=4)
    ref = make(ctx, scheme, q, nx, ny, dx, dy, g, bc)
    ref.simulate(t_end_for(scheme))
    want = np.stack(ref.download())
    sims = [make(ctx, scheme, [a[y0:y0 + r] for a in q], nx, r, dx, dy, g, bc) for y0, r in stripe_rows(ny, n)]
    striped = StripedSimulator(sims)
    striped.simulate(t_end_for(scheme))
    assert striped.simSteps() == ref.simSteps()
    assert striped.simTime() == ref.simTime()
    got = np.stack(striped.download())
    assert np.array_equal(got, want), float(np.max(np.abs(got - want)))


def test_one_nccl_rank_periodic_self_exchange(ctx):
    import torch
    import torch.distributed as dist

    nx, ny = 160, 120
    q, dx, dy, g = global_state("KP07_dimsplit", nx, ny, seed=5)
    ref = make(ctx, "KP07_dimsplit", q, nx, ny, dx, dy, g, PERIODIC)
    ref.simulate(3.0)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % free_port(), rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        sim = make(ctx, "KP07_dimsplit", q, nx, ny, dx, dy, g, PERIODIC)
        mpi = MPISimulator(sim, StripeGrid())
        mpi.simulate(3.0)
        assert mpi.simSteps() == ref.simSteps()
        for a, b in zip(mpi.download(), ref.download()):
            assert np.array_equal(a, b)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("scheme", ["KP07_dimsplit", "KP07", "HLL", "EE2D_KP07_dimsplit"])
def test_substep_bands_equal_substep(ctx, scheme):
    """A substep launched as bands of tile rows (edges first, then the
    interior, as MPISimulator overlaps them with the exchange) equals the
    single launch bit for bit, CFL reduction included."""
    nx, ny = 150, 230
    q, dx, dy, g = global_state(scheme, nx, ny, seed=6)
    a = make(ctx, scheme, q, nx, ny, dx, dy, g, MIXED)
    b = make(ctx, scheme, q, nx, ny, dx, dy, g, MIXED)
    rows = b.tile_rows()
    assert rows >= 3
    dt = np.float32(a.computeDt() * np.float32(0.45))
    for _ in range(3):
        for i in range(a.num_substeps):
            a.substep(dt, i)
            b.substep_rows(dt, i, 0, 1)
            b.substep_rows(dt, i, rows - 1, 1)
            b.substep_rows(dt, i, 1, rows - 2, last=True)
    assert a.computeDt() == b.computeDt()
    for x, y in zip(a.download(), b.download()):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("ny", [200, 181])  # 181: the last tile row of 60 holds one row
def test_nccl_overlap_equals_plain_exchange(ctx, ny):
    import torch
    import torch.distributed as dist

    nx = 160
    q, dx, dy, g = global_state("KP07_dimsplit", nx, ny, seed=7)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % free_port(), rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        outs = []
        for overlap in (False, True):
            sim = make(ctx, "KP07_dimsplit", q, nx, ny, dx, dy, g, PERIODIC)
            mpi = MPISimulator(sim, StripeGrid(), overlap=overlap)
            assert mpi.overlap == overlap
            mpi.simulate(3.0)
            outs.append((mpi.download(), mpi.simSteps()))
            # the reference's profiling dictionary, timed with CUDA events
            prof = mpi.profiling_data_mpi
            assert prof["n_time_steps"] == 2 * mpi.simSteps()
            assert prof["end"]["t_mpi_step"] - prof["start"]["t_mpi_step"] > 0.0
            assert prof["end"]["t_mpi_halo_exchange"] >= prof["end"]["t_mpi_halo_exchange_sendreceive"] >= 0.0
        (a, na), (b, nb) = outs
        assert na == nb
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
    finally:
        dist.destroy_process_group()
