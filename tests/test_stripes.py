"""Row-stripe domain decomposition (the MPISimulator counterpart), checked on the CPU.

The decomposition drivers run with oracle-backed stripes: in one process
(StripedSimulator) and as gloo ranks (MPISimulator over torch.distributed,
world sizes 2 and 3).  The stripes' arithmetic is the single-domain oracle's,
so the assembled state must equal a single-domain run bit for bit, with the
same number of steps; this checks the boundary assignment of each stripe, the
exchanged rows, the message order and the global time step.
"""

import numpy as np
import pytest

from stripe_helpers import OracleStripe, global_state, run_gloo

from finitevolumegpu_b200.MPISimulator import StripedSimulator, stripe_boundaries, stripe_rows
from finitevolumegpu_b200.Simulator import BoundaryCondition
from oracle.oracle import OracleSim

REFLECTIVE = 0x03030303
PERIODIC = 0x02020202
MIXED = 0x02020303  # north/south periodic, east/west reflective
NS_REFLECTIVE_EW_PERIODIC = 0x03030202


def single(scheme, nx, ny, bc, t_end):
    q, dx, dy, g = global_state(scheme, nx, ny)
    ref = OracleSim(scheme, q, nx, ny, dx, dy, g, cfl_scale=0.45, bc=bc)
    ref.simulate(t_end)
    return np.stack(ref.download()), ref.simSteps(), ref.simTime()


def t_end_for(scheme):
    return 0.02 if scheme == "EE2D_KP07_dimsplit" else 2.5


def test_stripe_rows_cover_domain():
    for ny, n in [(10, 3), (64, 4), (7, 7), (100, 1)]:
        parts = stripe_rows(ny, n)
        assert parts[0][0] == 0 and sum(r for _, r in parts) == ny
        assert all(parts[k + 1][0] == parts[k][0] + parts[k][1] for k in range(n - 1))
        assert max(r for _, r in parts) - min(r for _, r in parts) <= 1


def test_stripe_boundaries_follow_reference_rule():
    T = BoundaryCondition.Type
    bc = BoundaryCondition(BoundaryCondition.getTypes(NS_REFLECTIVE_EW_PERIODIC))
    new, has_s, has_n = stripe_boundaries(bc, 0, 3)
    assert (has_s, has_n) == (False, True) and new.south == T.Reflective and new.north == T.Dirichlet
    assert new.east == T.Periodic and new.west == T.Periodic
    new, has_s, has_n = stripe_boundaries(bc, 1, 3)
    assert (has_s, has_n) == (True, True) and new.south == T.Dirichlet and new.north == T.Dirichlet
    new, has_s, has_n = stripe_boundaries(bc, 2, 3)
    assert (has_s, has_n) == (True, False) and new.north == T.Reflective
    per = BoundaryCondition(BoundaryCondition.getTypes(PERIODIC))
    new, has_s, has_n = stripe_boundaries(per, 0, 1)
    assert (has_s, has_n) == (True, True) and new.north == T.Dirichlet and new.south == T.Dirichlet


@pytest.mark.parametrize("scheme,bc,n", [
    ("KP07_dimsplit", REFLECTIVE, 3),
    ("KP07_dimsplit", PERIODIC, 2),
    ("KP07_dimsplit", MIXED, 1),
    ("HLL", NS_REFLECTIVE_EW_PERIODIC, 4),
    ("KP07", MIXED, 3),
    ("WAF", REFLECTIVE, 2),
    ("EE2D_KP07_dimsplit", PERIODIC, 3),
])
def test_in_process_stripes_equal_single_domain(scheme, bc, n):
    nx, ny = 36, 45
    want, nt, t = single(scheme, nx, ny, bc, t_end_for(scheme))
    q, dx, dy, g = global_state(scheme, nx, ny)
    sims = [OracleStripe(scheme, [a[y0:y0 + r] for a in q], nx, r, dx, dy, g, cfl_scale=0.45, bc=bc)
            for y0, r in stripe_rows(ny, n)]
    striped = StripedSimulator(sims)
    striped.simulate(t_end_for(scheme))
    assert striped.simSteps() == nt and striped.simTime() == t
    got = np.stack(striped.download())
    assert np.array_equal(got, want), np.max(np.abs(got - want))


@pytest.mark.parametrize("world,scheme,bc", [
    (2, "KP07_dimsplit", PERIODIC),
    (3, "KP07_dimsplit", REFLECTIVE),
    (2, "EE2D_KP07_dimsplit", PERIODIC),
])
def test_gloo_ranks_equal_single_domain(tmp_path, world, scheme, bc):
    nx, ny = 30, 42
    want, nt, t = single(scheme, nx, ny, bc, t_end_for(scheme))
    res = run_gloo(world, scheme, nx, ny, bc, t_end_for(scheme), str(tmp_path / "out.npz"))
    assert int(res["nt"]) == nt and float(res["t"]) == t
    assert np.array_equal(res["state"], want), np.max(np.abs(res["state"] - want))


@pytest.mark.parametrize("world,scheme,bc", [
    (2, "KP07_dimsplit", PERIODIC),               # 21-row stripes: rows ny-2 and ny-1 in different tile rows
    (3, "KP07_dimsplit", REFLECTIVE),             # 14-row stripes: both in the last tile row
    (2, "KP07", MIXED),                           # RK2: stage 2 blends into the buffer being written
    (1, "HLL2", PERIODIC),                        # a stripe that is its own neighbour: local copies
    (2, "HLL", NS_REFLECTIVE_EW_PERIODIC),        # one ghost row
])
def test_gloo_overlapped_schedule_equals_single_domain(tmp_path, world, scheme, bc):
    """MPISimulator's overlapped substep (edge tile rows, the exchange into the
    buffer being written, then the interior rows) gives the single-domain run
    bit for bit: the edge bands hold every row that is sent."""
    nx, ny = 30, 42
    want, nt, t = single(scheme, nx, ny, bc, t_end_for(scheme))
    res = run_gloo(world, scheme, nx, ny, bc, t_end_for(scheme), str(tmp_path / "out.npz"), banded=True)
    assert int(res["nt"]) == nt and float(res["t"]) == t
    assert np.array_equal(res["state"], want), np.max(np.abs(res["state"] - want))


def test_run_simulation_returns_reference_profiling(tmp_path):
    """runSimulation over an MPISimulator returns the reference's profiling
    dictionaries, and the reference driver's aggregation (end - start per
    stage, n_time_steps) runs on them: two gloo ranks, overlapped schedule."""
    from stripe_helpers import run_profiling_gloo

    prof = run_profiling_gloo(2, str(tmp_path / "prof.json"))
    for stage in ("t_sim_init", "t_nc_write", "t_full_step", "t_mpi_step", "t_mpi_halo_exchange",
                  "t_mpi_halo_exchange_sendreceive", "t_mpi_halo_exchange_download", "t_mpi_halo_exchange_upload"):
        assert stage in prof and prof[stage] >= 0.0, (stage, prof)
    assert prof["t_mpi_step"] > 0.0 and prof["t_mpi_halo_exchange_sendreceive"] > 0.0
    assert prof["t_mpi_halo_exchange"] >= prof["t_mpi_halo_exchange_sendreceive"]
    assert prof["t_mpi_halo_exchange_download"] == 0 and prof["t_mpi_halo_exchange_upload"] == 0
    # two substeps per KP07_dimsplit step; at least the 2-second run's steps
    assert prof["n_time_steps"] >= 2 and prof["n_time_steps"] % 2 == 0
