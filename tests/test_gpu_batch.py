"""Batched and served simulations give the same results as plain ones.

Each simulation in a batch keeps its own CFL time step and t_end, so its
result must equal a plain simulator's simulate(t_end) of the same scenario,
alone or mixed with other simulations, whatever joins or leaves the batch in
between.  The product kernels are the same code in both paths, so the results
are compared exactly (tolerance 0), plus against the CPU oracle.
"""

import numpy as np
import pytest

from conftest import bump, dam_break, kelvin_helmholtz, rel_linf

import finitevolumegpu_b200 as fv
from finitevolumegpu_b200.batch import Batch
from finitevolumegpu_b200.server import Request, Server
from oracle.oracle import OracleSim

pytestmark = pytest.mark.gpu

PERIODIC = fv.BoundaryCondition(fv.BoundaryCondition.getTypes(0x02020202))


def scenario(scheme, nx, ny, kind, seed):
    rng = np.random.default_rng(seed)
    if scheme == "EE2D_KP07_dimsplit":
        return kelvin_helmholtz(nx, ny, phase=rng.uniform(0, 6.28)), 1.0 / nx, 1.0 / ny, 0.02 + 0.03 * rng.random()
    if kind == "bump":
        q = bump(nx, ny, amp=rng.uniform(0.1, 0.5), cx=rng.uniform(0.3, 0.7) * nx, cy=rng.uniform(0.3, 0.7) * ny,
                 sigma=min(20.0, min(nx, ny) / 4))
    else:
        q = dam_break(nx, ny, radius_frac=rng.uniform(0.1, 0.3))
    return list(q), 1.0, 1.0, float(rng.uniform(2.0, 8.0))


def plain(ctx, scheme, q, nx, ny, dx, dy, t_end, bc=None):
    cls = fv.SCHEMES[scheme]
    kw = {} if bc is None else {"boundary_conditions": bc}
    if scheme == "EE2D_KP07_dimsplit":
        sim = cls(ctx, *q, nx, ny, dx, dy, 0.0, 1.4, **kw)
    else:
        sim = cls(ctx, *q, nx, ny, dx, dy, 9.81, **kw)
    sim.simulate(t_end)
    return sim.download(), sim.simSteps(), sim.simTime()


SIZES = [(64, 64), (97, 150), (300, 70), (130, 131), (33, 200), (250, 250)]


@pytest.mark.parametrize("scheme", ["KP07_dimsplit", "HLL", "EE2D_KP07_dimsplit", "HLL2", "WAF", "FORCE", "LxF",
                                    "KP07"])
def test_batch_equals_plain(ctx, scheme):
    b = Batch(ctx, scheme, g=0.0 if scheme == "EE2D_KP07_dimsplit" else 9.81, max_instances=16)
    bc = PERIODIC if scheme == "EE2D_KP07_dimsplit" else None
    cases = {}
    for k, (nx, ny) in enumerate(SIZES):
        q, dx, dy, t_end = scenario(scheme, nx, ny, "bump" if k % 2 else "dam", k)
        slot = b.add(q, nx, ny, dx, dy, t_end, bc)
        cases[slot] = (q, nx, ny, dx, dy, t_end)
    b.run_to_completion()
    many = dict(zip(cases, b.download_many(list(cases), threads=4)))
    for slot, (q, nx, ny, dx, dy, t_end) in cases.items():
        st = b.status(slot)
        got = b.download(slot)
        for a, m in zip(got, many[slot]):
            assert np.array_equal(a, m)  # the threaded download returns the same arrays
        want, nt, t = plain(ctx, scheme, q, nx, ny, dx, dy, t_end, bc)
        assert st["nt"] == nt and st["t"] == t, (slot, st, nt, t)
        for a, w in zip(got, want):
            assert np.array_equal(a, w), (scheme, slot, rel_linf(a, w))


RAGGED = [(2, 2), (3, 200), (200, 3), (99, 57), (125, 29), (61, 61), (131, 7)]


@pytest.mark.parametrize("scheme", ["KP07_dimsplit", "HLL", "EE2D_KP07_dimsplit", "LxF", "KP07"])
def test_batch_ragged_sizes_equal_plain(ctx, scheme):
    """Batched tiles are copied into shared memory by the threads (16-byte
    chunks) where the plain kernels use a tensor copy; on degenerate and ragged
    grids (a chunk straddling the tensor map's nx + 8 columns, tiles reaching
    past the stored rows, strips narrower than a tile) both must hold the same
    values, so the results are equal bit for bit."""
    b = Batch(ctx, scheme, g=0.0 if scheme == "EE2D_KP07_dimsplit" else 9.81, max_instances=16)
    cases = {}
    for k, (nx, ny) in enumerate(RAGGED):
        q, dx, dy, t_end = scenario(scheme, nx, ny, "bump" if k % 2 else "dam", 100 + k)
        bc = PERIODIC if (scheme == "EE2D_KP07_dimsplit" or k % 3 == 1) else None
        slot = b.add(q, nx, ny, dx, dy, t_end, bc)
        cases[slot] = (q, nx, ny, dx, dy, t_end, bc)
    b.run_to_completion()
    for slot, (q, nx, ny, dx, dy, t_end, bc) in cases.items():
        st = b.status(slot)
        got = b.download(slot)
        want, nt, t = plain(ctx, scheme, q, nx, ny, dx, dy, t_end, bc)
        assert st["nt"] == nt and st["t"] == t, (scheme, nx, ny, st, nt, t)
        for a, w in zip(got, want):
            assert np.array_equal(a, w, equal_nan=True), (scheme, nx, ny, rel_linf(a, w))


def test_batch_kp07_first_order_equals_plain(ctx):
    """KP07 of order 1: one Runge-Kutta stage per step and computeDt's factor
    1 (GPUSimulators/KP07.py:138), for every simulation of the batch."""
    b = Batch(ctx, "KP07", order=1, cfl_scale=0.45, max_instances=4)
    cases = {}
    for k, (nx, ny) in enumerate([(97, 150), (130, 131)]):
        q, dx, dy, t_end = scenario("KP07", nx, ny, "bump" if k else "dam", k)
        cases[b.add(q, nx, ny, dx, dy, t_end)] = (q, nx, ny, dx, dy, t_end)
    b.run_to_completion()
    for slot, (q, nx, ny, dx, dy, t_end) in cases.items():
        sim = fv.KP07.KP07(ctx, *q, nx, ny, dx, dy, 9.81, cfl_scale=0.45, order=1)
        sim.simulate(t_end)
        st = b.status(slot)
        assert st["nt"] == sim.simSteps() and st["t"] == sim.simTime()
        for a, w in zip(b.download(slot), sim.download()):
            assert np.array_equal(a, w), (slot, rel_linf(a, w))


def test_batch_matches_oracle(ctx):
    b = Batch(ctx, "KP07_dimsplit", max_instances=4)
    q, dx, dy, t_end = scenario("KP07_dimsplit", 90, 70, "bump", 7)
    slot = b.add(q, 90, 70, dx, dy, t_end)
    b.run_to_completion()
    ref = OracleSim("KP07_dimsplit", q, 90, 70, dx, dy, 9.81)
    ref.simulate(t_end)
    assert b.status(slot)["nt"] == ref.nt
    for a, w in zip(b.download(slot), ref.download()):
        assert rel_linf(a, w) < 2e-5


def test_batch_work_list_grows(ctx):
    """Tiles beyond the initial work list (4096 entries) grow it, the second
    time after the step graphs were captured on the old list, and every
    simulation still equals its plain solve."""
    b = Batch(ctx, "KP07_dimsplit", max_instances=32, tile=0)
    info = b.info()
    nx, ny = 1024, 512
    per = -(-nx // info["tile_w"]) * -(-ny // info["tile_h"])  # 342 tiles of 60 x 28
    cases = {}

    def add_until(tiles):
        while len(cases) * per <= tiles:
            k = len(cases)
            q, dx, dy, t_end = scenario("KP07_dimsplit", nx, ny, "bump" if k % 2 else "dam", 100 + k)
            cases[b.add(q, nx, ny, dx, dy, t_end)] = (q, dx, dy, t_end)

    add_until(4096)
    b.run(2)
    b.sync()
    assert b.info()["work_items"] == len(cases) * per > 4096
    add_until(8192)
    b.run_to_completion()
    assert b.info()["work_items"] == len(cases) * per > 8192
    for slot, (q, dx, dy, t_end) in cases.items():
        want, nt, _ = plain(ctx, "KP07_dimsplit", q, nx, ny, dx, dy, t_end)
        assert b.status(slot)["nt"] == nt
        for a, w in zip(b.download(slot), want):
            assert np.array_equal(a, w)


def test_batch_join_and_leave(ctx):
    """Simulations join and leave between chunks without disturbing the others."""
    b = Batch(ctx, "KP07_dimsplit", max_instances=8)
    cases = {}
    for k, (nx, ny) in enumerate(SIZES[:3]):
        q, dx, dy, t_end = scenario("KP07_dimsplit", nx, ny, "bump", 10 + k)
        cases[b.add(q, nx, ny, dx, dy, t_end)] = (q, nx, ny, dx, dy, t_end)
    b.run(5)
    b.sync()
    victim = next(iter(cases))
    b.remove(victim)
    del cases[victim]
    for k, (nx, ny) in enumerate(SIZES[3:]):
        q, dx, dy, t_end = scenario("KP07_dimsplit", nx, ny, "dam", 20 + k)
        cases[b.add(q, nx, ny, dx, dy, t_end)] = (q, nx, ny, dx, dy, t_end)
    b.run_to_completion()
    for slot, (q, nx, ny, dx, dy, t_end) in cases.items():
        want, nt, _ = plain(ctx, "KP07_dimsplit", q, nx, ny, dx, dy, t_end)
        assert b.status(slot)["nt"] == nt
        for a, w in zip(b.download(slot), want):
            assert np.array_equal(a, w)


def test_server_same_alone_and_in_mix(ctx):
    """Requests arriving over time, three schemes mixed, each result equal to a solo run."""
    rng = np.random.default_rng(3)
    reqs = []
    schemes = ["KP07_dimsplit", "HLL", "EE2D_KP07_dimsplit"]
    for i in range(18):
        s = schemes[i % 3]
        nx, ny = int(rng.integers(40, 200)), int(rng.integers(40, 200))
        q, dx, dy, t_end = scenario(s, nx, ny, "bump" if i % 2 else "dam", 100 + i)
        bc = PERIODIC if s == "EE2D_KP07_dimsplit" else None
        reqs.append(Request(i, s, q, nx, ny, dx, dy, t_end, arrival=0.002 * i, boundary_conditions=bc))
    server = Server(ctx, budget_bytes=2e9, chunk_steps=4, max_instances=64)
    results, stats = server.serve(reqs)
    assert stats["requests"] == len(reqs)
    assert stats["p99_latency_s"] >= stats["p50_latency_s"] > 0
    by_id = {r.rid: r for r in results}
    for r in reqs:
        res = by_id[r.rid]
        want, nt, t = plain(ctx, r.scheme, r.variables, r.nx, r.ny, r.dx, r.dy, r.t_end, r.boundary_conditions)
        assert res.steps == nt and res.t == t
        for a, w in zip(res.state, want):
            assert np.array_equal(a, w), (r.rid, r.scheme, rel_linf(a, w))


def test_server_respects_memory_budget(ctx):
    """With a budget for about two scenarios at a time, all requests still complete."""
    reqs = []
    for i in range(6):
        q, dx, dy, t_end = scenario("KP07_dimsplit", 256, 256, "bump", 200 + i)
        reqs.append(Request(i, "KP07_dimsplit", q, 256, 256, dx, dy, t_end, arrival=0.0))
    server = Server(ctx, budget_bytes=2.5 * 2 * 3 * 260 * 288 * 4, chunk_steps=8, schemes=["KP07_dimsplit"])
    results, stats = server.serve(reqs)
    assert stats["requests"] == 6
    admitted = sorted(r.admitted for r in results)
    assert admitted[-1] > admitted[0]  # later requests waited for memory


def test_batch_failed_simulations_stop_and_the_others_match_plain(ctx):
    """Corrupted initial states fail alone: a NaN depth makes the initial time
    step NaN (control-block check); a NaN in hv alone leaves the time step
    finite (the reference's min over axes drops it), so the stage kernel's
    per-step health check must catch it.  Both stop, the other simulations
    of the batch equal their plain runs bit for bit."""
    b = Batch(ctx, "KP07_dimsplit", max_instances=8)
    cases = {}
    bad = {}
    for k, (nx, ny) in enumerate([(97, 150), (130, 131), (64, 64), (250, 120)]):
        q, dx, dy, t_end = scenario("KP07_dimsplit", nx, ny, "bump" if k % 2 else "dam", 40 + k)
        if k == 1:
            q = [a.copy() for a in q]
            q[0][ny // 2, nx // 3] = np.nan
        if k == 2:
            q = [a.copy() for a in q]
            q[2][5, 7] = np.nan
        slot = b.add(q, nx, ny, dx, dy, t_end)
        (bad if k in (1, 2) else cases)[slot] = (q, nx, ny, dx, dy, t_end)
    b.run_to_completion()
    for slot in bad:
        st = b.status(slot)
        assert st["done"] and st["failed"], st
        assert st["nt"] <= 1  # stopped at once
    for slot, (q, nx, ny, dx, dy, t_end) in cases.items():
        st = b.status(slot)
        assert st["done"] and not st["failed"]
        want, nt, t = plain(ctx, "KP07_dimsplit", q, nx, ny, dx, dy, t_end)
        assert st["nt"] == nt and st["t"] == t
        for a, w in zip(b.download(slot), want):
            assert np.array_equal(a, w)


def test_server_isolates_bad_requests(ctx):
    """A corrupted initial state comes back failed, a wrong shape rejected, an
    unknown scheme rejected; every other request equals its solo run."""
    reqs = []
    for i in range(9):
        s = ("KP07_dimsplit", "HLL", "KP07", "LxF")[i % 4]
        nx, ny = 60 + 13 * i, 90 - 5 * i
        q, dx, dy, t_end = scenario(s, nx, ny, "bump" if i % 3 else "dam", 300 + i)
        reqs.append(Request(i, s, q, nx, ny, dx, dy, t_end, arrival=0.001 * i))
    reqs[2].variables = [a.copy() for a in reqs[2].variables]
    reqs[2].variables[1][3, 4] = np.inf  # corrupted momentum
    reqs[5].variables = [a[:-1] for a in reqs[5].variables]  # one row short
    reqs[7].scheme = "MUSCL"  # no such scheme
    results, stats = Server(ctx, budget_bytes=2e9, chunk_steps=4, max_instances=32).serve(reqs)
    by = {r.rid: r for r in results}
    assert len(results) == 9
    assert by[2].status == "failed" and by[2].state is None
    assert by[5].status == "rejected" and "shape" in by[5].error
    assert by[7].status == "rejected"
    assert stats["requests"] == 6 and stats["failed"] == 1 and stats["rejected"] == 2
    for r in reqs:
        if r.rid in (2, 5, 7):
            continue
        res = by[r.rid]
        assert res.status == "done"
        want, nt, t = plain(ctx, r.scheme, r.variables, r.nx, r.ny, r.dx, r.dy, r.t_end)
        assert res.steps == nt and res.t == t
        for a, w in zip(res.state, want):
            assert np.array_equal(a, w), (r.rid, rel_linf(a, w))
