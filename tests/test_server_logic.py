"""The server's scheduling logic on the CPU, with a stand-in for the GPU batch:
every request is served exactly once with its own result, the device-memory
budget is never exceeded, bursts go through the admission threads and single
arrivals are admitted inline, an admission that finds the GPU full is
retried once memory has been released, and a request that cannot run or
whose state goes bad comes back rejected or failed while the others are
served as usual."""

import threading

import numpy as np
import pytest

import finitevolumegpu_b200.server as server
from finitevolumegpu_b200.server import Request, Server, state_bytes


class FakeBatch(object):
    """Advances each admitted scenario by dt = 1 per step up to its t_end."""

    instances = []
    full_once = set()  # rids whose first admission reports a full GPU
    fail_after = {}  # rid -> steps after which its state goes bad (the batch marks it failed)

    def __init__(self, context, scheme, g=9.81, gamma=1.4, cfl_scale=0.9, max_instances=4096, **kw):
        self.scheme = scheme
        self.lock = threading.Lock()
        self.slots = {}
        self.next = 0
        self.add_threads = set()
        FakeBatch.instances.append(self)

    def add(self, variables, nx, ny, dx, dy, t_end, boundary_conditions=None):
        assert len(variables) == 3, "KP07_dimsplit takes 3 conserved variables, got %d" % len(variables)
        assert all(a.shape == (ny, nx) for a in variables), "Wrong shape of data"
        rid = int(variables[0][0, 0])
        with self.lock:
            if rid in FakeBatch.full_once:
                FakeBatch.full_once.discard(rid)
                raise MemoryError("full")
            slot = self.next
            self.next += 1
            self.slots[slot] = {"rid": rid, "t": 0.0, "nt": 0, "t_end": float(t_end), "registered": True}
            self.add_threads.add(threading.current_thread().name)
        return slot

    def run(self, n):
        with self.lock:
            for st in self.slots.values():
                for _ in range(n):
                    if st["t"] < st["t_end"] and not st.get("bad"):
                        st["t"] += 1.0
                        st["nt"] += 1
                        if st["nt"] == FakeBatch.fail_after.get(st["rid"]):
                            st["bad"] = True

    def sync(self):
        pass

    def status(self, slot):
        with self.lock:
            st = self.slots[slot]
            bad = bool(st.get("bad"))
            return {"t": st["t"], "nt": st["nt"], "dt": 1.0, "done": bad or st["t"] >= st["t_end"], "failed": bad}

    nv = 3

    def download(self, slot, scratch=None):
        with self.lock:
            st = self.slots[slot]
            return [np.full((2, 2), st["rid"], dtype=np.float32)]

    def remove(self, slot):
        with self.lock:
            del self.slots[slot]


@pytest.fixture
def fake(monkeypatch):
    FakeBatch.instances = []
    FakeBatch.full_once = set()
    FakeBatch.fail_after = {}
    monkeypatch.setattr(server, "Batch", FakeBatch)
    return FakeBatch


def requests(n, spacing, sizes=(64, 96)):
    out = []
    for i in range(n):
        nx = sizes[i % len(sizes)]
        v = [np.full((nx, nx), i, dtype=np.float32)] * 3
        out.append(Request(i, "KP07_dimsplit", v, nx, nx, 1.0, 1.0, float(3 + i % 5), arrival=i * spacing))
    return out


def test_every_request_served_once_with_its_own_result(fake):
    reqs = requests(40, 0.0)  # one burst
    results, stats = Server(None, budget_bytes=1e12, chunk_steps=2, schemes=("KP07_dimsplit",)).serve(reqs)
    assert sorted(r.rid for r in results) == list(range(40))
    for r in results:
        assert r.state[0][0, 0] == r.rid
        assert r.steps == 3 + r.rid % 5 and r.t == r.steps
    assert stats["requests"] == 40
    # a burst of arrivals is uploaded by the admission threads
    assert any(name.startswith("fvgpu-admit") for b in fake.instances for name in b.add_threads)


def test_single_arrivals_admitted_inline(fake):
    reqs = requests(6, 0.02)
    results, _ = Server(None, budget_bytes=1e12, chunk_steps=1, schemes=("KP07_dimsplit",)).serve(reqs)
    assert sorted(r.rid for r in results) == list(range(6))
    names = set().union(*(b.add_threads for b in fake.instances))
    assert names == {threading.main_thread().name}


def test_budget_respected(fake, monkeypatch):
    reqs = requests(30, 0.0)
    need = max(state_bytes("KP07_dimsplit", r.nx, r.ny) for r in reqs)
    budget = 3.5 * need  # at most three scenarios on the device at a time
    peak = {"used": 0.0}
    srv = Server(None, budget_bytes=budget, chunk_steps=1, schemes=("KP07_dimsplit",))
    orig_run = FakeBatch.run

    def run(self, n):
        peak["used"] = max(peak["used"], srv.used)
        orig_run(self, n)

    monkeypatch.setattr(FakeBatch, "run", run)
    results, _ = srv.serve(reqs)
    assert sorted(r.rid for r in results) == list(range(30))
    assert peak["used"] <= budget
    assert srv.used == 0.0


def test_full_gpu_admission_is_retried(fake):
    reqs = requests(12, 0.0)
    fake.full_once = {3, 7}
    results, _ = Server(None, budget_bytes=1e12, chunk_steps=2, schemes=("KP07_dimsplit",)).serve(reqs)
    assert sorted(r.rid for r in results) == list(range(12))


def done_ids(results):
    return sorted(r.rid for r in results if r.status == "done")


def test_request_larger_than_the_budget_is_rejected(fake):
    reqs = requests(3, 0.0, sizes=(64, 200))  # 1 is 200 x 200
    budget = 0.9 * state_bytes("KP07_dimsplit", 200, 200)
    results, stats = Server(None, budget_bytes=budget, chunk_steps=1, schemes=("KP07_dimsplit",)).serve(reqs)
    by = {r.rid: r for r in results}
    assert by[1].status == "rejected" and "budget" in by[1].error and by[1].state is None
    assert done_ids(results) == [0, 2] and stats["rejected"] == 1


def test_unknown_scheme_is_rejected(fake):
    reqs = requests(2, 0.0)
    reqs[1].scheme = "MUSCL"  # no such scheme
    results, _ = Server(None, budget_bytes=1e12, chunk_steps=1, schemes=("KP07_dimsplit",)).serve(reqs)
    by = {r.rid: r for r in results}
    assert by[1].status == "rejected" and "MUSCL" in by[1].error
    assert done_ids(results) == [0]


@pytest.mark.parametrize("spacing", [0.0, 0.01])  # a burst (admission threads) and single arrivals (inline)
def test_malformed_requests_are_rejected_and_the_others_served(fake, spacing):
    reqs = requests(10, spacing)
    reqs[3].variables = reqs[3].variables[:2]  # a missing variable
    reqs[6].variables = [np.zeros((5, 5), dtype=np.float32)] * 3  # wrong shape
    results, stats = Server(None, budget_bytes=1e12, chunk_steps=1, schemes=("KP07_dimsplit",)).serve(reqs)
    by = {r.rid: r for r in results}
    assert len(results) == 10
    assert by[3].status == "rejected" and "3 conserved variables" in by[3].error
    assert by[6].status == "rejected" and "shape" in by[6].error
    assert done_ids(results) == [0, 1, 2, 4, 5, 7, 8, 9]
    for r in results:
        if r.status == "done":
            assert r.state[0][0, 0] == r.rid and r.steps == 3 + r.rid % 5
    assert stats["requests"] == 8 and stats["rejected"] == 2


def test_failed_scenario_released_and_the_others_served(fake):
    reqs = requests(12, 0.0)
    FakeBatch.fail_after = {4: 2, 9: 1}
    srv = Server(None, budget_bytes=1e12, chunk_steps=1, schemes=("KP07_dimsplit",))
    results, stats = srv.serve(reqs)
    by = {r.rid: r for r in results}
    assert by[4].status == "failed" and by[4].steps == 2 and by[4].state is None
    assert by[9].status == "failed" and by[9].steps == 1
    assert done_ids(results) == [i for i in range(12) if i not in (4, 9)]
    assert stats["failed"] == 2 and srv.used == 0.0
    assert all(not b.slots for b in fake.instances)  # every slot released


def test_lazy_initial_states_and_result_reduction(fake):
    """Initial states made at admission by a callable; results reduced on the return threads."""
    reqs = requests(8, 0.0)
    made = []
    for r in reqs:
        arrays = r.variables

        def make(arrays=arrays, rid=r.rid):
            made.append(rid)
            return arrays
        r.variables = make
    results, _ = Server(None, budget_bytes=1e12, chunk_steps=2, schemes=("KP07_dimsplit",)).serve(
        reqs, result_fn=lambda req, state: float(state[0].sum()))
    assert sorted(made) == list(range(8))
    assert done_ids(results) == list(range(8))
    assert all(r.state == 4.0 * r.rid for r in results)


@pytest.mark.parametrize("n,spacing", [(1, 0.0), (12, 0.0)])
def test_gpu_full_with_nothing_resident_is_rejected(fake, monkeypatch, n, spacing):
    """A MemoryError while no other scenario holds device memory rejects the
    request instead of retrying for ever: inline admission (one request) and
    through the admission threads (a burst that all fails)."""

    def add(self, *a, **kw):
        raise MemoryError("full")

    monkeypatch.setattr(FakeBatch, "add", add)
    srv = Server(None, budget_bytes=1e12, chunk_steps=1, schemes=("KP07_dimsplit",))
    results, stats = srv.serve(requests(n, spacing))
    assert len(results) == n and all(r.status == "rejected" and "does not fit" in r.error for r in results)
    assert srv.used == 0.0


def test_running_scenarios_capped(fake, monkeypatch):
    """Past max_running the arrivals wait to be admitted; all are served."""
    reqs = requests(40, 0.0)
    srv = Server(None, budget_bytes=1e12, chunk_steps=1, schemes=("KP07_dimsplit",), max_running=5)
    peak = {"n": 0}
    orig_run = FakeBatch.run

    def run(self, n):
        peak["n"] = max(peak["n"], len(self.slots))
        orig_run(self, n)

    monkeypatch.setattr(FakeBatch, "run", run)
    results, stats = srv.serve(reqs)
    assert done_ids(results) == list(range(40)) and stats["requests"] == 40
    assert peak["n"] <= 5
