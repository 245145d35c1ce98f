"""The server's scheduling logic on the CPU, with a stand-in for the GPU batch:
every request is served exactly once with its own result, the device-memory
budget is never exceeded, bursts go through the admission threads and single
arrivals are admitted inline, an admission that finds the GPU full is
retried once memory has been released, and requests that can never fit end
serve() with an error instead of waiting for ever."""

import threading

import numpy as np
import pytest

import finitevolumegpu_b200.server as server
from finitevolumegpu_b200.server import Request, Server, state_bytes


class FakeBatch(object):
    """Advances each admitted scenario by dt = 1 per step up to its t_end."""

    instances = []
    full_once = set()  # rids whose first admission reports a full GPU

    def __init__(self, context, scheme, g=9.81, gamma=1.4, cfl_scale=0.9, max_instances=4096, **kw):
        self.scheme = scheme
        self.lock = threading.Lock()
        self.slots = {}
        self.next = 0
        self.add_threads = set()
        FakeBatch.instances.append(self)

    def add(self, variables, nx, ny, dx, dy, t_end, boundary_conditions=None):
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
                    if st["t"] < st["t_end"]:
                        st["t"] += 1.0
                        st["nt"] += 1

    def sync(self):
        pass

    def status(self, slot):
        with self.lock:
            st = self.slots[slot]
            return {"t": st["t"], "nt": st["nt"], "dt": 1.0, "done": st["t"] >= st["t_end"]}

    def download(self, slot):
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


def test_request_larger_than_the_budget_is_refused(fake):
    reqs = requests(3, 0.0)
    budget = 0.5 * state_bytes("KP07_dimsplit", 64, 64)
    with pytest.raises(ValueError, match="request 0"):
        Server(None, budget_bytes=budget, chunk_steps=1, schemes=("KP07_dimsplit",)).serve(reqs)


def test_unknown_scheme_is_refused(fake):
    reqs = requests(2, 0.0)
    reqs[1].scheme = "LxF"  # unsplit: no batched kernels
    with pytest.raises(ValueError, match="request 1"):
        Server(None, budget_bytes=1e12, chunk_steps=1, schemes=("KP07_dimsplit",)).serve(reqs)


@pytest.mark.parametrize("n,spacing", [(1, 0.0), (12, 0.0)])
def test_gpu_full_with_nothing_resident_raises(fake, monkeypatch, n, spacing):
    """A MemoryError while no other scenario holds device memory ends serve()
    instead of retrying for ever: inline admission (one request) and through
    the admission threads (a burst that all fails)."""

    def add(self, *a, **kw):
        raise MemoryError("full")

    monkeypatch.setattr(FakeBatch, "add", add)
    srv = Server(None, budget_bytes=1e12, chunk_steps=1, schemes=("KP07_dimsplit",))
    with pytest.raises(MemoryError):
        srv.serve(requests(n, spacing))
