"""Serving scenarios with continuous batching.

A request is one scenario: scheme, grid, initial state and t_end.  The server
keeps the state of every admitted scenario resident in HBM inside one Batch
per scheme, advances all of them a few steps at a time (each batch on its own
stream, so the schemes overlap on the GPU), returns each scenario as soon as
it reaches its t_end, and admits waiting requests whenever their arrival time
has passed and the device-memory budget has room.  Requests that arrive
while others run join the running batches at the next chunk boundary.

Each scenario follows the reference's simulate(t_end) semantics on its own
(see batch.py), so its result does not depend on what else is in the batch.
Arrived requests are uploaded by admission threads and finished scenarios
are downloaded and released by return threads, so host-to-device uploads of
new requests, device-to-host reads of results and the queuing of the next
chunk overlap.

Failures stay with their request.  A request that cannot run (an unknown
scheme, a grid larger than the whole budget, the wrong
number or shape of arrays, a GPU with no room even when nothing else is
resident) comes back with status "rejected" and its reason; a scenario whose
state goes bad on the GPU (a non-finite value or a non-positive depth after
a step, or a non-finite time step, e.g. from a corrupted initial state; the
counterpart of the reference's check(), GPUSimulators/Common.py:772-780)
stops there, its slot and memory are released, and it comes back with status
"failed".  The other scenarios run on unchanged.
"""

from __future__ import annotations

import collections
import concurrent.futures
import dataclasses
import queue
import threading
import time
from typing import Dict, List, Optional

import numpy as np

from .batch import Batch
from .Simulator import BoundaryCondition

# Default physical parameters per scheme; a request may set its own g and gamma.
SCHEME_PARAMS = {
    "LxF": dict(g=9.81, gamma=1.4),
    "KP07": dict(g=9.81, gamma=1.4),
    "KP07_dimsplit": dict(g=9.81, gamma=1.4),
    "HLL": dict(g=9.81, gamma=1.4),
    "HLL2": dict(g=9.81, gamma=1.4),
    "WAF": dict(g=9.81, gamma=1.4),
    "FORCE": dict(g=9.81, gamma=1.4),
    "EE2D_KP07_dimsplit": dict(g=0.0, gamma=1.4),
}


@dataclasses.dataclass
class Request:
    rid: int
    scheme: str
    variables: object  # list of host arrays, or a callable returning them (called at admission)
    nx: int
    ny: int
    dx: float
    dy: float
    t_end: float
    arrival: float = 0.0  # seconds after the start of serve()
    boundary_conditions: Optional[BoundaryCondition] = None
    g: Optional[float] = None      # gravity; None: the scheme's default (SCHEME_PARAMS)
    gamma: Optional[float] = None  # ratio of specific heats (Euler); None: the default

    def batch_key(self):
        d = SCHEME_PARAMS[self.scheme]
        return (self.scheme, float(d["g"] if self.g is None else self.g),
                float(d["gamma"] if self.gamma is None else self.gamma))


@dataclasses.dataclass
class Result:
    rid: int
    scheme: str
    state: object  # the downloaded arrays (or what serve()'s result_fn made of them); None unless done
    steps: int
    t: float
    arrival: float
    admitted: Optional[float]
    finished: float
    status: str = "done"  # "done", "failed" (its state went bad on the GPU) or "rejected" (could not run)
    error: Optional[str] = None

    @property
    def latency(self):
        return self.finished - self.arrival


def state_bytes(scheme, nx, ny, tile_w=60, tile_h=28):
    """Device bytes one scenario holds (two state buffers plus tile scratch)."""
    nv = 4 if scheme == "EE2D_KP07_dimsplit" else 3
    pitch = (nx + 8 + 31) // 32 * 32
    tiles = -(-nx // tile_w) * -(-ny // tile_h)
    return 2 * nv * (ny + 4) * pitch * 4 + tiles * 36 + 512


class Server(object):
    def __init__(self, context, budget_bytes=120e9, chunk_steps=8, max_instances=4096, schemes=None,
                 cfl_scale=0.9, return_threads=3, admit_threads=3, max_running=256):
        """max_running: scenarios held at once (on the GPU, being uploaded or
        waiting to be returned).  Past
        the server's capacity the extra arrivals wait to be admitted instead of
        all sharing the GPU: each chunk then stays short, the admitted scenarios
        finish at the device's rate and the host copies do not crowd the cores."""
        self.context = context
        self.max_running = max(1, int(max_running))
        self.return_threads = max(1, int(return_threads))
        self.admit_threads = max(1, int(admit_threads))
        self.budget = float(budget_bytes)
        self.chunk = int(chunk_steps)
        self.cfl_scale = cfl_scale
        self.max_instances = max_instances
        # one batch per (scheme, g, gamma), created when a request first needs it
        self.batches: Dict[tuple, Batch] = {}
        for s in (schemes or ("KP07_dimsplit", "HLL", "EE2D_KP07_dimsplit")):
            self._batch((s, float(SCHEME_PARAMS[s]["g"]), float(SCHEME_PARAMS[s]["gamma"])))
        self.used = 0.0

    def _batch(self, key):
        b = self.batches.get(key)
        if b is None:
            scheme, g, gamma = key
            b = self.batches[key] = Batch(self.context, scheme, g=g, gamma=gamma, cfl_scale=self.cfl_scale,
                                          max_instances=self.max_instances)
        return b

    def serve(self, requests: List[Request], clock=time.perf_counter, result_fn=None):
        """Serve `requests` (arrival times relative to the call) until all are done.

        The calling thread queues the next chunk of steps for every batch with
        running scenarios, hands arrived requests to the admission threads
        while the budget allows (their uploads run on each batch's copy stream
        and they join the first chunk queued after their upload was issued),
        then waits for the chunk and hands the scenarios that reached t_end to
        the return threads.  These download and release them while the
        calling thread queues and admits the next chunk: their state is final
        (later chunks skip them), and their memory returns to the budget once
        released.  Several return threads copy results out in parallel.

        Every request comes back as one Result: "done" with its state
        (``result_fn(request, arrays)`` if given, on a return thread, e.g. to
        keep a checksum instead of the arrays; the arrays it receives live in
        a buffer the thread reuses, so it copies what it keeps), or
        "rejected" / "failed" with the reason (see the module docstring).
        Returns (results, stats); the stats count and time the done requests.
        """
        pending = collections.deque()
        running = {}  # (batch key, slot) -> (request, admitted, bytes): on the GPU, not yet at t_end
        results: List[Result] = []
        lock = threading.Lock()
        returns = queue.Queue()
        shared = {"cells": 0, "outstanding": 0, "error": None}
        timers = collections.Counter()
        t0 = clock()

        def finish(r, status, error, admitted=None, steps=0, t=0.0):
            with lock:
                results.append(Result(r.rid, r.scheme, None, steps, t, r.arrival, admitted, clock() - t0, status,
                                      error))

        for r in sorted(requests, key=lambda r: r.arrival):
            if r.scheme not in SCHEME_PARAMS:
                finish(r, "rejected", "unknown scheme %r" % (r.scheme,))
            elif state_bytes(r.scheme, r.nx, r.ny) > self.budget:
                finish(r, "rejected", "a %d x %d grid needs more device memory than the budget of %.3g bytes"
                       % (r.nx, r.ny, self.budget))
            else:
                pending.append(r)

        def return_finished():
            scratch = np.empty(0, dtype=np.float32)  # this thread's download buffer when result_fn reduces
            while True:
                item = returns.get()
                if item is None:
                    return
                (bk, slot), r, admitted, need = item
                s = bk[0]
                ta = clock()
                try:
                    b = self.batches[bk]
                    st = b.status(slot)
                    if result_fn is not None:
                        n = b.nv * r.nx * r.ny
                        if scratch.size < n:
                            scratch = np.empty(n, dtype=np.float32)
                        state = b.download(slot, scratch)
                    else:
                        state = b.download(slot)
                    b.remove(slot)
                    if result_fn is not None:
                        state = result_fn(r, state)
                except Exception as e:  # reported by serve()
                    with lock:
                        shared["error"] = e
                        shared["outstanding"] -= 1
                    continue
                done = clock() - t0
                with lock:
                    self.used -= need
                    results.append(Result(r.rid, s, state, st["nt"], st["t"], r.arrival, admitted, done))
                    shared["cells"] += r.nx * r.ny * st["nt"]
                    shared["outstanding"] -= 1
                    timers["return"] += clock() - ta

        def admit(b, r):
            """Uploads one request; its slot, or raises (MemoryError: no room now;
            AssertionError / ValueError / TypeError: the request is malformed)."""
            ta = clock()
            variables = r.variables() if callable(r.variables) else r.variables
            slot = b.add(variables, r.nx, r.ny, r.dx, r.dy, r.t_end, r.boundary_conditions)
            with lock:
                timers["admit_upload"] += clock() - ta
            return slot

        malformed = (AssertionError, ValueError, TypeError, IndexError)

        workers = [threading.Thread(target=return_finished, name="fvgpu-return-%d" % k, daemon=True)
                   for k in range(self.return_threads)]
        for w in workers:
            w.start()
        admitting = []  # (future, request, batch key, bytes) of uploads in flight
        busy_since = None
        pool = concurrent.futures.ThreadPoolExecutor(self.admit_threads, thread_name_prefix="fvgpu-admit")
        try:
            while True:
                with lock:
                    outstanding = shared["outstanding"]
                    if shared["error"] is not None:
                        raise shared["error"]
                # 0. admissions whose upload has been issued join the running set
                still = []
                requeue = []
                for fut, r, bk, need in admitting:
                    if not fut.done():
                        still.append((fut, r, bk, need))
                        continue
                    try:
                        slot = fut.result()
                    except MemoryError:  # the GPU is full after all: retry once others have left
                        with lock:
                            self.used -= need
                        requeue.append(r)
                        continue
                    except malformed as e:
                        with lock:
                            self.used -= need
                        finish(r, "rejected", "%s: %s" % (type(e).__name__, e))
                        continue
                    running[(bk, slot)] = (r, clock() - t0, need)
                admitting = still
                if requeue:
                    if not (running or admitting or outstanding):
                        for r in requeue:  # waiting cannot help: nothing else holds device memory
                            finish(r, "rejected", "does not fit on the GPU with no other scenario resident")
                    else:
                        pending.extendleft(sorted(requeue, key=lambda r: r.arrival, reverse=True))
                if not (pending or running or outstanding or admitting):
                    break
                # 1. queue the next chunk
                active = {key[0] for key in running}
                ta = clock()
                for s in active:
                    self.batches[s].run(self.chunk)
                timers["queue"] += clock() - ta
                if active and busy_since is None:
                    busy_since = ta - t0
                # 2. admit arrived requests while the budget allows: a burst of
                #    them goes to the admission threads, whose uploads proceed in
                #    parallel; one or two are admitted here, which keeps them in
                #    the very next chunk
                ta = clock()
                now = ta - t0
                ready = 0
                for r in pending:
                    if r.arrival > now:
                        break
                    ready += 1
                burst = ready > self.admit_threads
                while pending and pending[0].arrival <= now:
                    # on the GPU, being uploaded or waiting to be returned
                    with lock:
                        held = len(running) + len(admitting) + shared["outstanding"]
                    if held >= self.max_running:
                        break
                    r = pending[0]
                    need = state_bytes(r.scheme, r.nx, r.ny)
                    with lock:
                        if self.used + need > self.budget:
                            break
                        self.used += need
                    bk = r.batch_key()
                    if burst:
                        pending.popleft()
                        admitting.append((pool.submit(admit, self._batch(bk), r), r, bk, need))
                        continue
                    try:
                        slot = admit(self._batch(bk), r)
                    except MemoryError:
                        with lock:
                            self.used -= need
                        if not (running or admitting or outstanding):
                            pending.popleft()
                            finish(r, "rejected", "does not fit on the GPU with no other scenario resident")
                            continue
                        break
                    except malformed as e:
                        with lock:
                            self.used -= need
                        pending.popleft()
                        finish(r, "rejected", "%s: %s" % (type(e).__name__, e))
                        continue
                    pending.popleft()
                    running[(bk, slot)] = (r, clock() - t0, need)
                timers["admit"] += clock() - ta
                # 3. wait for the chunk; hand the scenarios at t_end to the return
                #    threads and release the ones that failed
                ta = clock()
                for s in active:
                    self.batches[s].sync()
                for key in [k for k in running if k[0] in active]:
                    st = self.batches[key[0]].status(key[1])
                    if not st["done"]:
                        continue
                    r, admitted, need = running.pop(key)
                    if st["failed"]:
                        self.batches[key[0]].remove(key[1])
                        with lock:
                            self.used -= need
                        finish(r, "failed", "non-finite value or non-positive depth after step %d (t=%g)"
                               % (st["nt"], st["t"]), admitted, st["nt"], st["t"])
                        continue
                    with lock:
                        shared["outstanding"] += 1
                    returns.put((key, r, admitted, need))
                timers["wait"] += clock() - ta
                if not active:
                    # nothing on the GPU: wait for the next arrival, an upload or returns to free memory
                    wait = (pending[0].arrival - (clock() - t0)) if pending else 0.001
                    time.sleep(min(max(wait, 0.0005), 0.005))
        finally:
            pool.shutdown(wait=True)
            for _ in workers:
                returns.put(None)
            for w in workers:
                w.join()
        if shared["error"] is not None:
            raise shared["error"]
        cells = shared["cells"]
        elapsed = clock() - t0
        done = [r for r in results if r.status == "done"]
        lat = np.array([r.latency for r in done]) if done else np.zeros(1)
        stats = {
            "requests": len(done),
            "rejected": sum(r.status == "rejected" for r in results),
            "failed": sum(r.status == "failed" for r in results),
            "elapsed_s": elapsed,
            "cell_updates": cells,
            "cell_updates_per_s": cells / max(elapsed - (busy_since or 0.0), 1e-9),
            "p50_latency_s": float(np.percentile(lat, 50)),
            "p99_latency_s": float(np.percentile(lat, 99)),
            "mean_latency_s": float(lat.mean()),
            "host_seconds": {k: round(v, 4) for k, v in timers.items()},
        }
        return results, stats
