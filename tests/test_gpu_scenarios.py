"""The reference's Euler test cases (shock-bubble, Kelvin-Helmholtz,
Rayleigh-Taylor with gravity) as served requests: mixed in one server run,
each result equals a plain EE2D_KP07_dimsplit(context, **arguments) run of
the same case bit for bit."""

import numpy as np
import pytest

import finitevolumegpu_b200 as fv
from finitevolumegpu_b200 import InitialConditions as IC
from finitevolumegpu_b200.server import Server

pytestmark = pytest.mark.gpu


def test_reference_scenarios_served_equal_plain(ctx):
    np.random.seed(5)
    cases = [
        (IC.genShockBubble(96, 24, 1.4), 0.04),
        (IC.genKelvinHelmholtz(64, 48, 1.4), 0.05),
        (IC.genRayleighTaylor(24, 72, 1.4, version=0), 0.3),
        (IC.genRayleighTaylor(16, 48, 1.4, version=1), 0.3),
        (IC.genShockBubble(64, 16, 1.4), 0.03),
    ]
    reqs = [IC.request_from_arguments(i, d, t_end, arrival=0.002 * i) for i, (d, t_end) in enumerate(cases)]
    results, stats = Server(ctx, budget_bytes=2e9, chunk_steps=4, max_instances=16).serve(reqs)
    assert stats["requests"] == len(cases)
    by_id = {r.rid: r for r in results}
    for i, (d, t_end) in enumerate(cases):
        sim = fv.EE2D_KP07_dimsplit.EE2D_KP07_dimsplit(ctx, **d)
        sim.simulate(t_end)
        res = by_id[i]
        assert res.steps == sim.simSteps() and res.t == sim.simTime()
        for a, w in zip(res.state, sim.download()):
            assert np.array_equal(a, w), (i, float(np.max(np.abs(a - w))))
