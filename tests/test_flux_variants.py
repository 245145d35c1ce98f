"""The oracle's flux and limiter functions against golden vectors of the
reference's own (tests/golden/make_flux_golden.py: GPUSimulators/cuda/
SWECommon.h HLL_flux, HLLC_flux and GodC_1D_flux, and every limiter of
GPUSimulators/cuda/limiters.h, compiled unmodified with the reference's
fast-math options and evaluated on a B200).

Bounds: fluxes within 2e-6 of each variable's scale (fast-math division and
square root against IEEE FP32); limiters within 4 ulp or 2**-22.  The one deliberate
difference is vanAlbada2: the reference's expression ``2r / (r*r* + 1)``
(limiters.h:112-114) parses as 2r / (r*r*(+1)) = 2/r, not van Albada's
2r / (r^2 + 1), and is NaN at r = 0.  The oracle and the kernels use van
Albada's formula; the test pins both readings against the golden values.
"""

import os

import numpy as np
import pytest

from oracle.oracle import flux_eval, limiter_eval

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "flux_ref.npz")
G, DX, DT = 9.81, 0.5, 0.02


@pytest.fixture(scope="module")
def golden():
    with np.load(GOLDEN) as f:
        return {k: f[k] for k in f.files}


@pytest.mark.parametrize("kind,key", [(0, "hll"), (1, "hllc"), (2, "godc")])
def test_fluxes_match_reference(golden, kind, key):
    out = flux_eval(kind, golden["ql"], golden["qr"], G, DX, DT)
    ref = golden[key]
    assert np.all(np.isfinite(ref))
    scale = np.abs(ref).max(axis=0)
    assert np.max(np.abs(out - ref) / scale) < 2e-6


def test_flux_kinds_differ(golden):
    """The three goldens are three different fluxes (a harness that evaluated one
    function three times would pass the test above)."""
    assert np.abs(golden["hll"] - golden["hllc"]).max() > 1.0
    assert np.abs(golden["hll"] - golden["godc"]).max() > 1.0


@pytest.mark.parametrize("lim", [0, 1, 2, 3, 4, 6, 7, 8])
def test_limiters_match_reference(golden, lim):
    r = golden["r"]
    beta = float(golden["beta_%d" % lim])
    out = limiter_eval(lim, r, beta)
    ref = golden["limiter_%d" % lim]
    ulp = np.spacing(np.maximum(np.abs(ref), np.float32(1e-30)).astype(np.float32))
    # 2**-22 absolute covers vanAlbada1's cancellation in r*r + r near r = -1,
    # which the reference's fast-math build contracts into one fused multiply-add
    assert np.all(np.abs(out - ref) <= np.maximum(4 * ulp, 2.0 ** -22))


def test_van_albada2_reading(golden):
    r = golden["r"]
    ref = golden["limiter_5"]
    zero = r == 0
    assert np.all(np.isnan(ref[zero]))
    nz = ~zero
    two_over_r = (np.float32(2) / r[nz]).astype(np.float32)
    assert np.allclose(ref[nz], two_over_r, rtol=4e-7, atol=0)
    ours = limiter_eval(5, r)
    want = (2.0 * r.astype(np.float64) / (r.astype(np.float64) ** 2 + 1.0)).astype(np.float32)
    assert np.allclose(ours, want, rtol=4e-7, atol=1e-30)
