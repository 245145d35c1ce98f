"""Extent downloads and uploads of u0 (CudaArray2D.download/upload with
extent, GPUSimulators/Common.py:543-616): a region of the array that includes
the ghost cells, in the reference's coordinates."""

import numpy as np
import pytest

from conftest import bump

import finitevolumegpu_b200 as fv

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scheme,gc", [("KP07_dimsplit", 2), ("HLL", 1)])
def test_extent_download_matches_interior_and_ghosts(ctx, scheme, gc):
    nx, ny = 37, 23
    h, hu, hv = bump(nx, ny)
    # upload with ghost cells, so their values are known
    full = [np.pad(a, gc, mode="constant", constant_values=c) for a, c in ((h, 7.0), (hu, 8.0), (hv, 9.0))]
    sim = fv.SCHEMES[scheme](ctx, *full, nx, ny, 1.0, 1.0, 9.81)
    for v in range(3):
        whole = sim.u0[v].download(extent=[0, 0, nx + 2 * gc, ny + 2 * gc])
        assert np.array_equal(whole, full[v])
        part = sim.u0[v].download(extent=[gc + 3, gc + 2, 11, 5])
        assert np.array_equal(part, full[v][gc + 2:gc + 7, gc + 3:gc + 14])
        assert np.array_equal(sim.u0[v].download(), full[v][gc:-gc, gc:-gc])


def test_extent_upload_then_download(ctx):
    nx, ny = 40, 30
    q = list(bump(nx, ny))
    sim = fv.KP07_dimsplit.KP07_dimsplit(ctx, *q, nx, ny, 1.0, 1.0, 9.81)
    patch = np.arange(6 * 9, dtype=np.float32).reshape(6, 9)
    sim.u0[1].upload(None, patch, extent=[0, 4, 9, 6])  # touches the west ghost columns
    got = sim.u0[1].download(extent=[0, 4, 9, 6])
    assert np.array_equal(got, patch)
    interior = sim.u0[1].download()
    assert np.array_equal(interior[2:8, 0:7], patch[:, 2:])


def test_extent_outside_rejected(ctx):
    nx, ny = 16, 16
    sim = fv.KP07_dimsplit.KP07_dimsplit(ctx, *bump(nx, ny), nx, ny, 1.0, 1.0, 9.81)
    with pytest.raises(AssertionError):
        sim.u0[0].download(extent=[0, 0, nx + 5, 4])
    with pytest.raises(AssertionError):
        sim.u0[0].download(extent=[-1, 0, 4, 4])
