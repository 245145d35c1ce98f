"""Golden vectors of the reference's unused flux and limiter functions.

Runs HLL_flux, HLLC_flux and GodC_1D_flux (GPUSimulators/cuda/SWECommon.h) and
the limiters of GPUSimulators/cuda/limiters.h, compiled unmodified from the
reference tree into oracle/_ref/libref_flux.so (``make -C oracle ref``), on
seeded inputs on the GPU, and writes the inputs and outputs to the file named
by the first argument (tests/golden/flux_ref.npz is the committed copy).
"""

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "..", "..", "oracle", "_ref", "libref_flux.so")


def face_pairs(rng, n):
    """Subsonic and supersonic, wet face pairs of (h, hu, hv)."""
    hl = rng.uniform(0.05, 3.0, n)
    hr = rng.uniform(0.05, 3.0, n)
    ul = rng.uniform(-6.0, 6.0, n)
    ur = rng.uniform(-6.0, 6.0, n)
    vl = rng.uniform(-1.0, 1.0, n)
    vr = rng.uniform(-1.0, 1.0, n)
    ql = np.stack([hl, hl * ul, hl * vl], axis=1).astype(np.float32)
    qr = np.stack([hr, hr * ur, hr * vr], axis=1).astype(np.float32)
    return ql, qr


def main(dst):
    L = ctypes.CDLL(LIB)
    P = ctypes.POINTER(ctypes.c_float)
    L.ref_flux_eval.argtypes = [ctypes.c_int, ctypes.c_int, P, P, ctypes.c_float, ctypes.c_float, ctypes.c_float, P]
    L.ref_limiter_eval.argtypes = [ctypes.c_int, ctypes.c_int, P, ctypes.c_float, P]
    rng = np.random.default_rng(2024)
    out = {}
    ql, qr = face_pairs(rng, 4096)
    out["ql"], out["qr"] = ql, qr
    for kind, name in enumerate(("hll", "hllc", "godc")):
        f = np.empty_like(ql)
        assert L.ref_flux_eval(kind, ql.shape[0], ql.ctypes.data_as(P), qr.ctypes.data_as(P), 9.81, 0.5, 0.02,
                               f.ctypes.data_as(P)) == 0
        out[name] = f
    r = np.concatenate([rng.uniform(-3.0, 5.0, 4000), [0.0, 1.0, -1.0, 2.0, 0.5, 1e-3]]).astype(np.float32)
    out["r"] = r
    for lid, beta in ((0, 1.9), (1, 0.0), (2, 0.0), (3, 0.0), (4, 0.0), (5, 0.0), (6, 0.0), (7, 1.5), (8, 1.5)):
        y = np.empty_like(r)
        assert L.ref_limiter_eval(lid, r.size, r.ctypes.data_as(P), beta, y.ctypes.data_as(P)) == 0
        out["limiter_%d" % lid] = y
        out["beta_%d" % lid] = np.float32(beta)
    np.savez_compressed(dst, **out)
    print("wrote", dst)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "flux_ref.npz"))
