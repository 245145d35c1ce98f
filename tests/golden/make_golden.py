"""Generate golden vectors from the reference's own CUDA kernels.

Runs on a machine with a B200 and the prebuilt oracle/_ref libraries (the
reference's kernel sources compiled unmodified for sm_100a with the compat
header, see oracle/Makefile).  For every scheme it records seeded small
initial states and the state after a fixed number of steps of the
reference's host semantics (oracle.ref_kernels.RefKernelSim), into
tests/golden/ref_<scheme>_<case>.npz.  The CPU tests check the oracle against
these files; the GPU tests check libfvgpu against the oracle and the
reference kernels directly.

    python tests/golden/make_golden.py [outdir]
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref_kernels  # noqa: E402

SWE = ["LxF", "FORCE", "HLL", "HLL2", "WAF", "KP07", "KP07_dimsplit"]


def bump(nx, ny, seed):
    rng = np.random.default_rng(seed)
    amp = rng.uniform(0.1, 0.5)
    cx, cy = rng.uniform(0.3, 0.7) * nx, rng.uniform(0.3, 0.7) * ny
    y, x = np.mgrid[0:ny, 0:nx] + 0.5
    h = 1.0 + amp * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * 6.0 ** 2))
    hu = 0.02 * np.sin(2 * np.pi * y / ny)
    hv = -0.01 * np.cos(2 * np.pi * x / nx)
    return [a.astype(np.float32) for a in (h, hu, hv)]


def dam(nx, ny, seed):
    rng = np.random.default_rng(seed)
    R = rng.uniform(0.1, 0.3) * nx
    y, x = np.mgrid[0:ny, 0:nx] + 0.5
    h = np.where(np.hypot(x - nx / 2, y - ny / 2) < R, 1.0, 0.1)
    z = np.zeros_like(h)
    return [a.astype(np.float32) for a in (h, z, z)]


def kh(nx, ny, seed, gamma=1.4):
    rng = np.random.default_rng(seed)
    phi = rng.uniform(0, 2 * np.pi)
    y = (np.arange(ny) + 0.5) / ny
    x = (np.arange(nx) + 0.5) / nx
    X, Y = np.meshgrid(x, y)
    band = (Y >= 0.25) & (Y < 0.75)
    rho = np.where(band, 2.0, 1.0)
    u = np.where(band, 0.5, -0.5)
    v = 0.01 * np.sin(4 * np.pi * X + phi)
    E = 2.5 / (gamma - 1.0) + 0.5 * rho * (u ** 2 + v ** 2)
    return [a.astype(np.float32) for a in (rho, rho * u, rho * v, E)]


CASES = []
for s in SWE:
    CASES.append(dict(scheme=s, case="bump_reflective", init="bump", nx=48, ny=36, bc=0x03030303, t=3.0,
                      cfl_scale=0.45, g=9.81, dx=1.0, dy=1.0, seed=1))
    CASES.append(dict(scheme=s, case="dam_periodic", init="dam", nx=40, ny=40, bc=0x02020202, t=4.0,
                      cfl_scale=0.9, g=9.81, dx=1.0, dy=1.0, seed=2))
CASES.append(dict(scheme="EE2D_KP07_dimsplit", case="kh_periodic", init="kh", nx=48, ny=32, bc=0x02020202, t=0.05,
                  cfl_scale=0.45, g=0.0, dx=1.0 / 48, dy=1.0 / 32, seed=3))
CASES.append(dict(scheme="EE2D_KP07_dimsplit", case="kh_gravity_mixed", init="kh", nx=32, ny=48, bc=0x02020303,
                  t=0.05, cfl_scale=0.45, g=0.5, dx=1.0 / 32, dy=1.0 / 48, seed=4))


def initial(c):
    f = {"bump": bump, "dam": dam, "kh": kh}[c["init"]]
    return f(c["nx"], c["ny"], c["seed"])


def main(outdir=HERE):
    for c in CASES:
        q = initial(c)
        kw = dict(cfl_scale=c["cfl_scale"], bc=c["bc"])
        if c["scheme"] == "EE2D_KP07_dimsplit":
            kw["gamma"] = 1.4
        sim = ref_kernels.RefKernelSim(c["scheme"], q, c["nx"], c["ny"], c["dx"], c["dy"], c["g"], **kw)
        sim.simulate(c["t"])
        out = sim.download()
        name = os.path.join(outdir, "ref_%s_%s.npz" % (c["scheme"], c["case"]))
        meta = {k: v for k, v in c.items()}
        np.savez_compressed(name, inputs=np.stack(q), outputs=np.stack(out), nt=sim.nt, t=sim.t,
                            meta=np.array(repr(meta)))
        print("%-45s nt=%d t=%.6f" % (os.path.basename(name), sim.nt, sim.t), flush=True)
        sim.close()


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
