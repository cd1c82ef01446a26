"""Generate the configuration-1 golden fixture with the CPU oracle.

The 3-D MHD lid-driven cavity at its stated size: uniform 32^3 cells,
Re = 400, Ha = 10, uniform B0 along y, the low-Rem electric-potential form
with insulating walls, dt = 1e-3, pressure and potential PCG to 1e-10
relative residual, U0 = N(0, 1e-6) (numpy default_rng(0)).  The oracle
steps it 1000 times and the script stores

* ``ldc32_step20.json`` -- after 20 steps: the SHA-256 of the float64
  bytes of U (3 components), p and phi, their L2 norms and the solver
  iteration totals (the CPU test re-runs these 20 steps and must reproduce
  them bit for bit, which pins the fixture to the oracle);
* ``ldc32_step1000.npz`` -- after 1000 steps: U (3 components), p, phi,
  J (3 components), the oracle's div U / div B probes and iteration totals.

Run from the repository root:  python -m tests.golden.make_ldc32
(about 15 minutes on 8 host threads).
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from moons_b200 import capi as G  # noqa: E402
from moons_b200 import configs  # noqa: E402

N = 32
SEED = 0
STEPS = 1000
CHECK = 20
FIELDS_SHORT = [("U0", G.MHD_U, 0), ("U1", G.MHD_U, 1), ("U2", G.MHD_U, 2), ("p", G.MHD_P, 0), ("phi", G.MHD_PHI, 0)]
FIELDS_LONG = FIELDS_SHORT + [("J0", G.MHD_J, 0), ("J1", G.MHD_J, 1), ("J2", G.MHD_J, 2)]


def build_case(backend):
    return configs.make(backend, configs.ldc, seed=SEED, n=N)


def digest(sim) -> dict:
    out = {}
    for name, which, c in FIELDS_SHORT:
        a = np.ascontiguousarray(sim.download(which, c), dtype=np.float64)
        out[name] = {"sha256": hashlib.sha256(a.tobytes(order="F")).hexdigest(),
                     "l2": float(np.linalg.norm(a))}
    return out


def main():
    import oracle.oracle as O
    sim = build_case(O)
    t0 = time.time()
    tot = {}

    def add(info):
        for k in ("iters_U", "iters_p", "iters_phi"):
            tot[k] = tot.get(k, 0) + int(info[k])

    add(sim.step(CHECK))
    short = {"steps": CHECK, "iters": dict(tot), "fields": digest(sim)}
    with open(os.path.join(HERE, "ldc32_step20.json"), "w") as f:
        json.dump(short, f, indent=1)
    done = CHECK
    while done < STEPS:
        k = min(100, STEPS - done)
        add(sim.step(k))
        done += k
        print(f"{done} steps, {time.time() - t0:.0f} s", flush=True)
    du, db = sim.divergence()
    arrays = {name: sim.download(which, c) for name, which, c in FIELDS_LONG}
    np.savez_compressed(os.path.join(HERE, "ldc32_step1000.npz"), steps=STEPS, div_u=du, div_b=db,
                        iters_U=tot["iters_U"], iters_p=tot["iters_p"], iters_phi=tot["iters_phi"], **arrays)
    print("done", tot, du, db, f"{time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()
