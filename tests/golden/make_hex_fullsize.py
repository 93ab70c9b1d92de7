"""Generate the full-size FP64 seismogram fixture of the 3-D elastic hex
workload: 64^3 hexahedra of 200 m (12.8 km cube), order 4, vp 6000 / vs 3464
/ rho 2700 with a 5 % Gaussian random-field perturbation (seed 1), a
moment-tensor Ricker source (f0 1.5 Hz), 64 receivers on the top surface,
4000 steps at dt = 0.4 * 2 / sqrt(lambda_max(M^-1 K)).

The seismograms come from the FP64 CPU oracle (oracle/oracle.c, corrected
mode with cached geometry: the restatement of Problem::assembleIntoGlobalDof
/ Order2Newmark of the reference, src/cxx/Problem/Problem.cpp:143-214 and
src/cxx/Problem/Order2Newmark.cpp:68-114) on exactly the inputs that
salvus_b200.configs.elastic_hex(nel=64, order=4) builds, so the GPU test can
rebuild the same inputs and compare.  About 2.5-3 h on 6 host threads.

    python tests/golden/make_hex_fullsize.py [--threads 6] [--steps 4000]

Writes tests/golden/hex_elastic_64cube_4000steps.npz with
  seis  [64][3][steps] FP64 receiver displacements after each step
  dt, steps, nel, order, lambda_max, eig_iterations, eig_seed
"""
import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import pyoracle as po  # noqa: E402
from salvus_b200 import configs  # noqa: E402

OUT = os.path.join(HERE, "hex_elastic_64cube_4000steps.npz")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=6)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--nel", type=int, default=64)
    ap.add_argument("--chunk", type=int, default=200)
    ap.add_argument("--eig-iterations", type=int, default=60)
    ap.add_argument("--out", default=OUT)
    a = ap.parse_args()
    t0 = time.time()
    cfg = configs.elastic_hex(nel=a.nel, order=4)
    o = po.Problem(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                   configs.oracle_params(cfg), threads=a.threads)
    print(f"oracle built: G={o.G} ({time.time() - t0:.0f} s)", flush=True)
    lam = o.max_eigenvalue(a.eig_iterations, 1)
    dt = 0.4 * 2.0 / np.sqrt(lam)
    print(f"lambda_max={lam:.9e} dt={dt:.9e} ({time.time() - t0:.0f} s)", flush=True)
    s = cfg["sources"][0]
    o.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                 s["moment_tensor"], kind=1)
    for r in cfg["receivers"]:
        o.add_receiver(r)
    parts = []
    done = 0
    while done < a.steps:
        k = min(a.chunk, a.steps - done)
        parts.append(o.run(k, dt))
        done += k
        print(f"{done}/{a.steps} steps ({time.time() - t0:.0f} s)", flush=True)
    seis = np.concatenate(parts, axis=2)
    np.savez_compressed(a.out, seis=seis, dt=dt, steps=a.steps, nel=a.nel, order=4,
                        lambda_max=lam, eig_iterations=a.eig_iterations, eig_seed=1)
    print(f"wrote {a.out} ({os.path.getsize(a.out)} bytes, {time.time() - t0:.0f} s)", flush=True)


if __name__ == "__main__":
    main()
