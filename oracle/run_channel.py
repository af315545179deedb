"""Run the oracle channel step for one configuration and save field snapshots.

TEST INFRASTRUCTURE ONLY: the GPU tests and bench.py's CPU-baseline leg run
this as a subprocess, so that the reference's own PPE (oracle/_ref, one global
instance per process, main.f90:80) is initialised once per run whatever else
the calling process has done.

    python -m oracle.run_channel --grid 512 384 256 --stretch 2.0 --re-tau 1000 \\
        --seed 11 --noise 0.1 --snap 10 100 --out DIR

The step is main.f90:137-208: the restated Fortran stencils (oracle_stencil.c)
around the PPE.  --ppe ref (default, Thomas only) uses the reference's own C
execute_poisson_solver compiled unmodified; --ppe port uses the restated PPE
(oracle_ppe.c, bit-identical to the reference build on the golden vectors),
which also runs PDD (--nparts P).  Both use all OpenMP threads of the host.

Output: DIR/{u,v,w,p}_{n}.npy for every snapshot step n (interior points,
shape (nz, ny, nx), float64) and DIR/meta.json with the wall-clock seconds of
every step.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def main(argv=None) -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", type=int, nargs=3, required=True)
    ap.add_argument("--stretch", type=float, default=1.5)
    ap.add_argument("--re-tau", type=float, default=180.0)
    ap.add_argument("--dt", type=float, default=1e-4)
    ap.add_argument("--u-crf", type=float, default=0.0)
    ap.add_argument("--seed", type=int, default=42)
    ap.add_argument("--noise", type=float, default=0.1)
    ap.add_argument("--nparts", type=int, default=0)
    ap.add_argument("--ppe", choices=["ref", "port"], default="ref")
    ap.add_argument("--snap", type=int, nargs="+", required=True, help="steps after which to save the fields")
    ap.add_argument("--out", required=True)
    a = ap.parse_args(argv)

    import numpy as np
    from oracle import oracle as O
    nx, ny, nz = a.grid
    g = O.Grid(nx, ny, nz, stretch=a.stretch, re_tau=a.re_tau, dt=a.dt, u_crf=a.u_crf)
    u, v, w, p = g.init_flow(a.seed, a.noise)
    u1, v1, w1 = g.zeros(), g.zeros(), g.zeros()
    use_ref = a.ppe == "ref" and a.nparts == 0 and O.ref_available()
    if use_ref:
        ppe = O.RefPPE(nx, ny, nz, g.g.dx, g.g.dy, g.dzf_global)
        what = "reference C PPE (src/src_c built unmodified) + C restatement of the Fortran stencils"
    else:
        ppe = O.PPE(nx, ny, nz, g.g.dx, g.g.dy, g.dzf_global, nparts=a.nparts)
        what = "C restatement of the PPE" + (f" (PDD, {a.nparts} partitions)" if a.nparts else "") + \
               " and of the Fortran stencils"
    os.makedirs(a.out, exist_ok=True)
    snaps = sorted(set(a.snap))
    times = []
    for n in range(1, snaps[-1] + 1):
        t0 = time.perf_counter()
        g.step(ppe, u, v, w, u1, v1, w1, p)
        times.append(time.perf_counter() - t0)
        if n in snaps:
            for name, f in (("u", u), ("v", v), ("w", w), ("p", p)):
                np.save(os.path.join(a.out, f"{name}_{n}.npy"), f[1:-1, 1:-1, 1:-1])
    if hasattr(ppe, "close"):
        ppe.close()
    threads = int(os.environ.get("OMP_NUM_THREADS", "0")) or len(os.sched_getaffinity(0))
    json.dump({"grid": [nx, ny, nz], "what": what, "step_seconds": times, "threads": threads,
               "snapshots": snaps}, open(os.path.join(a.out, "meta.json"), "w"))


def run(out_dir: str, grid, snaps, *, stretch=1.5, re_tau=180.0, dt=1e-4, u_crf=0.0, seed=42, noise=0.1,
        nparts=0, ppe="ref", timeout=3600.0) -> dict:
    """Run main() in a fresh process; returns the meta.json contents."""
    import subprocess
    cmd = [sys.executable, "-m", "oracle.run_channel", "--grid", *map(str, grid), "--stretch", repr(stretch),
           "--re-tau", repr(re_tau), "--dt", repr(dt), "--u-crf", repr(u_crf), "--seed", str(seed),
           "--noise", repr(noise), "--nparts", str(nparts), "--ppe", ppe, "--snap", *map(str, snaps),
           "--out", out_dir]
    env = dict(os.environ)
    env.setdefault("OMP_NUM_THREADS", str(len(os.sched_getaffinity(0))))
    subprocess.run(cmd, cwd=ROOT, env=env, check=True, timeout=timeout)
    return json.load(open(os.path.join(out_dir, "meta.json")))


def load(out_dir: str, step: int):
    """(u, v, w, p) interior arrays of a snapshot, memory-mapped."""
    import numpy as np
    return tuple(np.load(os.path.join(out_dir, f"{n}_{step}.npy"), mmap_mode="r") for n in "uvwp")


if __name__ == "__main__":
    main()
