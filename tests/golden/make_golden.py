"""Generate the golden fixtures of tests/golden/ from the reference itself.

Run in a container that holds the reference tree (the GPU box does not):

    PL_REFERENCE=<reference checkout> make -C oracle   # builds oracle/_ref/ from its own C sources
    python tests/golden/make_golden.py

PPE fixtures (ppe_*.npz): the reference's execute_poisson_solver
(src/src_c/mod_poisson_solver.c:468-605) compiled unmodified (oracle/_ref,
Thomas build or -D_PDD build run on p_col forked ranks) applied to a seeded
N(0,1) right-hand side from which the dzf-weighted mean was removed (the
solvability condition of the Neumann problem).

Step fixture (step_*.npz): the reference PPE inside the C restatement of the
Fortran step (oracle/oracle_stencil.c, main.f90:137-208), from the repository's
seeded initial field; the Fortran stencils cannot be compiled here (no Fortran
compiler), so this fixture pins the step only as far as the PPE is concerned.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

PPE_CASES = [
    # name, nx, ny, nz, stretch, p_col, pdd
    ("ppe_thomas_16x12x8", 16, 12, 8, 1.5, 1, False),
    ("ppe_thomas_32x24x16", 32, 24, 16, 1.8, 1, False),
    ("ppe_thomas_48x36x20", 48, 36, 20, 2.0, 1, False),
    ("ppe_pdd1_32x24x16", 32, 24, 16, 1.8, 1, True),
    ("ppe_pdd2_32x24x32", 32, 24, 32, 1.8, 2, True),
    ("ppe_pdd4_32x24x32", 32, 24, 32, 1.8, 4, True),
    ("ppe_pdd4_32x24x30", 32, 24, 30, 1.8, 4, True),
    ("ppe_pdd8_16x12x64", 16, 12, 64, 2.0, 8, True),
]


def solvable_rhs(nx, ny, nz, dzf, seed):
    rng = np.random.default_rng(seed)
    r = rng.standard_normal((nz, ny, nx))
    wgt = dzf[1:-1]
    r -= (r.mean(axis=(1, 2)) * wgt).sum() / wgt.sum()
    var = np.zeros((nz + 2, ny + 2, nx + 2))
    var[1:-1, 1:-1, 1:-1] = r
    return var


def make_ppe():
    for idx, (name, nx, ny, nz, s, p_col, pdd) in enumerate(PPE_CASES):
        g = O.Grid(nx, ny, nz, stretch=s)
        dzf = g.dzf_global
        var = solvable_rhs(nx, ny, nz, dzf, 1000 + idx)
        out, _ = O.ref_ppe_run(var, nx, ny, nz, g.g.dx, g.g.dy, dzf, p_row=1, p_col=p_col, pdd=pdd)
        np.savez_compressed(os.path.join(OUT, name + ".npz"), nx=nx, ny=ny, nz=nz, stretch=s, p_col=p_col,
                            pdd=int(pdd), dx=g.g.dx, dy=g.g.dy, dzf=dzf, rhs=var[1:-1, 1:-1, 1:-1],
                            p=out[1:-1, 1:-1, 1:-1])
        print(name, "mean(p)", out[1:-1, 1:-1, 1:-1].mean())


def make_step():
    nx, ny, nz, nsteps = 32, 24, 16, 5
    g = O.Grid(nx, ny, nz, stretch=1.5, re_tau=180.0, dt=1e-4)
    u, v, w, p = g.init_flow(42, 0.1)
    u0, v0, w0 = u.copy(), v.copy(), w.copy()
    ref = O.RefPPE(nx, ny, nz, g.g.dx, g.g.dy, g.dzf_global)
    u1, v1, w1 = g.zeros(), g.zeros(), g.zeros()
    for _ in range(nsteps):
        g.step(ref, u, v, w, u1, v1, w1, p)
    ref.close()
    div, ijk = g.max_div(u, v, w)
    np.savez_compressed(os.path.join(OUT, "step_32x24x16_5.npz"), nx=nx, ny=ny, nz=nz, nsteps=nsteps, seed=42,
                        noise=0.1, stretch=1.5, re=g.g.re, dt=1e-4, u0=u0, v0=v0, w0=w0, u=u, v=v, w=w, p=p,
                        div=div)
    print("step fixture div", div)


if __name__ == "__main__":
    if not O.ref_available():
        sys.exit("oracle/_ref is not built (make -C oracle with the reference tree present)")
    make_ppe()
    make_step()
