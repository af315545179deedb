"""Run a few RK2 projection steps of one precision, for profilers.

    python -m powerllel_channel_b200.prof_step --grid 512 384 128 --precision mixed --steps 2

The command ncu wraps when it captures the step's kernels: it creates one
channel, fills it with the seeded Poiseuille + noise field and runs
``--warmup`` then ``--steps`` steps, printing the per-kernel times of the
library's own event profile (``pl_channel_profile``) at the end.
"""
from __future__ import annotations

import argparse
import json

import powerllel_channel_b200 as plb


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", type=int, nargs=3, default=(512, 384, 128))
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--trid-parts", type=int, default=0)
    ap.add_argument("--no-profile", action="store_true", help="skip the event profile at the end")
    a = ap.parse_args()
    nx, ny, nz = a.grid
    prec = plb.PL_MIXED if a.precision == "mixed" else plb.PL_FP64
    cfg = plb.ChannelConfig(nx=nx, ny=ny, nz=nz, stretch_ratio=2.0, re_tau=1000.0, dt=1e-4, precision=prec,
                            trid_parts=a.trid_parts)
    ch = plb.Channel(cfg)
    ch.init_flow(11, 0.1)
    ch.step(a.warmup + a.steps)
    ch.synchronize()
    out = {"grid": [nx, ny, nz], "precision": a.precision, "diag": ch.diagnostics()}
    if not a.no_profile:
        out["kernels_ms"] = {k: round(t, 4) for k, t in ch.profile(1)}
    print(json.dumps(out))
    ch.close()


if __name__ == "__main__":
    main()
