"""Benchmark of the RK2 projection step (PowerLLEL_Channel hot path) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload: 512x384x256 channel (Lx=2pi, Ly=pi, Lz=2; tanh stretching 2.0;
Re_tau=1000 -> re=(Re_tau/0.09)^(1/0.88); dt=1e-4; Thomas), initial field =
Poiseuille + uniform noise 0.1 from seed 11 (seeded synthetic input, no
dataset).  One step = main.f90:137-208 (RK1, RK2, calcRHS, PPE, correctVel,
forceVel with boundary fills).  Each FP64 field is 403 MB > L2 (126 MB), so
no L2 flush is needed between steps.

Arms: --impl b200 (default) times this library; --impl reference times the
reference's own C PPE (src/src_c built unmodified in oracle/_ref) inside the C
restatement of the Fortran stencils on the host cores.

N > 1 (torchrun, one rank per GPU, NCCL): weak scaling over z slabs, as the
reference decomposes with p_row = 1.  Every GPU holds a 512x384x256 slab of
the 512x384x(256 N) channel, the wall-normal systems are solved by PDD with N
partitions (one per GPU) and the planes move between the slabs' phases over
NCCL on each slab's stream (powerllel_channel_b200.slab).  The value is N
slab-steps per step time: steps/s in units of the 512x384x256 workload; the
step time is the slowest rank's.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX, NY, NZ = 512, 384, 256
RE_TAU, STRETCH, SEED, NOISE, DT, PARTS = 1000.0, 2.0, 11, 0.1, 1e-4, 0
METRIC = "RK2 steps/s @512x384x256: mixed vs FP64 on same GPU at rel err<=1e-5"
WORKLOAD = "channel 512x384x256, Re_tau 1000, tanh stretch 2.0, Thomas, dt 1e-4, seed 11, noise 0.1"

# the benchmark configurations (grid, Re_tau, tanh stretch, PDD partitions
# (0 = Thomas), seed, perturbation); C3 is the workload of the headline line
CONFIGS = {
    "C1": ((64, 64, 64), 180.0, 1.5, 0, 42, 0.1),
    "C2": ((256, 192, 128), 550.0, 1.8, 4, 7, 0.05),
    "C3": ((512, 384, 256), 1000.0, 2.0, 0, 11, 0.1),
    "C4": ((1024, 768, 512), 2000.0, 2.0, 8, 11, 0.1),
}


def set_config(name):
    global NX, NY, NZ, RE_TAU, STRETCH, PARTS, SEED, NOISE, METRIC, WORKLOAD
    (NX, NY, NZ), RE_TAU, STRETCH, PARTS, SEED, NOISE = CONFIGS[name]
    grid = f"{NX}x{NY}x{NZ}"
    METRIC = METRIC.replace("512x384x256", grid)
    WORKLOAD = (f"channel {grid}, Re_tau {RE_TAU:g}, tanh stretch {STRETCH:g}, "
                f"{'PDD over %d partitions' % PARTS if PARTS else 'Thomas'}, dt {DT:g}, seed {SEED}, noise {NOISE:g}")

# algorithmic bytes per grid point per launch slot, by kernel and path: the
# compulsory field passes (reads + writes of whole fields at their storage
# width); Mean_h of forceVel is fused into RK2 and the shift into the
# correction, so no separate force pass exists.  Thomas: the right-hand side
# and the solution once each, plus its two FP64 class tables (mult, 1/b),
# each row of which serves four columns: 2 x 8 B / 4 = 4 B per point.
# rhs_xfft: calcRHS fused into the forward x transform (u, v, w read once,
# the transform written once)
ALG_BYTES = {
    "fp64": {"rk_fused": 48, "rk1": 48, "rk2": 72, "calc_rhs": 32, "rhs_xfft": 32, "ppe_xfft_fwd": 16, "ppe_yfft_fwd": 16,
             "ppe_thomas": 20, "ppe_pdd": 24, "ppe_yfft_bwd": 16, "ppe_xfft_bwd": 16, "correct_force": 56},
    "mixed": {"rk_fused": 52, "rk1": 36, "rk2": 64, "calc_rhs": 28, "rhs_xfft": 28, "ppe_xfft_fwd": 8, "ppe_yfft_fwd": 8,
              "ppe_thomas": 12, "ppe_pdd": 16, "ppe_yfft_bwd": 8, "ppe_xfft_bwd": 24, "correct_force": 52},
}
# mixed: rk_fused reads u (FP64) and the FP32 pressure prediction and writes
# u_hat (FP64): 24 + 4 + 24; ppe_xfft_bwd reads the FP32 half-complex line and
# writes the FP32 increment, plus the FP32 pressure update (reads the
# prediction and p_n, writes p_n+1 and the next prediction): 4 + 4 + 16
# kernel launches per step (this library's kernels only), Thomas, and PDD up
# to 32 partitions (one kernel); PDD over more partitions adds the mixed
# path's widening of the FP32 right-hand side into the FP64 sweep buffer
LAUNCHES = {"fp64": 7, "mixed": 8}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_from_profiles(kernel):
    """dram read+write bytes per launch of `kernel` from the committed ncu
    summary (profiles/dram_traffic_512x384x256.txt), else None."""
    p = os.path.join(ROOT, "profiles", "dram_traffic_512x384x256.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        parts = line.split()
        if len(parts) >= 2 and parts[0] == kernel:
            try:
                return float(parts[1])
            except ValueError:
                return None
    return None


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during the timed
    region: read through NVML every 5 ms between begin() and end(), which
    _timed calls around the timed steps alone; without NVML, nvidia-smi
    (`-lms 200`, the whole span from start() to stop()).  Reads only."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits (nvml.h nvmlClocksEventReason*)
    REASON_BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
                   "hw_thermal_slowdown": 0x40}

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.nvml = None
        self.lines = []
        self.samples = []
        self.on = threading.Event()
        self.done = threading.Event()

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:  # the NVML device of this CUDA device (CUDA_VISIBLE_DEVICES may renumber)
            uuid = "GPU-" + str(torch.cuda.get_device_properties(self.index).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid.encode())
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def start(self):
        try:
            self.nvml, self.handle = self._nvml_handle()
            self.smax = float(self.nvml.nvmlDeviceGetMaxClockInfo(self.handle, self.nvml.NVML_CLOCK_SM))
            get = getattr(self.nvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                self.nvml.nvmlDeviceGetCurrentClocksThrottleReasons
            self.reasons_of = lambda: int(get(self.handle))
            self.th = threading.Thread(target=self._poll, daemon=True)
            self.th.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def begin(self):
        self.on.set()

    def end(self):
        self.on.clear()

    def _poll(self):
        while not self.done.is_set():
            if self.on.wait(timeout=0.05) and not self.done.is_set():
                try:
                    sm = float(self.nvml.nvmlDeviceGetClockInfo(self.handle, self.nvml.NVML_CLOCK_SM))
                    self.samples.append((sm, self.reasons_of()))
                except Exception:
                    pass
                time.sleep(0.005)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml is not None:
            self.done.set()
            self.on.set()
            self.th.join(timeout=5)
            try:
                self.nvml.nvmlShutdown()
            except Exception:
                pass
            sm = [x for x, _ in self.samples]
            reasons = sorted(n for n, bit in self.REASON_BITS.items() if any(r & bit for _, r in self.samples))
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.smax,
                    "reasons": reasons, "samples": len(sm), "source": "nvml, timed steps only"}
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi, warm-up and timed steps"}


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_reference_steps(nsteps_max, warmup, budget_s=150.0):
    """The reference's C PPE (oracle/_ref) inside the restated Fortran step on
    all host threads; returns (steps_per_s, threads, sample description)."""
    from oracle import oracle as O
    threads = cpu_threads()
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    g = O.Grid(NX, NY, NZ, stretch=STRETCH, re_tau=RE_TAU, dt=DT)
    u, v, w, p = g.init_flow(SEED, NOISE)
    u1, v1, w1 = g.zeros(), g.zeros(), g.zeros()
    if O.ref_available() and PARTS == 0:
        ppe = O.RefPPE(NX, NY, NZ, g.g.dx, g.g.dy, g.dzf_global)
        what = "reference C PPE (src/src_c built unmodified) + C restatement of the Fortran stencils"
    else:
        ppe = O.PPE(NX, NY, NZ, g.g.dx, g.g.dy, g.dzf_global, nparts=PARTS)
        what = "C restatement of the PPE" + (f" (PDD, {PARTS} partitions)" if PARTS else "") + \
               " and of the Fortran stencils"
    t0 = time.perf_counter()
    for _ in range(max(1, warmup)):
        g.step(ppe, u, v, w, u1, v1, w1, p)
    t_first = (time.perf_counter() - t0) / max(1, warmup)
    n = max(1, min(nsteps_max, int(budget_s / max(t_first, 1e-3))))
    t0 = time.perf_counter()
    for _ in range(n):
        g.step(ppe, u, v, w, u1, v1, w1, p)
    dt = time.perf_counter() - t0
    if hasattr(ppe, "close"):
        ppe.close()
    sample = f"{n} full {NX}x{NY}x{NZ} step(s) after {max(1, warmup)} warm-up, {threads} OpenMP threads: {what}"
    return n / dt, threads, sample


def dist_setup(n_gpus, backend="nccl"):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    """all ranks reach this point (no-op on one rank)"""
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world, device="cuda"):
    """the largest x over the ranks: a multi-GPU time is its slowest rank's
    (device: where the reduction's tensor lives, "cuda" for NCCL, "cpu" for gloo)"""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference(args):
    # the CPU arm needs no process group: rank 0 alone runs, the others exit
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sps, threads, sample = cpu_reference_steps(args.steps, args.warmup)
    line = {
        "impl": "reference", "metric": METRIC, "value": sps, "unit": "steps/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / sps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "precision": "fp64 (reference path)", "parallelism": "host cores"},
        "cpu_baseline": {"value": sps, "unit": "steps/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": sps, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _timed(ch, K, W, body, world, clocks=None):
    """device time of K calls of body after W untimed ones: CUDA events on
    the channel's stream, barrier and synchronisation on both sides, the
    slowest rank's; `clocks` (a started ClockSampler) samples while the K
    calls are enqueued and run"""
    import torch
    for _ in range(W):
        body()
    ch.synchronize()
    torch.cuda.synchronize()
    st = torch.cuda.ExternalStream(ch.stream_handle)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    if clocks is not None:
        clocks.begin()
    e0.record(st)
    for _ in range(K):
        body()
    e1.record(st)
    ch.synchronize()
    torch.cuda.synchronize()
    if clocks is not None:
        clocks.end()
    barrier(world)
    return max_over_ranks(e0.elapsed_time(e1), world)


def run_slabs(args, world, rank, local):
    """N GPUs, one z slab each (weak scaling): see the module docstring"""
    import torch
    import powerllel_channel_b200 as plb
    from powerllel_channel_b200 import slab as S
    nzg = NZ * world
    nzs = S.slab_sizes(nzg, world)[1]
    peak, peak_kind = peaks()
    npts = NX * NY * nzs[rank]
    workload = (f"channel {NX}x{NY}x{nzg} as {world} z slabs of {NX}x{NY}x{NZ} (one per GPU), Re_tau {RE_TAU:g}, "
                f"tanh stretch {STRETCH:g}, PDD over {world} partitions, dt {DT:g}, seed {SEED}, noise {NOISE:g}")

    def measure(prec):
        cfg = plb.ChannelConfig(nx=NX, ny=NY, nz=nzg, stretch_ratio=STRETCH, re_tau=RE_TAU, dt=DT, precision=prec,
                                trid_parts=world)
        sl = S.Slab(cfg, rank, world)
        tr = S.DistTransport(sl)
        S.init_flow([sl], tr, nzs, SEED, NOISE)
        clocks = ClockSampler(local)
        clocks.start()
        ms = _timed(sl, args.steps, args.warmup, lambda: S.step([sl], tr, nzs), world, clocks)
        clk = clocks.stop()
        # per-phase device times over 3 steps (events on the slab's stream)
        st = torch.cuda.ExternalStream(sl.stream_handle)
        names, evs = [], []

        def mark(name):
            e = torch.cuda.Event(enable_timing=True)
            e.record(st)
            names.append(name)
            evs.append(e)
        mark("start")
        for _ in range(3):
            S.step([sl], tr, nzs, mark)
        sl.synchronize()
        nper = (len(evs) - 1) // 3
        prof = []
        for q in range(nper):
            t = sum(evs[s * nper + q].elapsed_time(evs[s * nper + q + 1]) for s in range(3)) / 3
            prof.append((names[q + 1], t))
        return sl, tr, ms, clk, prof

    sl, tr, ms64, clk64, prof64 = measure(plb.PL_FP64)
    sl.close()
    sl, tr, msm, clkm, profm = measure(plb.PL_MIXED)
    sps64 = world * args.steps / (ms64 / 1000.0)
    spsm = world * args.steps / (msm / 1000.0)
    top = max((kv for kv in profm if not kv[0].startswith("x_")), key=lambda kv: kv[1])
    alg = ALG_BYTES["mixed"].get(top[0], 0) * npts
    achieved = alg / (top[1] / 1000.0) / 1e9
    traffic = traffic_from_profiles(top[0])

    # end to end: every step uploads this rank's u, v, w slab from pinned
    # host memory, steps, downloads them
    host = torch.empty(3 * sl.compact_elems, dtype=torch.float64).pin_memory()
    sl.download_compact(host.data_ptr())
    sl.synchronize()
    nbytes = 3 * sl.compact_elems * 8
    ke = max(3, min(args.steps, 10))

    def e2e_body():
        sl.upload_compact(host.data_ptr())
        S.step([sl], tr, nzs)
        sl.download_compact(host.data_ptr())

    ms_e2e = _timed(sl, ke, 1, e2e_body, world)
    e2e_sps = world * ke / (ms_e2e / 1000.0)
    launches = S.launches_per_step(sl)
    sl.close()
    del host

    if rank == 0:
        def table(prof):
            tot = sum(t for _, t in prof)
            return {n: {"ms": round(t, 4), "share": round(t / tot, 4)} for n, t in prof}
        line = {
            "metric": METRIC, "value": spsm, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": msm / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "mixed: f32 stencils/FFT/pressure state, f64 u,v,w and tridiagonal",
            "data": "synthetic",
            "config": {"workload": workload, "precision": "mixed", "grid": [NX, NY, nzg], "slab": [NX, NY, NZ],
                       "l2": "inputs larger than L2 (403 MB per FP64 field per GPU), no flush",
                       "parallelism": f"{world} z slabs, PDD across GPUs, NCCL plane exchanges",
                       "value": "slab-steps/s (512x384x256 steps/s)"},
            "fp64_steps_per_s": sps64, "fp64_ms_per_step": ms64 / args.steps,
            "mixed_over_fp64": spsm / sps64,
            "clocks": clkm, "clocks_fp64": clk64,
            "e2e": {"value": e2e_sps, "unit": "steps/s", "h2d_bytes_per_step": nbytes,
                    "d2h_bytes_per_step": nbytes, "per": "rank"},
            "gpu_launches": launches * args.steps,
            "roofline": {"bound": "hbm", "kernel": top[0], "achieved": round(achieved, 1), "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "traffic": traffic, "alg_bytes": alg},
            "phases_mixed_rank0": table(profm), "phases_fp64_rank0": table(prof64),
            "cpu_baseline": None,
        }
        print(json.dumps(line), flush=True)
    import torch.distributed as dist
    dist.destroy_process_group()


def run_b200(args):
    world, rank, local = dist_setup(args.gpus)
    import numpy as np
    import torch
    torch.cuda.set_device(local)
    if world > 1:
        run_slabs(args, world, rank, local)
        return
    import powerllel_channel_b200 as plb

    def timed(ch, K, W, body, clocks=None):
        return _timed(ch, K, W, body, world, clocks)

    peak, peak_kind = peaks()
    npts = NX * NY * NZ

    def measure(prec_name, prec):
        cfg = plb.ChannelConfig(nx=NX, ny=NY, nz=NZ, stretch_ratio=STRETCH, re_tau=RE_TAU, dt=DT, precision=prec,
                                trid_parts=PARTS)
        ch = plb.Channel(cfg)
        ch.init_flow(SEED, NOISE)
        clocks = ClockSampler(local)
        clocks.start()
        ms = timed(ch, args.steps, args.warmup, lambda: ch.step(1), clocks)
        clk = clocks.stop()
        prof = ch.profile(3)
        alg = ALG_BYTES[prec_name]
        tot_ms = sum(t for _, t in prof)
        kernels = {name: {"ms": round(t, 4), "share": round(t / tot_ms, 4),
                          "alg_gbs": round(alg.get(name, 0) * npts / (t / 1000.0) / 1e9, 1)}
                   for name, t in prof}
        return ch, ms, clk, prof, kernels

    ch64, ms64, clk64, prof64, kern64 = measure("fp64", plb.PL_FP64)
    ch64.close()
    chm, msm, clkm, profm, kernm = measure("mixed", plb.PL_MIXED)
    sps64 = world * args.steps / (ms64 / 1000.0)
    spsm = world * args.steps / (msm / 1000.0)

    # dominant kernel of the headline (mixed) step -> roofline
    top = max(profm, key=lambda kv: kv[1])
    alg = ALG_BYTES["mixed"].get(top[0], 0) * npts
    achieved = alg / (top[1] / 1000.0) / 1e9
    traffic = traffic_from_profiles(top[0])

    # end to end through the C ABI with host (pinned) buffers: every step
    # uploads u,v,w, steps, downloads u,v,w
    host = torch.empty(3 * chm.compact_elems, dtype=torch.float64).pin_memory()
    chm.download_compact(host.data_ptr())
    chm.synchronize()
    nbytes = 3 * chm.compact_elems * 8
    ke = max(3, min(args.steps, 10))

    def e2e_body():
        chm.upload_compact(host.data_ptr())
        chm.step(1)
        chm.download_compact(host.data_ptr())

    ms_e2e = timed(chm, ke, 1, e2e_body)
    e2e_sps = world * ke / (ms_e2e / 1000.0)
    chm.close()
    del host

    # accuracy after 100 steps from the same initial field: both paths against
    # the oracle (the reference's own C PPE inside the restated stencils, run
    # in a subprocess on all host threads).  That oracle run is also the CPU
    # baseline: its steps after the first are the timed sample.
    acc, cpu = None, None
    if rank == 0 and world == 1 and not args.no_accuracy and (NX, NY, NZ, PARTS) == (512, 384, 256, 0):
        import tempfile
        from oracle import run_channel as R  # the checker and the CPU-baseline leg
        gpu_fields, gpu_div = {}, {}
        for name, prec in (("fp64", plb.PL_FP64), ("mixed", plb.PL_MIXED)):
            cfg = plb.ChannelConfig(nx=NX, ny=NY, nz=NZ, stretch_ratio=STRETCH, re_tau=RE_TAU, dt=DT, precision=prec)
            ch = plb.Channel(cfg)
            ch.init_flow(SEED, NOISE)
            ch.step(100)
            gpu_fields[name] = [ch.get_field(q)[1:-1, 1:-1, 1:-1] for q in range(4)]
            gpu_div[name] = ch.diagnostics()["div_max"]
            ch.close()
        with tempfile.TemporaryDirectory() as td:
            meta = R.run(td, (NX, NY, NZ), [100], stretch=STRETCH, re_tau=RE_TAU, dt=DT, seed=SEED, noise=NOISE)
            ref = R.load(td, 100)
            acc = {"steps": 100, "reference": "oracle: " + meta["what"],
                   "p": "modulo its mean (the Neumann null mode)"}
            for name in ("fp64", "mixed"):
                for q, n in enumerate("uvwp"):
                    a, b = gpu_fields[name][q], np.asarray(ref[q])
                    if n == "p":
                        a, b = a - a.mean(), b - b.mean()
                    acc[f"{name}_{n}_rel_l2"] = float(np.linalg.norm(a - b) / np.linalg.norm(b))
                    acc[f"{name}_{n}_rel_max"] = float(np.abs(a - b).max() / np.abs(b).max())
                acc[f"div_max_{name}"] = gpu_div[name]
            del ref
        del gpu_fields
        st = meta["step_seconds"][1:]
        if not args.no_cpu_baseline:
            cpu = {"value": len(st) / sum(st), "unit": "steps/s", "cores": meta["threads"], "kind": "port",
                   "sample": f"steps 2-{len(st) + 1} of the {NX}x{NY}x{NZ} 100-step oracle run of the accuracy "
                             f"check, {meta['threads']} OpenMP threads: {meta['what']}"}

    if cpu is None and rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            sps_cpu, threads, sample = cpu_reference_steps(2, 1, budget_s=25.0)
            cpu = {"value": sps_cpu, "unit": "steps/s", "cores": threads, "kind": "port", "sample": sample}
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "steps/s", "cores": cpu_threads(), "kind": "port",
                   "sample": f"unavailable: {e}"}

    if rank == 0:
        fbytes = NX * NY * (NZ + 2) * 8
        line = {
            "metric": METRIC, "value": spsm, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": msm / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "mixed: f32 stencils/FFT/pressure state, f64 u,v,w and tridiagonal",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "precision": "mixed", "grid": [NX, NY, NZ],
                       "l2": (f"inputs larger than L2 ({fbytes / 1e6:.0f} MB per FP64 field), no flush"
                              if fbytes > 126e6 else
                              f"{fbytes / 1e6:.1f} MB per FP64 field: the working set stays in L2 (no flush)"),
                       "trid_parts": PARTS, "parallelism": "1 GPU"},
            "fp64_steps_per_s": sps64, "fp64_ms_per_step": ms64 / args.steps,
            "mixed_over_fp64": spsm / sps64,
            "accuracy_after_100_steps": acc,
            "clocks": clkm, "clocks_fp64": clk64,
            "e2e": {"value": e2e_sps, "unit": "steps/s", "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes},
            "gpu_launches": (LAUNCHES["mixed"] + (1 if PARTS > 32 else 0)) * args.steps,
            "roofline": {"bound": "hbm", "kernel": top[0], "achieved": round(achieved, 1), "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "traffic": traffic, "alg_bytes": alg},
            "kernels_mixed": kernm, "kernels_fp64": kern64,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_capture(args):
    """One precision path only, no timing and no JSON line: the command a
    profiler wraps.  Builds the channel, fills the seeded initial field and
    runs --warmup then --steps steps (step 3 on is a steady-state step of the
    mixed path: its pressure prediction and increment are live)."""
    import torch
    torch.cuda.set_device(0)
    import powerllel_channel_b200 as plb
    prec = plb.PL_MIXED if args.capture == "mixed" else plb.PL_FP64
    cfg = plb.ChannelConfig(nx=NX, ny=NY, nz=NZ, stretch_ratio=STRETCH, re_tau=RE_TAU, dt=DT, precision=prec,
                            trid_parts=args.trid_parts or PARTS)
    ch = plb.Channel(cfg)
    ch.init_flow(SEED, NOISE)
    ch.step(args.warmup + args.steps)
    ch.synchronize()
    print(json.dumps({"capture": args.capture, "grid": [NX, NY, NZ], "steps": args.warmup + args.steps,
                      "diag": ch.diagnostics()}), flush=True)
    ch.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the 100-step accuracy comparison")
    ap.add_argument("--grid", type=int, nargs=3, default=None,
                    help="override the grid (profiling captures on a smaller case); the bench line is only "
                         "valid at the default 512 384 256")
    ap.add_argument("--capture", choices=["fp64", "mixed"], default=None,
                    help="run one precision path untimed (the command an ncu capture wraps)")
    ap.add_argument("--trid-parts", type=int, default=0, help="--capture only: PDD partitions (0 = Thomas)")
    ap.add_argument("--config", choices=sorted(CONFIGS), default=None,
                    help="one of the benchmark configurations (default: C3, the headline workload); the 100-step "
                         "accuracy comparison runs for C3 only")
    args = ap.parse_args()
    if args.config:
        set_config(args.config)
    if args.warmup < 3:
        args.warmup = 3
    if args.grid:
        global NX, NY, NZ, WORKLOAD
        NX, NY, NZ = args.grid
        WORKLOAD = WORKLOAD.replace("512x384x256", f"{NX}x{NY}x{NZ}")
    if args.capture:
        run_capture(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
