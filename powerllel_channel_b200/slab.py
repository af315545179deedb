"""z slabs of a multi-GPU run: the host side of include/powerllel_b200.h part 5.

The reference decomposes the domain over p_row x p_col MPI ranks; with
p_row = 1 every rank holds a z slab, the x and y transforms are local and the
wall-normal systems are solved by PDD with one partition per rank
(mod_poisson_solver.c:105-176, 361-466).  Here one GPU holds one slab
(:class:`Slab`, over the C ABI) and a step is the library's slab phases with
the exchanges of the reference between them (:func:`step`):

=====================  ==========================================  =========================================
phase                  exchange after it                           reference counterpart
=====================  ==========================================  =========================================
pl_slab_rk             sum of u dzf/lz over the ranks              MPI_ALLREDUCE of Mean_h, mod_utils.f90:127
pl_slab_mean_finish    w plane nz -> upper neighbour's plane 0     updateHalo, mod_updateBound.f90:364-396
pl_slab_rhs_sweep      first swept plane -> lower neighbour        MPI_Sendrecv, mod_poisson_solver.c:415-417
pl_slab_pdd_iface      y3 -> upper neighbour's y1                  MPI_Sendrecv, :444-446
pl_slab_finish         first pressure plane -> lower neighbour     updateBoundP's halo, mod_updateBound.f90:186-239
pl_slab_correct        two u, v, w planes each way                 updateBoundVel's halo, :30-55
=====================  ==========================================  =========================================

The fused RK kernel reads two planes beyond its slab, so one velocity exchange
per step (after the correction) serves both RK stages.  The plane tmp_v, which
init_pdd_array exchanges once (:172-174), is computed by every rank from the
global tables.

A transport moves the planes.  :class:`DistTransport` is one slab per rank
over ``torch.distributed`` (NCCL between GPUs, gloo between CPU processes);
:class:`LocalTransport` holds several slabs in one process on one device and
copies the planes, which checks the slab kernels and the exchange schedule on
a single GPU: every slab's kernels are separate launches that wait on nothing
but the host.

The PDD part of the schedule (:func:`pdd_solve`) takes any object with the
slab PPE phases, so the same schedule also runs over a CPU stand-in in the
tests.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import ChannelConfig, Diag, PL_MIXED, PowerLLELError, _check, lib

# pl_slab_plane fields
F_U, F_V, F_W, F_P, F_SWEEP, F_TVAR, F_Y3, F_Y1, F_MEAN, F_MEAN_INIT = range(10)


def _bind():
    L = lib()
    if getattr(L, "_slab_bound", False):
        return L
    from . import _Config
    L.pl_channel_create_slab.argtypes = [C.POINTER(C.c_void_p), C.POINTER(_Config), C.c_int, C.c_int]
    L.pl_slab_info.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
    L.pl_slab_plane.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_size_t)]
    L.pl_slab_plane.restype = C.c_void_p
    L.pl_slab_init_fill.argtypes = [C.c_void_p, C.c_uint64, C.c_double]
    for name in ("pl_slab_init_finish", "pl_slab_rk", "pl_slab_mean_finish", "pl_slab_rhs_sweep",
                 "pl_slab_pdd_iface", "pl_slab_finish", "pl_slab_correct"):
        getattr(L, name).argtypes = [C.c_void_p]
    L._slab_bound = True
    return L


class _DevArray:
    """A device buffer as an object torch.as_tensor accepts (no copy)."""

    def __init__(self, ptr: int, nbytes: int, itemsize: int):
        self.__cuda_array_interface__ = {"shape": (nbytes // itemsize,), "typestr": "<f8" if itemsize == 8 else "<f4",
                                         "data": (int(ptr), False), "version": 3}


class Slab:
    """One z slab of the global channel ``cfg`` (``cfg.trid_parts`` must equal
    ``z_ranks``) on the current CUDA device."""

    def __init__(self, cfg: ChannelConfig, z_rank: int, z_ranks: int):
        L = _bind()
        self.cfg = cfg
        self._c = cfg.to_c()
        h = C.c_void_p()
        _check(L.pl_channel_create_slab(C.byref(h), C.byref(self._c), int(z_rank), int(z_ranks)),
               "pl_channel_create_slab")
        self._h = h
        info = (C.c_int * 4)()
        L.pl_slab_info(h, info)
        self.kst, self.nz, self.rank, self.ranks = (int(x) for x in info)
        self.mixed = cfg.precision == PL_MIXED

    # the phases -----------------------------------------------------------
    def _run(self, name):
        _check(getattr(lib(), name)(self._h), name)

    def init_fill(self, seed, noise):
        _check(lib().pl_slab_init_fill(self._h, int(seed), float(noise)), "pl_slab_init_fill")

    def init_finish(self):
        self._run("pl_slab_init_finish")

    def rk(self):
        self._run("pl_slab_rk")

    def mean_finish(self):
        self._run("pl_slab_mean_finish")

    def rhs_sweep(self):
        self._run("pl_slab_rhs_sweep")

    def pdd_iface(self):
        self._run("pl_slab_pdd_iface")

    def finish(self):
        self._run("pl_slab_finish")

    def correct(self):
        self._run("pl_slab_correct")

    # planes ---------------------------------------------------------------
    def plane(self, field: int, k: int = 0):
        """(device address, bytes, item size) of an exchanged plane"""
        nb = C.c_size_t()
        ptr = lib().pl_slab_plane(self._h, int(field), int(k), C.byref(nb))
        if not ptr:
            raise PowerLLELError(lib().pl_last_error().decode())
        itemsize = 4 if (field == F_P and self.mixed) else 8
        return ptr, nb.value, itemsize

    def tensor(self, field: int, k: int = 0):
        import torch
        ptr, nb, isz = self.plane(field, k)
        return torch.as_tensor(_DevArray(ptr, nb, isz), device="cuda")

    @property
    def stream_handle(self) -> int:
        return lib().pl_channel_stream(self._h) or 0

    @property
    def compact_elems(self) -> int:
        """doubles per field of upload_compact / download_compact: the slab's
        planes 0 .. nz+1, nx x ny each"""
        return self.cfg.nx * self.cfg.ny * (self.nz + 2)

    def upload_compact(self, host_ptr: int) -> None:
        """u, v, w (planes 0 .. nz+1 each, back to back) from host memory,
        asynchronously on the slab's stream"""
        _check(lib().pl_channel_upload_compact(self._h, C.c_void_p(host_ptr)), "pl_channel_upload_compact")

    def download_compact(self, host_ptr: int) -> None:
        _check(lib().pl_channel_download_compact(self._h, C.c_void_p(host_ptr)), "pl_channel_download_compact")

    def synchronize(self):
        _check(lib().pl_channel_synchronize(self._h), "pl_channel_synchronize")

    def diagnostics(self) -> dict:
        d = Diag()
        _check(lib().pl_channel_diagnostics(self._h, C.byref(d)), "pl_channel_diagnostics")
        out = d.as_dict()
        for key in ("div_ijk", "cfl_ijk"):
            i, j, k = out[key]
            out[key] = (i, j, k + self.kst)
        return out

    def get_field(self, which: int) -> np.ndarray:
        """the slab's planes 0 .. nz+1 in the reference's ghosted layout
        (u, v, w; 3 = p with its zero-gradient ghosts)"""
        nx, ny = self.cfg.nx, self.cfg.ny
        out = np.empty((self.nz + 2, ny + 2, nx + 2))
        _check(lib().pl_channel_get_field(self._h, int(which), out.ctypes.data_as(C.POINTER(C.c_double))),
               "pl_channel_get_field")
        return out

    def close(self):
        if self._h:
            lib().pl_channel_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# transports: exchange(pairs), allreduce_sum(field)
# a pair is (src_rank, src_field, src_k, dst_rank, dst_field, dst_k)
# ---------------------------------------------------------------------------
class LocalTransport:
    """All slabs in this process (one device): planes move by device copies.
    Before a copy every slab's stream has finished, after it the device has."""

    def __init__(self, slabs):
        self.slabs = {s.rank: s for s in slabs}

    def _sync(self):
        import torch
        for s in self.slabs.values():
            s.synchronize()
        torch.cuda.synchronize()

    def exchange(self, pairs):
        self._sync()
        for sr, sf, sk, dr, df, dk in pairs:
            self.slabs[dr].tensor(df, dk).copy_(self.slabs[sr].tensor(sf, sk))
        self._sync()

    def allreduce_sum(self, field):
        self._sync()
        total = sum(s.tensor(field).clone() for s in self.slabs.values())
        for s in self.slabs.values():
            s.tensor(field).copy_(total)
        self._sync()


class DistTransport:
    """One slab per rank over torch.distributed.  The operations are issued on
    the slab's own CUDA stream, so they order with its kernels without a host
    synchronisation (NCCL); on CPU tensors (gloo) they are plain blocking
    calls.  Every rank issues the same pairs in the same order."""

    def __init__(self, slab, group=None, tensor_of=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.slab = slab
        self.rank = slab.rank
        self.tensor_of = tensor_of or (lambda f, k: slab.tensor(f, k))
        self._stream = None
        if tensor_of is None:
            import torch
            self._stream = torch.cuda.ExternalStream(slab.stream_handle)

    def _ctx(self):
        import contextlib
        if self._stream is None:
            return contextlib.nullcontext()
        import torch
        return torch.cuda.stream(self._stream)

    def exchange(self, pairs):
        dist = self.dist
        ops = []
        for sr, sf, sk, dr, df, dk in pairs:
            if sr == self.rank:
                ops.append(dist.P2POp(dist.isend, self.tensor_of(sf, sk), dr, self.group))
            if dr == self.rank:
                ops.append(dist.P2POp(dist.irecv, self.tensor_of(df, dk), sr, self.group))
        if not ops:
            return
        with self._ctx():
            for req in dist.batch_isend_irecv(ops):
                req.wait()

    def allreduce_sum(self, field):
        with self._ctx():
            self.dist.all_reduce(self.tensor_of(field, 0), op=self.dist.ReduceOp.SUM, group=self.group)


# ---------------------------------------------------------------------------
# the schedule
# ---------------------------------------------------------------------------
def _pairs_up(nzs, src_field, src_k, dst_field, dst_k):
    """rank r's plane -> rank r+1 (src_k / dst_k may depend on the rank's nz)"""
    return [(r, src_field, src_k(nzs[r]), r + 1, dst_field, dst_k(nzs[r + 1])) for r in range(len(nzs) - 1)]


def _pairs_down(nzs, src_field, src_k, dst_field, dst_k):
    """rank r+1's plane -> rank r"""
    return [(r + 1, src_field, src_k(nzs[r + 1]), r, dst_field, dst_k(nzs[r])) for r in range(len(nzs) - 1)]


def velocity_halo_pairs(nzs):
    """two planes of u, v, w each way across every interface"""
    pairs = []
    for f in (F_U, F_V, F_W):
        for d in (1, 2):
            pairs += _pairs_down(nzs, f, lambda n, d=d: d, f, lambda n, d=d: n + d)      # planes 1, 2 -> nz+1, nz+2
            pairs += _pairs_up(nzs, f, lambda n, d=d: n - 2 + d, f, lambda n, d=d: d - 2)  # nz-1, nz -> -1, 0
    return pairs


def _noop(name):
    pass


def pdd_solve(slabs, transport, nzs, mark=_noop):
    """the PDD part of the solve: local sweeps, the first swept plane down,
    the interface solves, y3 up, the corrections and inverse transforms"""
    for s in slabs:
        s.rhs_sweep()
    mark("rhs_sweep")
    transport.exchange(_pairs_down(nzs, F_SWEEP, lambda n: 0, F_TVAR, lambda n: 0))
    mark("x_tvar")
    for s in slabs:
        s.pdd_iface()
    mark("pdd_iface")
    transport.exchange(_pairs_up(nzs, F_Y3, lambda n: 0, F_Y1, lambda n: 0))
    mark("x_y3")
    for s in slabs:
        s.finish()
    mark("pdd_finish")


def step(slabs, transport, nzs, mark=_noop):
    """one RK2 projection step (main.f90:137-208) over the slabs of this
    process; nzs: every rank's plane count.  mark(name) is called after
    each phase and exchange is issued (a profiler records an event there)."""
    for s in slabs:
        s.rk()
    mark("rk_fused")
    transport.allreduce_sum(F_MEAN)
    mark("x_mean")
    for s in slabs:
        s.mean_finish()
    mark("mean_finish")
    transport.exchange(_pairs_up(nzs, F_W, lambda n: n, F_W, lambda n: 0))
    mark("x_w")
    pdd_solve(slabs, transport, nzs, mark)
    transport.exchange(_pairs_down(nzs, F_P, lambda n: 0, F_P, lambda n: n))
    mark("x_p")
    for s in slabs:
        s.correct()
    mark("correct_force")
    transport.exchange(velocity_halo_pairs(nzs))
    mark("x_vel")


def launches_per_step(slab) -> int:
    """this library's kernel launches in one step of ``slab``: RK 1, the
    Mean_h finish 1, the fused divergence + x transform, y transform and
    sweep 3 (mixed: + the plane sums and the FP64 widening), the interface
    solve 1 (not on the top slab), correction + inverse y and x transforms 3,
    velocity correction 1"""
    return 1 + 1 + (5 if slab.mixed else 3) + (1 if slab.rank < slab.ranks - 1 else 0) + 3 + 1


def init_flow(slabs, transport, nzs, seed, noise):
    """initFlow over the slabs: the seeded field (global counters), the
    cross-rank Mean_h normalisation, the velocity halos"""
    for s in slabs:
        s.init_fill(seed, noise)
    transport.allreduce_sum(F_MEAN_INIT)
    for s in slabs:
        s.init_finish()
    transport.exchange(velocity_halo_pairs(nzs))


def slab_sizes(nz: int, ranks: int):
    """decomp_2d.c:261-283: (first plane, plane count) of every rank"""
    size = nz // ranks
    nu = nz - size * ranks
    nl = ranks - nu
    st, sz = [], []
    start = 0
    for r in range(ranks):
        n = size if r < nl else size + 1
        st.append(start)
        sz.append(n)
        start += n
    return st, sz


def diagnostics(per_slab):
    """checkNaN / calcMaxCFL / calcMaxDiv over the slabs' results (the
    reference's max-location reduction, mod_utils.f90:165-181: the largest
    value, the first in k, j, i order among equal ones)"""
    div = max(per_slab, key=lambda d: (d["div_max"], -d["div_ijk"][2]))
    cfl = max(per_slab, key=lambda d: (d["cfl_max"], -d["cfl_ijk"][2]))
    return {"div_max": div["div_max"], "div_ijk": div["div_ijk"], "cfl_max": cfl["cfl_max"],
            "cfl_ijk": cfl["cfl_ijk"], "nan_count": sum(d["nan_count"] for d in per_slab)}
