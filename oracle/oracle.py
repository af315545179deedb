"""CPU oracle for the PowerLLEL_Channel RK2 projection step (ctypes wrappers).

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / reference arm of ``bench.py`` may import this module, and only
as the checker or the timed CPU baseline.  The product package
``powerllel_channel_b200`` never imports it.

Two CPU implementations are wrapped:

* ``liboracle.so``  -- this repository's C restatement (oracle_*.c) of the
  reference's PPE (src/src_c/mod_poisson_solver.c), of the FFTW R2HC/HC2R
  definitions and of the Fortran stencils (mod_calcVel, mod_calcRHS,
  mod_updateBound, mod_utils, mod_mesh, mod_initFlow, main.f90:131-208).
* ``_ref/``         -- the reference's own C PPE (src/src_c) compiled unmodified
  against shim/mpi.h and shim/fftw3.h by oracle/Makefile; ``ref_ppe_run`` (Thomas)
  and ``ref_ppe_pdd_run`` (PDD, forked ranks) executables and ``libref_ppe.so``.

Arrays are numpy float64 in the reference layout: Fortran order with one ghost
layer, i.e. a C-contiguous array of shape (nz+2, ny+2, nx+2) indexed [k, j, i].
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_dp = C.POINTER(C.c_double)


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


class _Grid(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double),
        ("dx", C.c_double), ("dy", C.c_double), ("dx_inv", C.c_double), ("dy_inv", C.c_double),
        ("re", C.c_double), ("re_inv", C.c_double), ("u_ref", C.c_double), ("l_ref", C.c_double),
        ("dt", C.c_double), ("u_crf", C.c_double),
        ("is_forced", C.c_int * 3), ("vel_force", C.c_double * 3),
        ("dzf_global", _dp), ("zc_global", _dp), ("dzf", _dp), ("dzf_inv", _dp),
        ("dzc", _dp), ("dzc_inv", _dp), ("dzflzi", _dp),
    ]


_lib = None


def build(force: bool = False) -> None:
    """Build liboracle.so (and _ref/ when the reference tree exists)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        gp = C.POINTER(_Grid)
        L.orc_grid_init.argtypes = [gp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                    C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                    C.c_double, C.c_double, C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.orc_grid_free.argtypes = [gp]
        L.orc_uniform.argtypes = [C.c_uint64, C.c_uint64]
        L.orc_uniform.restype = C.c_double
        L.orc_init_flow.argtypes = [gp, C.c_uint64, C.c_double, _dp, _dp, _dp, _dp]
        for name in ("orc_rk1", "orc_rk2"):
            getattr(L, name).argtypes = [gp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.orc_update_bound_vel.argtypes = [gp, _dp, _dp, _dp]
        L.orc_update_bound_p.argtypes = [gp, _dp]
        L.orc_calc_rhs.argtypes = [gp, _dp, _dp, _dp, _dp]
        L.orc_correct_vel.argtypes = [gp, _dp, _dp, _dp, _dp]
        L.orc_mean_h.argtypes = [gp, _dp]
        L.orc_mean_h.restype = C.c_double
        L.orc_force_vel.argtypes = [gp, _dp, _dp, _dp]
        for name in ("orc_max_div", "orc_max_cfl"):
            getattr(L, name).argtypes = [gp, _dp, _dp, _dp, C.POINTER(C.c_int)]
            getattr(L, name).restype = C.c_double
        L.orc_has_nan.argtypes = [gp, _dp]
        L.orc_has_nan.restype = C.c_int
        L.orc_ppe_init.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, _dp, C.c_int]
        L.orc_ppe_init.restype = C.c_void_p
        L.orc_ppe_execute.argtypes = [C.c_void_p, _dp]
        L.orc_slab_forward.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
        L.orc_slab_iface.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp]
        L.orc_slab_finish.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp]
        L.orc_slab_extent.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.orc_ppe_free.argtypes = [C.c_void_p]
        L.orc_ppe_pivots.argtypes = [C.c_void_p]
        L.orc_ppe_pivots.restype = _dp
        L.orc_step.argtypes = [gp, C.c_void_p, C.c_void_p, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        _lib = L
    return _lib


def re_from_retau(re_tau: float) -> float:
    """Invert the reference's own correlation retau = 0.09*re**0.88
    (mod_initFlow.f90:109)."""
    return (re_tau / 0.09) ** (1.0 / 0.88)


class Grid:
    """Mesh + physical parameters (mod_mesh.f90:26-84, mod_parameters.f90)."""

    def __init__(self, nx, ny, nz, lx=2 * math.pi, ly=math.pi, lz=2.0, stretch=1.5, mesh_type=1,
                 stretch_func=0, re=None, re_tau=180.0, u_ref=1.0, l_ref=1.0, dt=1e-4, u_crf=0.0,
                 is_forced=(1, 0, 0), vel_force=(1.0, 0.0, 0.0)):
        L = lib()
        self.g = _Grid()
        if re is None:
            re = re_from_retau(re_tau)
        f = (C.c_int * 3)(*[int(x) for x in is_forced])
        vf = (C.c_double * 3)(*vel_force)
        L.orc_grid_init(C.byref(self.g), nx, ny, nz, lx, ly, lz, mesh_type, stretch_func, stretch, re, u_ref,
                        l_ref, dt, u_crf, f, vf)
        self.nx, self.ny, self.nz = nx, ny, nz
        self.shape = (nz + 2, ny + 2, nx + 2)

    def __del__(self):
        try:
            lib().orc_grid_free(C.byref(self.g))
        except Exception:
            pass

    def arr1d(self, name):
        p = getattr(self.g, name)
        return np.ctypeslib.as_array(p, shape=(self.nz + 2,)).copy()

    @property
    def dzf_global(self):
        return self.arr1d("dzf_global")

    def zeros(self):
        return np.zeros(self.shape, dtype=np.float64)

    def init_flow(self, seed, noise):
        u, v, w, p = (self.zeros() for _ in range(4))
        lib().orc_init_flow(C.byref(self.g), seed, noise, _ptr(u), _ptr(v), _ptr(w), _ptr(p))
        return u, v, w, p

    # stencils -------------------------------------------------------------
    def rk1(self, u, v, w):
        u1, v1, w1 = self.zeros(), self.zeros(), self.zeros()
        lib().orc_rk1(C.byref(self.g), _ptr(u), _ptr(v), _ptr(w), _ptr(u1), _ptr(v1), _ptr(w1))
        return u1, v1, w1

    def rk2(self, u, v, w, u1, v1, w1):
        lib().orc_rk2(C.byref(self.g), _ptr(u), _ptr(v), _ptr(w), _ptr(u1), _ptr(v1), _ptr(w1))

    def bound_vel(self, u, v, w):
        lib().orc_update_bound_vel(C.byref(self.g), _ptr(u), _ptr(v), _ptr(w))

    def bound_p(self, p):
        lib().orc_update_bound_p(C.byref(self.g), _ptr(p))

    def calc_rhs(self, u, v, w, p):
        lib().orc_calc_rhs(C.byref(self.g), _ptr(u), _ptr(v), _ptr(w), _ptr(p))

    def correct_vel(self, p, u, v, w):
        lib().orc_correct_vel(C.byref(self.g), _ptr(p), _ptr(u), _ptr(v), _ptr(w))

    def mean_h(self, var):
        return lib().orc_mean_h(C.byref(self.g), _ptr(var))

    def force_vel(self, u, v, w):
        lib().orc_force_vel(C.byref(self.g), _ptr(u), _ptr(v), _ptr(w))

    def max_div(self, u, v, w):
        ijk = (C.c_int * 3)()
        val = lib().orc_max_div(C.byref(self.g), _ptr(u), _ptr(v), _ptr(w), ijk)
        return val, tuple(ijk)

    def max_cfl(self, u, v, w):
        ijk = (C.c_int * 3)()
        val = lib().orc_max_cfl(C.byref(self.g), _ptr(u), _ptr(v), _ptr(w), ijk)
        return val, tuple(ijk)

    def step(self, ppe, u, v, w, u1, v1, w1, p):
        """main.f90:137-208 with ``ppe`` either a PPE (restated) or RefPPE."""
        fn, ctx = ppe.callback()
        lib().orc_step(C.byref(self.g), fn, ctx, _ptr(u), _ptr(v), _ptr(w), _ptr(u1), _ptr(v1), _ptr(w1),
                       _ptr(p))


class PPE:
    """Restated PPE solver; nparts=0 Thomas, nparts>=1 PDD with nparts z-partitions."""

    def __init__(self, nx, ny, nz, dx, dy, dzf_global, nparts=0):
        self.dzf = np.ascontiguousarray(dzf_global, dtype=np.float64)
        self.h = lib().orc_ppe_init(nx, ny, nz, dx, dy, _ptr(self.dzf), nparts)
        self.n = (nx, ny, nz)
        self.nparts = max(1, nparts)

    def execute(self, var):
        lib().orc_ppe_execute(self.h, _ptr(var))

    def pivots(self):
        nx, ny, nz = self.n
        p = lib().orc_ppe_pivots(self.h)
        return np.ctypeslib.as_array(p, shape=(nz, ny, nx)).copy()

    def callback(self):
        return C.cast(lib().orc_ppe_execute_cb, C.c_void_p), self.h

    def __del__(self):
        try:
            lib().orc_ppe_free(self.h)
        except Exception:
            pass


class SlabPPE:
    """CPU stand-in of one GPU's z slab for the PDD part of the slab schedule
    (powerllel_channel_b200.slab.pdd_solve): partition m of the restated PDD
    solve, with the same phase names and exchanged planes as the library's
    slab.  rhs: the partition's planes of the right-hand side ([k][j][i])."""

    def __init__(self, ppe: "PPE", m: int, rhs: np.ndarray):
        import torch
        nx, ny, _ = ppe.n
        kst, ksz = C.c_int(), C.c_int()
        lib().orc_slab_extent(ppe.h, m, C.byref(kst), C.byref(ksz))
        self.ppe, self.rank, self.kst, self.nz = ppe, m, kst.value, ksz.value
        self.ranks = ppe.nparts
        self.x = np.ascontiguousarray(rhs, dtype=np.float64)
        self.xs = np.zeros_like(self.x)
        self.out = np.zeros_like(self.x)
        self.planes = {5: torch.zeros(nx * ny, dtype=torch.float64), 6: torch.zeros(nx * ny, dtype=torch.float64),
                       7: torch.zeros(nx * ny, dtype=torch.float64), 2: torch.zeros(nx * ny, dtype=torch.float64)}
        self.nxy = nx * ny

    def tensor(self, field, k=0):
        import torch
        if field == 4:  # the sweep buffer's plane k, shared with self.xs
            return torch.from_numpy(self.xs.reshape(self.nz, -1)[k])
        return self.planes[field]

    def rhs_sweep(self):
        lib().orc_slab_forward(self.ppe.h, self.rank, _ptr(self.x), _ptr(self.xs))

    def pdd_iface(self):
        if self.rank + 1 < self.ranks:
            y2 = self.planes[2].numpy()
            lib().orc_slab_iface(self.ppe.h, self.rank, _ptr(self.xs), _ptr(self.planes[5].numpy()), _ptr(y2),
                                 _ptr(self.planes[6].numpy()))

    def finish(self):
        y1 = _ptr(self.planes[7].numpy()) if self.rank > 0 else None
        y2 = _ptr(self.planes[2].numpy()) if self.rank + 1 < self.ranks else None
        lib().orc_slab_finish(self.ppe.h, self.rank, _ptr(self.xs), y1, y2, _ptr(self.out))


def ref_available() -> bool:
    return all(os.path.exists(os.path.join(REF_DIR, f)) for f in ("libref_ppe.so", "ref_ppe_run", "ref_ppe_pdd_run"))


def ref_ppe_run(var, nx, ny, nz, dx, dy, dzf_global, p_row=1, p_col=1, pdd=False, nrep=1, env=None):
    """Run the reference's own execute_poisson_solver on the ghosted array ``var``
    (p_row x p_col forked ranks).  Returns (solution, {"init_s", "exec_s"})."""
    exe = os.path.join(REF_DIR, "ref_ppe_pdd_run" if pdd else "ref_ppe_run")
    with tempfile.TemporaryDirectory() as td:
        fd, fi, fo = (os.path.join(td, n) for n in ("dzf.bin", "in.bin", "out.bin"))
        np.ascontiguousarray(dzf_global, dtype=np.float64).tofile(fd)
        np.ascontiguousarray(var, dtype=np.float64).tofile(fi)
        r = subprocess.run([exe, str(p_row), str(p_col), str(nx), str(ny), str(nz), repr(float(dx)),
                            repr(float(dy)), fd, fi, fo, str(nrep)], capture_output=True, text=True,
                           env=env, check=True)
        out = np.fromfile(fo, dtype=np.float64).reshape(var.shape)
    t = r.stdout.split()
    return out, {"init_s": float(t[1]), "exec_s": float(t[3])}


_ref_lib = None


class RefPPE:
    """The reference's own init/execute/free_poisson_solver in this process (one
    rank, Thomas build), initialised once like main.f90:80 and executed per
    step like main.f90:177.  The reference keeps one global solver instance
    (and its decomp_2d_finalize does not reset its freed work buffers, so a
    second decomp_2d_init double-frees); hence one live RefPPE per process,
    and no re-initialisation after close()."""

    _cb_type = C.CFUNCTYPE(None, C.c_void_p, _dp)
    _live = False
    _used = False

    def __init__(self, nx, ny, nz, dx, dy, dzf_global):
        global _ref_lib
        if RefPPE._live or RefPPE._used:
            raise RuntimeError("the reference PPE supports one init per process")
        if _ref_lib is None:
            _ref_lib = C.CDLL(os.path.join(REF_DIR, "libref_ppe.so"))
            _ref_lib.ref_ppe_setup.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, _dp]
            _ref_lib.ref_ppe_exec.argtypes = [_dp]
            _ref_lib.ref_ppe_teardown.argtypes = []
        self.dzf = np.ascontiguousarray(dzf_global, dtype=np.float64)
        _ref_lib.ref_ppe_setup(nx, ny, nz, dx, dy, _ptr(self.dzf))
        RefPPE._live = True
        RefPPE._used = True

        def _solve(ctx, var):
            _ref_lib.ref_ppe_exec(var)

        self._cb = self._cb_type(_solve)

    def execute(self, var):
        _ref_lib.ref_ppe_exec(_ptr(var))

    def callback(self):
        return C.cast(self._cb, C.c_void_p), None

    def close(self):
        if RefPPE._live:
            _ref_lib.ref_ppe_teardown()
            RefPPE._live = False
