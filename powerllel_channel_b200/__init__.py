"""PowerLLEL_Channel RK2 projection step on one NVIDIA B200.

Host-side mirror of the reference's interfaces over the C ABI of
``libpowerllel_b200.so`` (declared in ``include/powerllel_b200.h``):

* :class:`PoissonSolver` -- the reference PPE call sequence
  ``init_poisson_solver / execute_poisson_solver / free_poisson_solver``
  (src/src_c/mod_poisson_solver.c:178,468,607) on host arrays in the reference's
  ghosted Fortran layout;
* :class:`DevicePoissonSolver` -- the same operator on device-resident arrays;
* :class:`Channel` -- the whole time step of main.f90:131-208 on device-resident
  fields, with the reference's configuration names (mod_parameters.f90).

The CUDA library is the only compute path: importing this package without the
built library raises, there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpowerllel_b200.so")

PL_FP64 = 0
PL_MIXED = 1

_dp = C.POINTER(C.c_double)
_lib = None


class PowerLLELError(RuntimeError):
    pass


class _Config(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double),
        ("mesh_type", C.c_int), ("stretch_func", C.c_int), ("stretch_ratio", C.c_double),
        ("re", C.c_double), ("u_ref", C.c_double), ("l_ref", C.c_double),
        ("dt", C.c_double), ("u_crf", C.c_double),
        ("is_forced", C.c_int * 3), ("vel_force", C.c_double * 3),
        ("trid_parts", C.c_int), ("precision", C.c_int),
    ]


class Diag(C.Structure):
    _fields_ = [
        ("div_max", C.c_double), ("cfl_max", C.c_double),
        ("div_ijk", C.c_int * 3), ("cfl_ijk", C.c_int * 3), ("nan_count", C.c_int),
    ]

    def as_dict(self):
        return {"div_max": self.div_max, "cfl_max": self.cfl_max, "div_ijk": tuple(self.div_ijk),
                "cfl_ijk": tuple(self.cfl_ijk), "nan_count": self.nan_count}


def lib():
    """Load libpowerllel_b200.so; raise if it is missing (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise PowerLLELError(f"{LIB_PATH} is missing: build it with `python -m powerllel_channel_b200.build` "
                             "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    L.init_poisson_solver.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, _dp, C.c_char_p,
                                      C.c_char_p, C.c_char_p, C.POINTER(C.c_int)]
    L.init_poisson_solver.restype = None
    L.execute_poisson_solver.argtypes = [_dp]
    L.execute_poisson_solver.restype = None
    L.free_poisson_solver.argtypes = []
    L.free_poisson_solver.restype = None
    L.pl_set_trid_partitions.argtypes = [C.c_int]
    L.pl_last_error.restype = C.c_char_p
    L.pl_ppe_create.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, _dp,
                                C.c_int, C.c_int]
    L.pl_ppe_solve.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.pl_ppe_destroy.argtypes = [C.c_void_p]
    L.pl_ppe_solve_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.pl_channel_create.argtypes = [C.POINTER(C.c_void_p), C.POINTER(_Config)]
    L.pl_channel_destroy.argtypes = [C.c_void_p]
    L.pl_channel_init_flow.argtypes = [C.c_void_p, C.c_uint64, C.c_double]
    L.pl_channel_step.argtypes = [C.c_void_p, C.c_int]
    L.pl_channel_synchronize.argtypes = [C.c_void_p]
    L.pl_channel_diagnostics.argtypes = [C.c_void_p, C.POINTER(Diag)]
    L.pl_channel_get_fields.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp]
    L.pl_channel_set_fields.argtypes = [C.c_void_p, _dp, _dp, _dp]
    L.pl_channel_get_field.argtypes = [C.c_void_p, C.c_int, _dp]
    L.pl_channel_upload_compact.argtypes = [C.c_void_p, C.c_void_p]
    L.pl_channel_download_compact.argtypes = [C.c_void_p, C.c_void_p]
    L.pl_channel_field.argtypes = [C.c_void_p, C.c_int]
    L.pl_channel_field.restype = C.c_void_p
    L.pl_channel_stream.argtypes = [C.c_void_p]
    L.pl_channel_stream.restype = C.c_void_p
    L.pl_channel_profile.argtypes = [C.c_void_p, C.c_int, _dp, C.c_char_p, C.c_int]
    L.pl_channel_set_body_force.argtypes = [C.c_void_p, _dp]
    L.pl_channel_kinetic_energy.argtypes = [C.c_void_p, _dp]
    L.pl_adjoint_ke_gradient.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, C.c_void_p, C.c_void_p, C.c_void_p, _dp]
    L.pl_stat_enable.argtypes = [C.c_void_p, C.c_uint, C.c_int, C.c_int]
    L.pl_stat_init.argtypes = [C.c_void_p]
    L.pl_stat_sample.argtypes = [C.c_void_p, C.c_int]
    L.pl_stat_info.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.pl_stat_get.argtypes = [C.c_void_p, C.c_int, _dp]
    L.pl_stat_disable.argtypes = [C.c_void_p]
    L.pl_monitor_skin_friction.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
    L.pl_monitor_forcing.argtypes = [C.c_void_p, _dp]
    L.pl_monitor_probe.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, _dp]
    L.pl_monitor_region.argtypes = [C.c_void_p, C.POINTER(C.c_int), _dp]
    for name in ("pl_phase_rk", "pl_phase_rk1", "pl_phase_rk2", "pl_phase_calc_rhs", "pl_phase_poisson", "pl_phase_correct_force"):
        getattr(L, name).argtypes = [C.c_void_p]
    _lib = L
    return L


def _check(rc: int, what: str):
    if rc != 0:
        raise PowerLLELError(f"{what}: {lib().pl_last_error().decode()}")


def _ptr(a: np.ndarray | None):
    if a is None:
        return None
    if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
        raise PowerLLELError("arrays must be C-contiguous float64")
    return a.ctypes.data_as(_dp)


def re_from_retau(re_tau: float) -> float:
    """Reynolds number from Re_tau by inverting the reference's own correlation
    retau = 0.09*re**0.88 (mod_initFlow.f90:109)."""
    return (re_tau / 0.09) ** (1.0 / 0.88)


# ----------------------------------------------------------------------------
# PPE, reference call sequence
# ----------------------------------------------------------------------------
class PoissonSolver:
    """init/execute/free_poisson_solver (mod_poisson_solver.c:178,468,607) on
    host arrays.  ``var`` is the ghosted (nz+2, ny+2, nx+2) float64 array of
    the reference (Fortran order); only its interior is read and overwritten.
    One live instance per process (the reference keeps one global solver)."""

    _live = False

    def __init__(self, nx, ny, nz, dx, dy, dzf_global, bctype=("PP", "PP", "NN"), nparts=0):
        L = lib()
        if PoissonSolver._live:
            raise PowerLLELError("one PoissonSolver per process (the reference's solver is a global)")
        _check(L.pl_set_trid_partitions(int(nparts)), "pl_set_trid_partitions")
        self._dzf = np.ascontiguousarray(dzf_global, dtype=np.float64)
        if self._dzf.shape != (nz + 2,):
            raise PowerLLELError("dzf_global must have nz+2 entries (mod_mesh.f90:35)")
        nb = (C.c_int * 18)(*([-2] * 18))  # one rank: every neighbour is MPI_PROC_NULL
        L.init_poisson_solver(nx, ny, nz, dx, dy, _ptr(self._dzf), bctype[0].encode(), bctype[1].encode(),
                              bctype[2].encode(), nb)
        self.shape = (nz + 2, ny + 2, nx + 2)
        PoissonSolver._live = True

    def execute(self, var: np.ndarray) -> None:
        if var.shape != self.shape:
            raise PowerLLELError(f"var must have shape {self.shape}")
        lib().execute_poisson_solver(_ptr(var))

    def free(self) -> None:
        if PoissonSolver._live:
            lib().free_poisson_solver()
            PoissonSolver._live = False

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.free()


def _device_array_ptr(t, n: int, fp64: bool) -> int:
    """The device address of a torch tensor handed to the solver, after the
    checks the C ABI cannot make: a CUDA tensor of n contiguous values of the
    plan's precision (float64 for PL_FP64, float32 for PL_MIXED).  A smaller
    or wider array would be read past its end."""
    want = "torch.float64" if fp64 else "torch.float32"
    if not getattr(t, "is_cuda", False):
        raise PowerLLELError("solve: the array must be a CUDA tensor")
    if str(t.dtype) != want:
        raise PowerLLELError(f"solve: the array is {t.dtype}, the plan needs {want}")
    if not t.is_contiguous() or t.numel() != n:
        raise PowerLLELError(f"solve: the array must be {n} contiguous values (nx*ny*nz)")
    return t.data_ptr()


class DevicePoissonSolver:
    """The PPE on a device array ([k][j][i], nx*ny*nz, float64 for PL_FP64,
    float32 for PL_MIXED).  ``solve`` takes a device pointer (int) or any
    object with ``data_ptr()`` (a torch CUDA tensor)."""

    def __init__(self, nx, ny, nz, dx, dy, dzf_global, nparts=0, precision=PL_FP64):
        L = lib()
        self._dzf = np.ascontiguousarray(dzf_global, dtype=np.float64)
        h = C.c_void_p()
        _check(L.pl_ppe_create(C.byref(h), nx, ny, nz, dx, dy, _ptr(self._dzf), int(nparts), int(precision)),
               "pl_ppe_create")
        self._h = h
        self.n = (nx, ny, nz)
        self.precision = precision

    def solve(self, d_var, stream=None) -> None:
        if hasattr(d_var, "data_ptr"):
            ptr = _device_array_ptr(d_var, self.n[0] * self.n[1] * self.n[2], self.precision == PL_FP64)
        else:
            ptr = int(d_var)
        st = None
        if stream is not None:
            st = C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))
        _check(lib().pl_ppe_solve(self._h, C.c_void_p(ptr), st), "pl_ppe_solve")

    def close(self):
        if self._h:
            lib().pl_ppe_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ----------------------------------------------------------------------------
# Whole time step
# ----------------------------------------------------------------------------
@dataclass
class ChannelConfig:
    """The reference's run parameters (mod_parameters.f90 namelists MESH,
    TIME, PHYSICAL, FORCE) for the channel: x, y periodic, z walls."""
    nx: int
    ny: int
    nz: int
    lx: float = 2 * math.pi
    ly: float = math.pi
    lz: float = 2.0
    mesh_type: int = 1
    stretch_func: int = 0
    stretch_ratio: float = 1.5
    re: float | None = None
    re_tau: float = 180.0
    u_ref: float = 1.0
    l_ref: float = 1.0
    dt: float = 1e-4
    u_crf: float = 0.0
    is_forced: tuple = (True, False, False)
    vel_force: tuple = (1.0, 0.0, 0.0)
    trid_parts: int = 0
    precision: int = PL_FP64

    def to_c(self) -> _Config:
        re = self.re if self.re is not None else re_from_retau(self.re_tau)
        c = _Config()
        c.nx, c.ny, c.nz = self.nx, self.ny, self.nz
        c.lx, c.ly, c.lz = self.lx, self.ly, self.lz
        c.mesh_type, c.stretch_func, c.stretch_ratio = self.mesh_type, self.stretch_func, self.stretch_ratio
        c.re, c.u_ref, c.l_ref, c.dt, c.u_crf = re, self.u_ref, self.l_ref, self.dt, self.u_crf
        c.is_forced = (C.c_int * 3)(*[int(bool(x)) for x in self.is_forced])
        c.vel_force = (C.c_double * 3)(*self.vel_force)
        c.trid_parts, c.precision = self.trid_parts, self.precision
        return c


class Channel:
    """Device-resident channel flow; ``step(n)`` runs n RK2 projection steps
    (main.f90:137-208) on the library's CUDA stream."""

    FIELD_U, FIELD_V, FIELD_W, FIELD_P = 0, 1, 2, 3

    def __init__(self, cfg: ChannelConfig):
        L = lib()
        self.cfg = cfg
        self._c = cfg.to_c()
        h = C.c_void_p()
        _check(L.pl_channel_create(C.byref(h), C.byref(self._c)), "pl_channel_create")
        self._h = h
        self.ghost_shape = (cfg.nz + 2, cfg.ny + 2, cfg.nx + 2)
        self.compact_elems = cfg.nx * cfg.ny * (cfg.nz + 2)

    def init_flow(self, seed: int, noise: float) -> None:
        _check(lib().pl_channel_init_flow(self._h, C.c_uint64(seed), noise), "pl_channel_init_flow")

    def step(self, nsteps: int = 1) -> None:
        _check(lib().pl_channel_step(self._h, int(nsteps)), "pl_channel_step")

    def phase(self, name: str) -> None:
        _check(getattr(lib(), "pl_phase_" + name)(self._h), "pl_phase_" + name)

    def synchronize(self) -> None:
        _check(lib().pl_channel_synchronize(self._h), "pl_channel_synchronize")

    def diagnostics(self) -> dict:
        d = Diag()
        _check(lib().pl_channel_diagnostics(self._h, C.byref(d)), "pl_channel_diagnostics")
        return d.as_dict()

    def get_fields(self):
        """(u, v, w, p) in the reference's ghosted layout, float64."""
        out = [np.zeros(self.ghost_shape) for _ in range(4)]
        _check(lib().pl_channel_get_fields(self._h, *[_ptr(a) for a in out]), "pl_channel_get_fields")
        return tuple(out)

    def get_field(self, which: int) -> np.ndarray:
        """One field (0..2 u,v,w; 3 p; 4..6 stage-1 u1,v1,w1) in the ghosted layout."""
        out = np.zeros(self.ghost_shape)
        _check(lib().pl_channel_get_field(self._h, int(which), _ptr(out)), "pl_channel_get_field")
        return out

    def set_fields(self, u, v, w) -> None:
        _check(lib().pl_channel_set_fields(self._h, _ptr(u), _ptr(v), _ptr(w)), "pl_channel_set_fields")

    def upload_compact(self, host_ptr: int) -> None:
        _check(lib().pl_channel_upload_compact(self._h, C.c_void_p(host_ptr)), "pl_channel_upload_compact")

    def download_compact(self, host_ptr: int) -> None:
        _check(lib().pl_channel_download_compact(self._h, C.c_void_p(host_ptr)), "pl_channel_download_compact")

    def set_body_force(self, f) -> None:
        """Uniform body force added to both RK stages (FP64 path)."""
        fa = np.ascontiguousarray(f, dtype=np.float64)
        _check(lib().pl_channel_set_body_force(self._h, _ptr(fa)), "pl_channel_set_body_force")

    def kinetic_energy(self) -> float:
        ke = np.zeros(1)
        _check(lib().pl_channel_kinetic_energy(self._h, _ptr(ke)), "pl_channel_kinetic_energy")
        return float(ke[0])

    def adjoint_ke_gradient(self, nsteps: int, every: int, d_gu, d_gv, d_gw):
        """Gradient of the kinetic energy after nsteps steps (hand-written
        adjoint, checkpoint every `every` steps) w.r.t. the current fields and
        the body force. d_g*: nx*ny*(nz+2) doubles on the device, as CUDA
        tensors (checked) or device addresses. Returns (J, dJ/df)."""
        ke = np.zeros(1)
        gf = np.zeros(3)
        g = [_device_array_ptr(a, self.compact_elems, True) if hasattr(a, "data_ptr") else int(a)
             for a in (d_gu, d_gv, d_gw)]
        _check(lib().pl_adjoint_ke_gradient(self._h, int(nsteps), int(every), _ptr(ke), C.c_void_p(g[0]),
                                            C.c_void_p(g[1]), C.c_void_p(g[2]), _ptr(gf)), "pl_adjoint_ke_gradient")
        return float(ke[0]), gf

    # statistics (mod_statistics.f90) -------------------------------------
    STAT_NAMES = ("u", "v", "w", "u2", "v2", "w2", "uv", "uw", "vw", "p", "p2")

    def stat_enable(self, names=STAT_NAMES, nt_init_stat: int = 0, sample_interval: int = 1) -> None:
        mask = 0
        for n in names:
            mask |= 1 << self.STAT_NAMES.index(n)
        _check(lib().pl_stat_enable(self._h, mask, int(nt_init_stat), int(sample_interval)), "pl_stat_enable")

    def stat_sample(self, nt: int) -> None:
        _check(lib().pl_stat_sample(self._h, int(nt)), "pl_stat_sample")

    def stat_info(self):
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        _check(lib().pl_stat_info(self._h, C.byref(a), C.byref(b), C.byref(c)), "pl_stat_info")
        return a.value, b.value, c.value

    def stat_get(self, name: str) -> np.ndarray:
        out = np.zeros((self.cfg.nz, self.cfg.ny, self.cfg.nx))
        _check(lib().pl_stat_get(self._h, self.STAT_NAMES.index(name), _ptr(out)), "pl_stat_get")
        return out

    def stat_disable(self) -> None:
        _check(lib().pl_stat_disable(self._h), "pl_stat_disable")

    # monitors (mod_monitor.f90) ------------------------------------------
    def skin_friction(self, wall: int):
        ut, cf = np.zeros(1), np.zeros(1)
        _check(lib().pl_monitor_skin_friction(self._h, int(wall), _ptr(ut), _ptr(cf)), "pl_monitor_skin_friction")
        return float(ut[0]), float(cf[0])

    def forcing_means(self) -> np.ndarray:
        out = np.zeros(3)
        _check(lib().pl_monitor_forcing(self._h, _ptr(out)), "pl_monitor_forcing")
        return out

    def probe(self, i: int, j: int, k: int) -> np.ndarray:
        out = np.zeros(4)
        _check(lib().pl_monitor_probe(self._h, int(i), int(j), int(k), _ptr(out)), "pl_monitor_probe")
        return out

    def region(self, ijk):
        """cell-centred (u, v, w, p) over ijk = (i0, i1, j0, j1, k0, k1), 1-based inclusive, clipped"""
        c = self.cfg
        i0, i1 = max(ijk[0], 1), min(ijk[1], c.nx)
        j0, j1 = max(ijk[2], 1), min(ijk[3], c.ny)
        k0, k1 = max(ijk[4], 1), min(ijk[5], c.nz)
        out = np.zeros((4, max(k1 - k0 + 1, 0), max(j1 - j0 + 1, 0), max(i1 - i0 + 1, 0)))
        arr = (C.c_int * 6)(*[int(x) for x in ijk])
        _check(lib().pl_monitor_region(self._h, arr, _ptr(out)), "pl_monitor_region")
        return out

    def field_ptr(self, which: int) -> int:
        return lib().pl_channel_field(self._h, which)

    def profile(self, nsteps: int = 3) -> list:
        """[(kernel, mean ms per step)] from CUDA events between launches."""
        ms = np.zeros(64)
        names = C.create_string_buffer(64 * 32)
        n = lib().pl_channel_profile(self._h, int(nsteps), _ptr(ms), names, 64)
        _check(0 if n >= 0 else -1, "pl_channel_profile")
        raw = names.raw
        return [(raw[32 * q:32 * q + 32].split(b"\0")[0].decode(), float(ms[q])) for q in range(n)]

    @property
    def stream_handle(self) -> int:
        return lib().pl_channel_stream(self._h) or 0

    def close(self):
        if self._h:
            lib().pl_channel_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
