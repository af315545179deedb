"""CPU tests of the library's host logic: the tridiagonal tables of
trid_tables.h (shared with the CUDA code) replayed with the kernels' column
algorithm must reproduce the reference's golden PPE outputs; the half-complex
transforms are taken from numpy here, so this isolates the table logic."""
import ctypes as C
import glob
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

_lib = None


def host_lib():
    global _lib
    if _lib is None:
        d = tempfile.mkdtemp(prefix="host_trid_")
        so = os.path.join(d, "libhost_trid.so")
        subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-ffp-contract=off", "-o", so,
                        os.path.join(ROOT, "tests", "host_trid.cpp")], check=True)
        _lib = C.CDLL(so)
        _lib.host_trid_solve.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                         C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_double)]
        _lib.host_trid_solve_twisted.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                                 C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int]
    return _lib


def r2hc(x, axis):
    n = x.shape[axis]
    X = np.fft.rfft(x, axis=axis)
    out = np.empty_like(x)
    idx = [slice(None)] * x.ndim
    for k in range(n // 2 + 1):
        idx[axis] = k
        out[tuple(idx)] = X.take(k, axis=axis).real
    for k in range(1, (n + 1) // 2):
        idx[axis] = n - k
        out[tuple(idx)] = X.take(k, axis=axis).imag
    return out


def hc2r(h, axis):
    n = h.shape[axis]
    X = np.zeros(h.shape[:axis] + (n // 2 + 1,) + h.shape[axis + 1:], dtype=complex)
    idx = [slice(None)] * h.ndim
    for k in range(n // 2 + 1):
        idx[axis] = k
        re = h[tuple(idx)]
        im = 0.0
        if 0 < k < n - k:
            j2 = list(idx)
            j2[axis] = n - k
            im = h[tuple(j2)]
        X[tuple(idx)] = re + 1j * im
    return np.fft.irfft(X, n=n, axis=axis) * n


GOLDEN_PPE = sorted(glob.glob(os.path.join(GOLDEN, "ppe_*.npz")))


@pytest.mark.parametrize("path", GOLDEN_PPE, ids=[os.path.basename(p)[:-4] for p in GOLDEN_PPE])
def test_trid_tables_reproduce_reference(path):
    d = np.load(path)
    nx, ny, nz = int(d["nx"]), int(d["ny"]), int(d["nz"])
    nparts = int(d["p_col"]) if int(d["pdd"]) else 0
    x = np.ascontiguousarray(r2hc(r2hc(d["rhs"], 2), 1))
    dzf = np.ascontiguousarray(d["dzf"])
    host_lib().host_trid_solve(nx, ny, nz, float(d["dx"]), float(d["dy"]), dzf.ctypes.data_as(C.POINTER(C.c_double)),
                               nparts, x.ctypes.data_as(C.POINTER(C.c_double)))
    p = hc2r(hc2r(x, 1), 2) / (nx * ny)
    ref = d["p"]
    err = np.abs((p - p.mean()) - (ref - ref.mean())).max() / np.abs(ref - ref.mean()).max()
    assert err < 1e-12, err


GOLDEN_THOMAS = [p for p in GOLDEN_PPE if not int(np.load(p)["pdd"]) and int(np.load(p)["nz"]) % 2 == 0]


@pytest.mark.parametrize("path", GOLDEN_THOMAS, ids=[os.path.basename(p)[:-4] for p in GOLDEN_THOMAS])
def test_twisted_sweep_matches_reference_thomas(path):
    """The mixed path's two-ended sweep (k_thomas_th's column algorithm, its
    tables from the same builder) against the reference's own Thomas solve:
    the same solution up to rounding, modulo the Neumann null mode's constant
    (its gauge is x_p = 0 at the middle row instead of the reference's
    round-off division)."""
    d = np.load(path)
    nx, ny, nz = int(d["nx"]), int(d["ny"]), int(d["nz"])
    x = np.ascontiguousarray(r2hc(r2hc(d["rhs"], 2), 1))
    dzf = np.ascontiguousarray(d["dzf"])
    rc = host_lib().host_trid_solve_twisted(nx, ny, nz, float(d["dx"]), float(d["dy"]),
                                            dzf.ctypes.data_as(C.POINTER(C.c_double)),
                                            x.ctypes.data_as(C.POINTER(C.c_double)), 0)
    assert rc == 0
    p = hc2r(hc2r(x, 1), 2) / (nx * ny)
    ref = d["p"]
    err = np.abs((p - p.mean()) - (ref - ref.mean())).max() / np.abs(ref - ref.mean()).max()
    assert err < 1e-12, err


@pytest.mark.parametrize("path", GOLDEN_THOMAS, ids=[os.path.basename(p)[:-4] for p in GOLDEN_THOMAS])
def test_twisted_sweep_fp32_kept_values(path):
    """k_thomas_th2 keeps the forward-swept values for the backward pass in
    FP32 (one tensor-memory cell per row), the recurrences in FP64: against
    the reference's Thomas solve the error stays below FP32's unit roundoff
    (measured 1.0e-8 to 1.7e-8 on these cases), the size of the rounding of
    the mixed path's FP32 result itself."""
    d = np.load(path)
    nx, ny, nz = int(d["nx"]), int(d["ny"]), int(d["nz"])
    x = np.ascontiguousarray(r2hc(r2hc(d["rhs"], 2), 1))
    dzf = np.ascontiguousarray(d["dzf"])
    rc = host_lib().host_trid_solve_twisted(nx, ny, nz, float(d["dx"]), float(d["dy"]),
                                            dzf.ctypes.data_as(C.POINTER(C.c_double)),
                                            x.ctypes.data_as(C.POINTER(C.c_double)), 1)
    assert rc == 0
    p = hc2r(hc2r(x, 1), 2) / (nx * ny)
    ref = d["p"]
    err = np.abs((p - p.mean()) - (ref - ref.mean())).max() / np.abs(ref - ref.mean()).max()
    assert 0.0 < err < 1e-7, err


def _pair_row(b, ny):
    """trid_pair_row (ppe.cu): processing row b -> plane row py, mirror rows adjacent"""
    if b == 0:
        return 0
    if b == ny - 1:
        return ny // 2
    jy = (b + 1) // 2
    return jy if b & 1 else ny - jy


@pytest.mark.parametrize("nx,ny", [(128, 24), (256, 256), (384, 192), (512, 384), (768, 32), (1024, 768)])
def test_thomas_th2_class_windows(nx, ny):
    """Index arithmetic of k_thomas_th2's cooperative copies (nx % 128 == 0):
    the processing rows visit every plane row once; a round's 128 columns are
    one run px0 .. px0+127 of plane row py, whose eigenvalue classes
    min(px, nx-px) + ncx min(py, ny-py) all lie in the window of 130 table
    values that starts at the even cbase; the window's 65 16-byte copies of
    every swept row (rows < nz) stay inside the tables' nz + 2 rows of tcs
    values."""
    ncx, ncy = nx // 2 + 1, ny // 2 + 1
    ncls = ncx * ncy
    tcs = (ncls + 1) // 2 * 2
    assert sorted(_pair_row(b, ny) for b in range(ny)) == list(range(ny))
    for b in range(ny):
        py = _pair_row(b, ny)
        jy = min(py, ny - py)
        for px0 in range(0, nx, 128):
            ixmin = min(px0, nx - px0 - 127)
            cbase = (ixmin + ncx * jy) & ~1
            offs = [min(px, nx - px) + ncx * jy - cbase for px in range(px0, px0 + 128)]
            assert cbase % 2 == 0 and min(offs) >= 0 and max(offs) < 130, (b, px0, min(offs), max(offs))
            # last value read of a swept row k <= nz-1, against the table's end
            for nz in (16, 256):
                assert (nz - 1) * tcs + cbase + 129 < (nz + 2) * tcs
