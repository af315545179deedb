"""CPU tests of the drop-in boundary: the C-ABI library builds, loads without a
GPU and exports every function include/*.h declares; the Python host layer
validates arguments before any device call.  No compute call runs here."""
import ctypes as C
import glob
import os
import re
import subprocess

import pytest

from conftest import ROOT


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        for m in re.finditer(r"^\s*(?:extern\s+)?[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", src, flags=re.M):
            name = m.group(1)
            if name not in ("if", "while", "for", "return", "sizeof", "typedef"):
                names.append(name)
    return sorted(set(names))


def test_header_declares_reference_interface():
    names = declared_functions()
    for n in ("init_poisson_solver", "execute_poisson_solver", "free_poisson_solver"):
        assert n in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    import powerllel_channel_b200 as plb
    from powerllel_channel_b200 import build as B
    B.build()
    lib = C.CDLL(plb.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", plb.LIB_PATH], capture_output=True, text=True).stdout
    for n in declared_functions():
        assert re.search(rf"\sT {n}$", out, flags=re.M), n


def test_library_is_sm100a():
    import powerllel_channel_b200 as plb
    out = subprocess.run(["cuobjdump", "--list-elf", plb.LIB_PATH], capture_output=True, text=True).stdout
    assert "sm_100a" in out


def test_reference_signatures_match():
    """The drop-in keeps the reference's prototypes (mod_poisson_solver.c:178-181,
    468, 607): same parameter lists, void results."""
    src = open(os.path.join(ROOT, "include", "powerllel_b200.h")).read()
    flat = " ".join(src.split())
    assert ("void init_poisson_solver(int nx_global, int ny_global, int nz_global, double dx, double dy, "
            "double *dzf_global, char bctype_x[], char bctype_y[], char bctype_z[], int neighbor_xyz[3][6]);") in flat
    assert "void execute_poisson_solver(double *var);" in flat
    assert "void free_poisson_solver(void);" in flat


def test_host_layer_rejects_bad_arrays():
    import numpy as np
    import powerllel_channel_b200 as plb
    with pytest.raises(plb.PowerLLELError):
        plb._ptr(np.zeros(4, dtype=np.float32))
    with pytest.raises(plb.PowerLLELError):
        plb._ptr(np.zeros((4, 4))[:, ::2])


def test_ppe_solve_rejects_misaligned_array():
    """pl_ppe_solve and pl_ppe_solve_noalloc reject a device array that does
    not start on a boundary of two elements before they read the plan or
    launch anything (neither address below is dereferenced), so the check
    runs without a GPU."""
    import powerllel_channel_b200 as plb
    from powerllel_channel_b200 import build as B
    B.build()
    lib = C.CDLL(plb.LIB_PATH)
    lib.pl_last_error.restype = C.c_char_p
    for fn in (lib.pl_ppe_solve, lib.pl_ppe_solve_noalloc):
        fn.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        fn.restype = C.c_int
        assert fn(C.c_void_p(0x1000), C.c_void_p(0x2004), None) != 0
        assert b"aligned to 8 bytes" in lib.pl_last_error()


def test_package_has_no_oracle_dependency():
    """The product never imports, links or runs the oracle."""
    pkg = os.path.join(ROOT, "powerllel_channel_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".h", ".cpp")):
                txt = open(os.path.join(dirpath, f)).read()
                assert "oracle" not in txt.lower().replace("no oracle", ""), f


def test_host_layer_checks_solver_tensors():
    """DevicePoissonSolver.solve checks a torch tensor before its address
    crosses the C ABI: device, dtype of the plan's precision, contiguity and
    size (nx*ny*nz values); the CUDA-only case is checked on CPU with a
    stand-in that reports a CUDA tensor."""
    import torch
    import powerllel_channel_b200 as plb

    class Fake:
        def __init__(self, t):
            self.t, self.is_cuda, self.dtype = t, True, t.dtype

        def is_contiguous(self):
            return self.t.is_contiguous()

        def numel(self):
            return self.t.numel()

        def data_ptr(self):
            return 0x1000

    with pytest.raises(plb.PowerLLELError, match="CUDA tensor"):
        plb._device_array_ptr(torch.zeros(8, dtype=torch.float64), 8, True)
    with pytest.raises(plb.PowerLLELError, match="needs torch.float64"):
        plb._device_array_ptr(Fake(torch.zeros(8, dtype=torch.float32)), 8, True)
    with pytest.raises(plb.PowerLLELError, match="needs torch.float32"):
        plb._device_array_ptr(Fake(torch.zeros(8, dtype=torch.float64)), 8, False)
    with pytest.raises(plb.PowerLLELError, match="contiguous"):
        plb._device_array_ptr(Fake(torch.zeros(4, 4)[:, ::2]), 8, False)
    with pytest.raises(plb.PowerLLELError, match="contiguous"):
        plb._device_array_ptr(Fake(torch.zeros(6)), 8, False)
    assert plb._device_array_ptr(Fake(torch.zeros(8)), 8, False) == 0x1000
