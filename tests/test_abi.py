"""The C-ABI library loads without a GPU and exports every entry point that
include/acgpu.h declares; the Python binding declares each of them."""
import ctypes
import re
from pathlib import Path

import pytest

from acgpu import _lib

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    text = (ROOT / "include" / "acgpu.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(acg_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "acg_create" in names and "acg_solve" in names and len(names) >= 15


@pytest.mark.parametrize("name", declared_functions())
def test_symbol_exported(name):
    L = ctypes.CDLL(str(_lib.LIB_PATH))
    assert hasattr(L, name), f"{name} declared in include/acgpu.h but not exported"


def test_binding_covers_header():
    bound = {s[0] for s in _lib.SIGNATURES}
    missing = set(declared_functions()) - bound
    assert not missing, f"not bound in acgpu/_lib.py: {sorted(missing)}"


def test_no_device_is_reported_not_crashed():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    rc = _lib.lib().acg_device_check()
    assert rc == -5  # ACG_ERR_NODEVICE
    assert _lib.lib().acg_last_error()


def test_bad_arguments_are_errors():
    import numpy as np
    L = _lib.lib()
    h = ctypes.c_void_p()
    z = np.zeros(1, np.int64)
    f = np.zeros(1)
    rc = L.acg_create(1, z, z, f, z, z, z, f, f, 0, 1, None, ctypes.byref(h))
    assert rc < 0
    st = np.zeros(4, np.uint64)
    assert L.acg_approxchol(1, z, z, f, st, ctypes.byref(h)) == -1
    # the asynchronous entries reject null handles and requests without a device
    req = ctypes.c_void_p()
    assert L.acg_solve_async(None, None, None, 1, 1, 1e-8, 10, 1.0, 5, 0, ctypes.byref(req)) == -1
    assert L.acg_poll(None) == -1
    assert L.acg_wait(None, None) == -1
    # diagnostics and group entries reject null handles before touching a device
    assert L.acg_time_sweep_levels(None, 1, 64, 1, 0, None, None, None, None, None) == -1
    assert L.acg_solve_group(None, f, f, 1e-8, 10, 1.0, 5, 0, None) == -1
    assert L.acg_time_kernels_batch(None, 1, 64, 1, None) == -1


def _header_struct_fields(tag):
    """Field names, in order, of `typedef struct { ... } tag;` in include/acgpu.h."""
    text = (ROOT / "include" / "acgpu.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    m = re.search(r"typedef struct\s*\{([^}]*)\}\s*" + tag + r"\s*;", text, flags=re.S)
    assert m, tag
    names = []
    for decl in m.group(1).split(";"):
        decl = decl.strip()
        if not decl:
            continue
        decl = re.sub(r"^(const\s+)?(unsigned\s+)?[A-Za-z_0-9]+\s+", "", decl)
        for part in decl.split(","):
            names.append(re.sub(r"\[.*\]", "", part).strip())
    return names


@pytest.mark.parametrize("tag,cls", [("acg_options", "AcgOptions"), ("acg_stats", "AcgStats"),
                                     ("acg_solve_info", "AcgSolveInfo"), ("acg_kernel_times", "AcgKernelTimes")])
def test_binding_structs_match_header(tag, cls):
    """The ctypes mirrors declare the header's fields in the header's order."""
    fields = [f[0] for f in getattr(_lib, cls)._fields_]
    assert fields == _header_struct_fields(tag)


def test_unknown_solver_option_is_rejected():
    """A misspelled tuning knob raises instead of being silently ignored (no device needed)."""
    import acgpu
    from acgpu import generators as G
    a = G.grid2(4)
    acgpu.seed(1)
    ldli = acgpu.approx_chol(a)
    with pytest.raises(ValueError, match="unknown solver option"):
        acgpu.DeviceLapSolver(a, ldli, options=dict(dense_tial=0))
