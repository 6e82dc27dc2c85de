"""The C-ABI library loads and exports every entry point include/pmgpu.h
declares, and its error convention holds without a GPU: handle-taking
entry points refuse a null handle with PMGPU_ERR_ARG and a message, the
destroy calls accept null, and a context cannot be made without a device
(PMGPU_ERR_CUDA, no fallback).  No device work is started."""
import ctypes
import os
import re

from protomol_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(?:int|void|char)\s*\**\s*(pmgpu_\w+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_lib.EXPORTED) <= names


def test_abi_version_without_device():
    lib = _lib.load()
    assert lib.pmgpu_abi_version() == 2


# entry points whose first argument is a system, ensemble or context handle
# (argument values past it are valid where they are checked first)
HANDLE_CALLS = [
    "pmgpu_run_discard", "pmgpu_run_wait", "pmgpu_run_query", "pmgpu_run", "pmgpu_run_async",
    "pmgpu_debug_set_column_capacity", "pmgpu_debug_set_list_capacity",
    "pmgpu_debug_limit_list_rows", "pmgpu_system_set_step", "pmgpu_system_set_positions",
    "pmgpu_system_get_positions", "pmgpu_system_set_velocities", "pmgpu_system_get_velocities",
    "pmgpu_evaluate", "pmgpu_force_cutoff_add", "pmgpu_force_pme_add", "pmgpu_force_gb_add",
    "pmgpu_force_set_enabled", "pmgpu_force_stats", "pmgpu_kernel_count", "pmgpu_ensemble_run",
]


def _default(t):
    if t in (ctypes.c_int, ctypes.c_long, ctypes.c_longlong, ctypes.c_int32, ctypes.c_int64):
        return t(32)
    if t in (ctypes.c_double, ctypes.c_float):
        return t(8.0)
    return None


def test_null_handles_are_refused_with_a_message():
    lib = _lib.load()
    lib.pmgpu_last_error.restype = ctypes.c_char_p
    for name in HANDLE_CALLS:
        f = getattr(lib, name)
        args = [_default(t) for t in (f.argtypes or [ctypes.c_void_p])]
        assert f(*args) == _lib.ERR_ARG, name
        assert lib.pmgpu_last_error(), name
    for name in ("pmgpu_system_destroy", "pmgpu_context_destroy"):
        assert getattr(lib, name)(None) == _lib.OK, name


def test_no_context_without_a_device():
    import torch
    if torch.cuda.is_available():
        return  # only meaningful on a host without a GPU
    lib = _lib.load()
    lib.pmgpu_last_error.restype = ctypes.c_char_p
    h = ctypes.c_void_p()
    assert lib.pmgpu_context_create(0, ctypes.byref(h)) == _lib.ERR_CUDA
    assert h.value is None and lib.pmgpu_last_error()
