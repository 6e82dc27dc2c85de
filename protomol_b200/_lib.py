"""ctypes binding of libpmgpu.so (the C ABI declared in include/pmgpu.h).

The shared library is built in-tree by ``__graft_entry__.build()`` (or
``make -C protomol_b200/csrc``).  There is no fallback: if the library is
missing or fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpmgpu.so")

# status codes (pmgpu.h)
OK, ERR_ARG, ERR_CUDA, ERR_OOM, ERR_OVERFLOW, ERR_NAN, ERR_UNSUPPORTED, ERR_STATE = range(8)
EXCL_NONE, EXCL_MODIFIED, EXCL_FULL = 0, 1, 2
SW_UNIVERSAL, SW_CUTOFF, SW_C1, SW_C2, SW_CN, SW_CMPCNCN = range(6)
SW_COMPLEMENT = 16  # flag on C1 / C2 / Cn
E_COULOMB, E_LENNARDJONES, E_BOND, E_ANGLE, E_DIHEDRAL, E_IMPROPER, E_OTHER = range(7)
E_COUNT = 7
PREC_MIXED, PREC_DOUBLE = 0, 1
EWALD_REAL, EWALD_RECIPROCAL, EWALD_CORRECTION, EWALD_ALL = 1, 2, 4, 7
INT_LEAPFROG, INT_LANGEVIN_LEAPFROG = 0, 1
FORCE_SCALE = 4294967296.0
GB_STATIC_MAX_ATOMS = 16384

EXPORTED = [
    "pmgpu_context_create", "pmgpu_context_destroy", "pmgpu_last_error",
    "pmgpu_abi_version", "pmgpu_system_create", "pmgpu_system_destroy",
    "pmgpu_system_set_positions", "pmgpu_system_get_positions",
    "pmgpu_system_set_velocities", "pmgpu_system_get_velocities",
    "pmgpu_system_get_forces", "pmgpu_system_get_energies", "pmgpu_system_stream",
    "pmgpu_system_device_state", "pmgpu_force_cutoff_add", "pmgpu_force_simplefull_add",
    "pmgpu_force_pme_add", "pmgpu_force_gb_add", "pmgpu_force_bonded_add",
    "pmgpu_force_set_enabled", "pmgpu_evaluate", "pmgpu_force_evaluate", "pmgpu_run",
    "pmgpu_set_count_pairs", "pmgpu_force_stats", "pmgpu_debug_cell_assign",
    "pmgpu_debug_pair_set", "pmgpu_profile_enable", "pmgpu_profile_read",
    "pmgpu_kernel_count", "pmgpu_gb_forces_noalloc", "pmgpu_run_async", "pmgpu_run_query",
    "pmgpu_run_wait", "pmgpu_mem_info", "pmgpu_footprint_estimate", "pmgpu_force_torsion_add",
    "pmgpu_fp32_peak", "pmgpu_force_gbace_add", "pmgpu_debug_set_list_capacity",
    "pmgpu_ensemble_create", "pmgpu_ensemble_destroy", "pmgpu_ensemble_run",
    "pmgpu_ensemble_set_splits", "pmgpu_ensemble_time_pairs", "pmgpu_ensemble_get_info",
    "pmgpu_ensemble_member", "pmgpu_debug_limit_list_rows", "pmgpu_system_set_step",
    "pmgpu_force_full_add", "pmgpu_force_simplefull_switched_add", "pmgpu_force_scpism_add",
    "pmgpu_force_born_add", "pmgpu_debug_set_column_capacity", "pmgpu_run_discard",
]
PHASES = ["list", "pairs", "pme", "correction", "bonded", "gb", "simplefull", "integrate"]


class EnsembleInfo(C.Structure):
    _fields_ = [("members", C.c_int), ("fft_buckets", C.c_int), ("kernels", C.c_longlong),
                ("graph_replays", C.c_longlong), ("steps", C.c_longlong)]


class PmgpuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"pmgpu error {code}: {msg}")
        self.code = code


class Topology(C.Structure):
    _fields_ = [
        ("n_atoms", C.c_int), ("charge", C.c_void_p), ("mass", C.c_void_p),
        ("type", C.c_void_p), ("molecule", C.c_void_p), ("n_types", C.c_int),
        ("lj", C.c_void_p), ("n_exclusions", C.c_int), ("exclusions", C.c_void_p),
        ("exclusion_table_class", C.c_void_p),
        ("coulomb_scaling", C.c_double), ("periodic", C.c_int), ("box", C.c_double * 12),
        ("n_bonds", C.c_int), ("bond_atoms", C.c_void_p), ("bond_params", C.c_void_p),
        ("n_angles", C.c_int), ("angle_atoms", C.c_void_p), ("angle_params", C.c_void_p),
        ("gb_vdwr", C.c_void_p), ("gb_scale", C.c_void_p), ("gb_offset", C.c_void_p),
        ("water", C.c_void_p), ("gb_obc", C.c_double * 3),
        ("n_dihedrals", C.c_int), ("dihedral_atoms", C.c_void_p), ("dihedral_params", C.c_void_p),
        ("n_impropers", C.c_int), ("improper_atoms", C.c_void_p), ("improper_params", C.c_void_p),
        ("scpism_sqrtalpha", C.c_void_p), ("scpism_alpha", C.c_void_p),
        ("scpism_zeta", C.c_void_p), ("scpism_eta", C.c_void_p), ("scpism_c", C.c_void_p),
        ("scpism_g", C.c_void_p), ("scpism_hbond", C.c_void_p),
        ("scpism_residue", C.c_void_p), ("scpism_name", C.c_void_p),
    ]


class Switch(C.Structure):
    _fields_ = [("kind", C.c_int), ("cutoff", C.c_double), ("switchon", C.c_double),
                ("switchoff", C.c_double), ("order", C.c_double)]


class Integrator(C.Structure):
    _fields_ = [("kind", C.c_int), ("timestep_fs", C.c_double), ("temperature", C.c_double),
                ("gamma_ps", C.c_double), ("seed", C.c_uint64)]


class Stats(C.Structure):
    _fields_ = [("pairs_in_cutoff", C.c_longlong), ("list_entries", C.c_longlong),
                ("clusters", C.c_longlong), ("list_builds", C.c_longlong),
                ("cells", C.c_int * 3), ("pair_kernel", C.c_int), ("list_capacity", C.c_int)]


_lib = None


def load() -> C.CDLL:
    """Load libpmgpu.so; raises if it is absent (no CPU fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    # PMGPU_LIB: another build of the same library (for comparing builds)
    path = os.environ.get("PMGPU_LIB", LIB_PATH)
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with __graft_entry__.build() "
                          "or `make -C protomol_b200/csrc`")
    lib = C.CDLL(path)
    vp, i32, dbl = C.c_void_p, C.c_int, C.c_double
    lib.pmgpu_last_error.restype = C.c_char_p
    lib.pmgpu_system_stream.restype = vp
    lib.pmgpu_system_stream.argtypes = [vp]
    for name in EXPORTED:
        getattr(lib, name)  # every declared symbol must resolve
    lib.pmgpu_context_create.argtypes = [i32, C.POINTER(vp)]
    lib.pmgpu_context_destroy.argtypes = [vp]
    lib.pmgpu_system_create.argtypes = [vp, C.POINTER(Topology), i32, C.POINTER(vp)]
    lib.pmgpu_system_destroy.argtypes = [vp]
    for n in ("set_positions", "get_positions", "set_velocities", "get_velocities",
              "get_forces"):
        getattr(lib, "pmgpu_system_" + n).argtypes = [vp, vp]
    lib.pmgpu_system_get_energies.argtypes = [vp, vp, vp]
    lib.pmgpu_system_device_state.argtypes = [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]
    lib.pmgpu_force_cutoff_add.argtypes = [vp, C.POINTER(Switch), C.POINTER(Switch), dbl, dbl,
                                           C.POINTER(i32)]
    lib.pmgpu_force_simplefull_add.argtypes = [vp, i32, i32, C.POINTER(i32)]
    lib.pmgpu_force_full_add.argtypes = [vp, C.POINTER(Switch), C.POINTER(Switch), dbl, dbl,
                                         C.POINTER(i32)]
    lib.pmgpu_force_simplefull_switched_add.argtypes = [vp, C.POINTER(Switch), C.POINTER(Switch),
                                                        C.POINTER(i32)]
    lib.pmgpu_force_scpism_add.argtypes = [vp, C.POINTER(Switch), C.POINTER(Switch), dbl,
                                           C.POINTER(i32)]
    lib.pmgpu_force_born_add.argtypes = [vp, i32, dbl, i32, dbl, dbl, C.POINTER(i32)]
    lib.pmgpu_force_pme_add.argtypes = [vp, dbl, dbl, i32, vp, i32, i32, dbl, C.POINTER(i32)]
    lib.pmgpu_force_gb_add.argtypes = [vp, dbl, dbl, C.POINTER(i32)]
    lib.pmgpu_force_gbace_add.argtypes = [vp, dbl, dbl, C.POINTER(i32)]
    lib.pmgpu_force_bonded_add.argtypes = [vp, i32, i32, C.POINTER(i32)]
    lib.pmgpu_force_torsion_add.argtypes = [vp, i32, i32, C.POINTER(i32)]
    lib.pmgpu_force_set_enabled.argtypes = [vp, i32, i32]
    lib.pmgpu_evaluate.argtypes = [vp, vp, vp]
    lib.pmgpu_force_evaluate.argtypes = [vp, i32, vp, vp, vp, vp]
    lib.pmgpu_run.argtypes = [vp, C.POINTER(Integrator), C.c_long]
    lib.pmgpu_set_count_pairs.argtypes = [vp, i32]
    lib.pmgpu_force_stats.argtypes = [vp, i32, C.POINTER(Stats)]
    lib.pmgpu_debug_cell_assign.argtypes = [vp, dbl, vp, vp]
    lib.pmgpu_debug_pair_set.argtypes = [vp, i32, vp, C.c_longlong, C.POINTER(C.c_longlong)]
    lib.pmgpu_debug_set_list_capacity.argtypes = [vp, i32]
    lib.pmgpu_debug_limit_list_rows.argtypes = [vp, i32]
    lib.pmgpu_debug_set_column_capacity.argtypes = [vp, i32]
    lib.pmgpu_system_set_step.argtypes = [vp, C.c_longlong]
    lib.pmgpu_profile_enable.argtypes = [vp, i32]
    lib.pmgpu_profile_read.argtypes = [vp, vp, vp, i32]
    lib.pmgpu_kernel_count.argtypes = [vp, C.POINTER(C.c_longlong)]
    lib.pmgpu_run_async.argtypes = [vp, C.POINTER(Integrator), C.c_long]
    lib.pmgpu_run_query.argtypes = [vp, C.POINTER(i32)]
    lib.pmgpu_run_wait.argtypes = [vp]
    lib.pmgpu_run_discard.argtypes = [vp]
    lib.pmgpu_mem_info.argtypes = [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
    lib.pmgpu_fp32_peak.argtypes = [vp, C.POINTER(C.c_double)]
    lib.pmgpu_footprint_estimate.argtypes = [i32, vp, dbl, vp, C.POINTER(C.c_longlong)]
    lib.pmgpu_gb_forces_noalloc.argtypes = [i32, vp, vp, vp, vp, vp, vp, C.POINTER(dbl),
                                            dbl, dbl, i32, vp, vp, vp]
    lib.pmgpu_ensemble_create.argtypes = [vp, i32, C.POINTER(vp)]
    lib.pmgpu_ensemble_destroy.argtypes = [vp]
    lib.pmgpu_ensemble_run.argtypes = [vp, C.POINTER(Integrator), C.c_long]
    lib.pmgpu_ensemble_set_splits.argtypes = [vp, vp]
    lib.pmgpu_ensemble_time_pairs.argtypes = [vp, vp, i32, C.POINTER(dbl)]
    lib.pmgpu_ensemble_get_info.argtypes = [vp, C.POINTER(EnsembleInfo)]
    lib.pmgpu_ensemble_member.argtypes = [vp, i32, C.POINTER(i32), C.POINTER(i32)]
    _lib = lib
    return lib


def check(code: int) -> None:
    if code != OK:
        msg = load().pmgpu_last_error().decode(errors="replace")
        raise PmgpuError(code, msg)


def ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)
