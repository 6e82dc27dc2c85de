"""protomol_b200: B200-native (sm_100a) implementation of ProtoMol's
nonbonded hot path behind ProtoMol's force-module interface.

The compute lives in ``libpmgpu.so`` (CUDA C++ behind the C ABI in
``include/pmgpu.h``); this package is the host-side mirror of the reference
interface (SystemForce / ForceFactory / Integrator) plus the synthetic
system generators used by the benchmark.
"""
from .engine import (  # noqa: F401
    ANGLE, BOND, COULOMB, LENNARDJONES, VIRIALXX, BondedSystemForce, Context, ForceFactory,
    GBACEForce, GBForce, GpuSystem, LangevinLeapfrogIntegrator, LeapfrogIntegrator,
    NonbondedCutoffSystemForce, NonbondedFullSystemForce, NonbondedSimpleFullSwitchedForce,
    NonbondedSimpleFullSystemForce, PMEwaldSystemForce, ScpismSystemForce, BornSystemForce,
    ScalarStructure, SystemForce, TorsionSystemForce)
from ._lib import PmgpuError, load  # noqa: F401
