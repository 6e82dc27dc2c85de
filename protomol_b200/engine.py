"""Host-side mirror of ProtoMol's force-module interface over libpmgpu.

ProtoMol names and semantics are kept so the parity tests read like the
reference's own use of the API:

* ``GpuSystem`` -- the device-resident state of one ``GenericTopology``
  (topology arrays, positions, velocities, force accumulators).
* ``SystemForce`` subclasses -- ``evaluate(positions, forces, energies)``
  ADDS into a ``Vector3DBlock``-layout array and a ``ScalarStructure``-layout
  energy array (force/system/SystemForce.h:32-35).
* ``ForceFactory.make(line)`` -- parses a ``.conf`` force line
  (factory/ForceFactory.cpp:21-242) into a GPU force.
* ``LeapfrogIntegrator`` / ``LangevinLeapfrogIntegrator`` -- ``run(n)`` on
  the device (integrator/leapfrog/LeapfrogIntegrator.cpp:89-104,
  integrator/base/LangevinLeapfrogIntegrator.cpp).
"""
from __future__ import annotations

import ctypes as C
import math
import re

import numpy as np

from . import _lib as L

# ScalarStructure::Index (type/ScalarStructure.h:26-67)
COULOMB, LENNARDJONES, BOND, ANGLE, DIHEDRAL, IMPROPER, OTHER = range(7)
VIRIALXX = 7
SCALAR_LAST = 36


# forms of the pair kernel (PMGPU_PAIRK_*)
PAIR_KERNELS = {0: "generic", 1: "lj_c2+ewald", 2: "lj_c2+coulomb_c2", 3: "lj_c2+coulomb_c1"}


def ScalarStructure() -> np.ndarray:
    """A zeroed ScalarStructure-layout energy/virial array."""
    return np.zeros(SCALAR_LAST)


def footprint_estimate(n_atoms: int, box, reach: float, grid=None) -> int:
    """Device bytes a periodic system needs (admission control)."""
    lib = L.load()
    b = np.ascontiguousarray(np.asarray(box, dtype=np.float64)[:3])
    g = None if grid is None else np.ascontiguousarray(np.asarray(grid, dtype=np.int32))
    out = C.c_longlong()
    L.check(lib.pmgpu_footprint_estimate(int(n_atoms), L.ptr(b), float(reach), L.ptr(g),
                                         C.byref(out)))
    return int(out.value)


class Context:
    """One CUDA device."""

    def __init__(self, device: int = 0):
        self.lib = L.load()
        h = C.c_void_p()
        L.check(self.lib.pmgpu_context_create(device, C.byref(h)))
        self.h = h
        self.device = device

    def mem_info(self) -> tuple[int, int]:
        """(free, total) device bytes."""
        f, t = C.c_longlong(), C.c_longlong()
        L.check(self.lib.pmgpu_mem_info(self.h, C.byref(f), C.byref(t)))
        return int(f.value), int(t.value)

    def fp32_peak(self) -> float:
        """Measured FP32 FMA throughput of the device, TFLOP/s."""
        t = C.c_double()
        L.check(self.lib.pmgpu_fp32_peak(self.h, C.byref(t)))
        return float(t.value)

    def close(self):
        if self.h:
            self.lib.pmgpu_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_PREC = {"mixed": L.PREC_MIXED, "double": L.PREC_DOUBLE}


class GpuSystem:
    """Device-resident copy of a topology (a ``MolecularSystem`` or any
    object with the same array attributes) and its dynamic state."""

    def __init__(self, ctx: Context, topo, precision: str = "mixed"):
        self.ctx = ctx
        self.lib = ctx.lib
        self.n = int(np.asarray(topo.pos).shape[0])
        n = self.n
        keep = {}

        def arr(name, a, dt):
            a = np.ascontiguousarray(np.asarray(a), dtype=dt).reshape(-1)
            keep[name] = a
            return a.ctypes.data

        t = L.Topology()
        t.n_atoms = n
        t.charge = arr("charge", topo.charge, np.float64)
        t.mass = arr("mass", topo.mass, np.float64)
        t.type = arr("type", topo.type, np.int32)
        t.molecule = arr("molecule", topo.molecule, np.int32)
        lj = np.asarray(topo.lj)
        t.n_types = int(lj.shape[0])
        t.lj = arr("lj", lj, np.float64)
        ex = np.asarray(topo.exclusions).reshape(-1, 3)
        t.n_exclusions = len(ex)
        t.exclusions = arr("excl", ex, np.int32) if len(ex) else None
        tc = getattr(topo, "exclusion_table_class", None)
        if tc is not None and len(ex):
            t.exclusion_table_class = arr("excl_tc", tc, np.int32)
        t.coulomb_scaling = float(getattr(topo, "coulomb_scaling", 1.0))
        t.periodic = 1 if topo.periodic else 0
        for i in range(12):
            t.box[i] = float(topo.box[i])
        bonds = np.asarray(getattr(topo, "bonds", np.zeros((0, 2)))).reshape(-1, 2)
        t.n_bonds = len(bonds)
        if len(bonds):
            t.bond_atoms = arr("bonds", bonds, np.int32)
            t.bond_params = arr("bondp", topo.bond_params, np.float64)
        angles = np.asarray(getattr(topo, "angles", np.zeros((0, 3)))).reshape(-1, 3)
        t.n_angles = len(angles)
        if len(angles):
            t.angle_atoms = arr("angles", angles, np.int32)
            t.angle_params = arr("anglep", topo.angle_params, np.float64)
        for kind in ("dihedral", "improper"):
            atoms = getattr(topo, kind + "s", None)
            if atoms is not None and len(np.asarray(atoms).reshape(-1)):
                atoms = np.asarray(atoms).reshape(-1, 4)
                setattr(t, "n_" + kind + "s", len(atoms))
                setattr(t, kind + "_atoms", arr(kind + "a", atoms, np.int32))
                setattr(t, kind + "_params",
                        arr(kind + "p", np.asarray(getattr(topo, kind + "_params")).reshape(-1, 3),
                            np.float64))
        if getattr(topo, "gb_vdwr", None) is not None:
            t.gb_vdwr = arr("vdwr", topo.gb_vdwr, np.float64)
            t.gb_scale = arr("scale", topo.gb_scale, np.float64)
            t.gb_offset = arr("offset", topo.gb_offset, np.float64)
            for i in range(3):
                t.gb_obc[i] = float(topo.gb_obc[i])
        if getattr(topo, "water", None) is not None:
            t.water = arr("water", topo.water, np.int32)
        scp = getattr(topo, "scpism", None)
        if scp is not None:
            for key in ("sqrtalpha", "alpha", "zeta", "eta", "c", "g"):
                setattr(t, "scpism_" + key, arr("scp_" + key, scp["scp_" + key], np.float64))
            for key in ("hbond", "residue", "name"):
                setattr(t, "scpism_" + key, arr("scp_" + key, scp["scp_" + key], np.int32))
        h = C.c_void_p()
        L.check(self.lib.pmgpu_system_create(ctx.h, C.byref(t), _PREC[precision], C.byref(h)))
        self.h = h
        self.precision = precision
        self.periodic = bool(topo.periodic)
        self.forces: list[SystemForce] = []
        self.set_positions(topo.pos)
        if getattr(topo, "vel", None) is not None:
            self.set_velocities(topo.vel)

    def close(self):
        if getattr(self, "h", None):
            self.lib.pmgpu_system_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- state
    def _vec(self, a):
        a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1))
        if a.size != 3 * self.n:
            raise ValueError(f"expected {3 * self.n} values, got {a.size}")
        return a

    def set_positions(self, pos):
        a = self._vec(pos)
        L.check(self.lib.pmgpu_system_set_positions(self.h, L.ptr(a)))

    def positions(self) -> np.ndarray:
        out = np.zeros((self.n, 3))
        L.check(self.lib.pmgpu_system_get_positions(self.h, L.ptr(out)))
        return out

    def set_step(self, step: int) -> None:
        """The step counter that keys the Langevin noise (0 for a new
        system)."""
        L.check(self.lib.pmgpu_system_set_step(self.h, int(step)))

    def set_velocities(self, vel):
        a = self._vec(vel)
        L.check(self.lib.pmgpu_system_set_velocities(self.h, L.ptr(a)))

    def velocities(self) -> np.ndarray:
        out = np.zeros((self.n, 3))
        L.check(self.lib.pmgpu_system_get_velocities(self.h, L.ptr(out)))
        return out

    def forces_total(self) -> np.ndarray:
        out = np.zeros((self.n, 3))
        L.check(self.lib.pmgpu_system_get_forces(self.h, L.ptr(out)))
        return out

    def evaluate(self, virial: bool = False):
        """Evaluate all enabled forces at the resident positions; returns
        (energies[7], virial[3,3] or None)."""
        e = np.zeros(L.E_COUNT)
        v = np.zeros(9) if virial else None
        L.check(self.lib.pmgpu_evaluate(self.h, L.ptr(e), L.ptr(v)))
        return e, (v.reshape(3, 3) if v is not None else None)

    def evaluate_forces(self) -> np.ndarray:
        """Force-only evaluation of all enabled forces at the resident
        positions (the kernels of an inner MD step, no energies); returns the
        total force (n, 3)."""
        L.check(self.lib.pmgpu_evaluate(self.h, None, None))
        return self.forces_total()

    def energies(self):
        """(energies[7], virial[3,3]) of the last evaluation or run segment,
        without evaluating again."""
        e = np.zeros(L.E_COUNT)
        v = np.zeros(9)
        L.check(self.lib.pmgpu_system_get_energies(self.h, L.ptr(e), L.ptr(v)))
        return e, v.reshape(3, 3)

    def stream(self) -> int:
        return self.lib.pmgpu_system_stream(self.h)

    def device_state(self):
        p, v, f = C.c_void_p(), C.c_void_p(), C.c_void_p()
        L.check(self.lib.pmgpu_system_device_state(self.h, C.byref(p), C.byref(v), C.byref(f)))
        return p.value, v.value, f.value

    def profile(self, enable: bool | None = None, reset: bool = False) -> dict:
        """Per-phase device time (ms) and launch counts since the last reset
        (CUDA events inside the library); optionally switch profiling."""
        if enable is not None:
            L.check(self.lib.pmgpu_profile_enable(self.h, 1 if enable else 0))
        ms = np.zeros(len(L.PHASES))
        ln = np.zeros(len(L.PHASES), np.int64)
        L.check(self.lib.pmgpu_profile_read(self.h, L.ptr(ms), L.ptr(ln), 1 if reset else 0))
        return {p: (float(ms[k]), int(ln[k])) for k, p in enumerate(L.PHASES)}

    def kernel_count(self) -> int:
        c = C.c_longlong()
        L.check(self.lib.pmgpu_kernel_count(self.h, C.byref(c)))
        return int(c.value)

    def set_list_capacity(self, tiles_per_row: int) -> None:
        """Fix the pair lists' capacity (testing the growth path)."""
        L.check(self.lib.pmgpu_debug_set_list_capacity(self.h, int(tiles_per_row)))

    def set_column_capacity(self, atoms_per_column: int) -> None:
        """Fix the atoms a pair-list column bucket holds (testing the growth
        path)."""
        L.check(self.lib.pmgpu_debug_set_column_capacity(self.h, int(atoms_per_column)))

    def limit_list_rows(self, tiles_per_row: int) -> None:
        """Limit the tiles a list row may hold in later builds, keeping the
        current list and forces (testing the growth path inside segments)."""
        L.check(self.lib.pmgpu_debug_limit_list_rows(self.h, int(tiles_per_row)))

    def cell_assign(self, cellsize: float):
        cells = np.zeros((self.n, 3), np.int32)
        dims = np.zeros(3, np.int32)
        L.check(self.lib.pmgpu_debug_cell_assign(self.h, float(cellsize), L.ptr(cells),
                                                 L.ptr(dims)))
        return cells, dims


# ------------------------------------------------------------------ forces
def _switch(kind: str, cutoff: float, switchon: float = 0.0, switchoff: float = 0.0,
            order: float = 0.0) -> L.Switch:
    """A switching function by its ProtoMol name: Universal, Cutoff, C1, C2,
    Cn, CmpCnCn (ProtoMol's id "ComplimentCnCn"), or ComplementC1 /
    ComplementC2 / ComplementCn."""
    name = kind.lower()
    comp = name.startswith("complement")
    if comp:
        name = name[len("complement"):]
    k = {"universal": L.SW_UNIVERSAL, "cutoff": L.SW_CUTOFF, "c1": L.SW_C1, "c2": L.SW_C2,
         "cn": L.SW_CN, "cmpcncn": L.SW_CMPCNCN, "complimentcncn": L.SW_CMPCNCN}[name]
    if comp:
        k |= L.SW_COMPLEMENT
    return L.Switch(k, float(cutoff), float(switchon), float(switchoff), float(order))


class SystemForce:
    """A force term registered on a GpuSystem (one ProtoMol ``force`` line)."""
    keyword = "SystemForce"

    def __init__(self, system: GpuSystem, fid: int):
        self.system = system
        self.id = fid
        system.forces.append(self)

    def evaluate(self, positions, forces: np.ndarray, energies: np.ndarray | None,
                 virial: bool = False) -> None:
        """SystemForce::evaluate: uploads positions, evaluates this term,
        ADDS into forces (n,3) and energies (ScalarStructure layout).  With
        energies None (and no virial) the term is evaluated force-only."""
        s = self.system
        pos = s._vec(positions)
        f = np.ascontiguousarray(forces, dtype=np.float64)
        if f.size != 3 * s.n:
            raise ValueError("forces must hold 3n values")
        e = np.zeros(L.E_COUNT) if (energies is not None or virial) else None
        v = np.zeros(9) if virial else None
        L.check(s.lib.pmgpu_force_evaluate(s.h, self.id, L.ptr(pos), L.ptr(f), L.ptr(e),
                                           L.ptr(v)))
        if f is not forces:
            forces[...] = f.reshape(forces.shape)
        if energies is not None:
            energies[:L.E_COUNT] += e
            if virial:
                energies[VIRIALXX:VIRIALXX + 9] += v

    def set_enabled(self, on: bool) -> None:
        L.check(self.system.lib.pmgpu_force_set_enabled(self.system.h, self.id, 1 if on else 0))

    def stats(self) -> dict:
        st = L.Stats()
        L.check(self.system.lib.pmgpu_force_stats(self.system.h, self.id, C.byref(st)))
        return dict(pairs_in_cutoff=st.pairs_in_cutoff, list_entries=st.list_entries,
                    clusters=st.clusters, list_builds=st.list_builds, cells=tuple(st.cells),
                    pair_kernel=PAIR_KERNELS.get(st.pair_kernel, st.pair_kernel),
                    list_capacity=st.list_capacity)

    def pair_set(self, cap: int = 1 << 24) -> np.ndarray:
        """The unordered pair set (i < j) this force evaluates at the
        resident positions."""
        s = self.system
        buf = np.zeros((cap, 2), np.int32)
        cnt = C.c_longlong()
        L.check(s.lib.pmgpu_debug_pair_set(s.h, self.id, L.ptr(buf), cap, C.byref(cnt)))
        if cnt.value > cap:
            return self.pair_set(int(cnt.value) + 1)
        return buf[:cnt.value]


class NonbondedCutoffSystemForce(SystemForce):
    """``LennardJones [Coulomb] -algorithm NonbondedCutoff`` on the device
    (force/nonbonded/NonbondedCutoffSystemForce.h, OneAtomPair /
    OneAtomPairTwo)."""
    keyword = "NonbondedCutoff"

    def __init__(self, system: GpuSystem, lj: L.Switch | None, coulomb: L.Switch | None,
                 cutoff: float, cellsize: float = 0.0):
        fid = C.c_int()
        L.check(system.lib.pmgpu_force_cutoff_add(
            system.h, C.byref(lj) if lj else None, C.byref(coulomb) if coulomb else None,
            float(cutoff), float(cellsize), C.byref(fid)))
        super().__init__(system, fid.value)


class NonbondedFullSystemForce(SystemForce):
    """``LennardJones|Coulomb -algorithm NonbondedFull``: the lattice sum
    (force/nonbonded/NonbondedFullSystemForce.h, OneAtomPairFull) over the
    cluster-pair list, every periodic image within the switch cutoff."""
    keyword = "NonbondedFull"

    def __init__(self, system: GpuSystem, lj: L.Switch | None, coulomb: L.Switch | None,
                 cutoff: float, cellsize: float = 0.0):
        fid = C.c_int()
        L.check(system.lib.pmgpu_force_full_add(
            system.h, C.byref(lj) if lj else None, C.byref(coulomb) if coulomb else None,
            float(cutoff), float(cellsize), C.byref(fid)))
        super().__init__(system, fid.value)


class NonbondedSimpleFullSwitchedForce(SystemForce):
    """``LennardJones|Coulomb -algorithm NonbondedSimpleFull
    -switchingFunction ...``: every pair with switching functions
    (Complement ones included), vacuum or the periodic minimal image."""
    keyword = "NonbondedSimpleFull"

    def __init__(self, system: GpuSystem, lj: L.Switch | None, coulomb: L.Switch | None):
        fid = C.c_int()
        L.check(system.lib.pmgpu_force_simplefull_switched_add(
            system.h, C.byref(lj) if lj else None, C.byref(coulomb) if coulomb else None,
            C.byref(fid)))
        super().__init__(system, fid.value)


class ScpismSystemForce(SystemForce):
    """``[LennardJones] CoulombSCPISM -algorithm NonbondedCutoff|
    NonbondedSimpleFull``: the SCPISM screened Coulomb term
    (force/coulomb/CoulombSCPISMForce.h) over every pair within the switch
    cutoffs, FP64."""
    keyword = "CoulombSCPISM"

    def __init__(self, system: GpuSystem, lj: L.Switch | None, coulomb: L.Switch,
                 dielectric: float = 80.0):
        fid = C.c_int()
        L.check(system.lib.pmgpu_force_scpism_add(
            system.h, C.byref(lj) if lj else None, C.byref(coulomb), float(dielectric),
            C.byref(fid)))
        super().__init__(system, fid.value)


class BornSystemForce(SystemForce):
    """``BornRadii`` + ``BornSelf`` (force/born/BornRadii.h,
    BornSelfForce.h): the SCPISM Born radii and self force, evaluated as one
    term (the radii pass, then the self pass)."""
    keyword = "BornSelf"

    def __init__(self, system: GpuSystem, radii_switch: int = 3, radii_cutoff: float = 5.0,
                 self_switch: int = 3, self_cutoff: float = 5.0, dielectric: float = 80.0):
        fid = C.c_int()
        L.check(system.lib.pmgpu_force_born_add(system.h, int(radii_switch), float(radii_cutoff),
                                                int(self_switch), float(self_cutoff),
                                                float(dielectric), C.byref(fid)))
        super().__init__(system, fid.value)


class NonbondedSimpleFullSystemForce(SystemForce):
    """``LennardJones|Coulomb -algorithm NonbondedSimpleFull`` (vacuum all pairs
    with exclusions)."""
    keyword = "NonbondedSimpleFull"

    def __init__(self, system: GpuSystem, lj: bool, coulomb: bool):
        fid = C.c_int()
        L.check(system.lib.pmgpu_force_simplefull_add(system.h, int(lj), int(coulomb),
                                                      C.byref(fid)))
        super().__init__(system, fid.value)


class PMEwaldSystemForce(SystemForce):
    """``Coulomb -algorithm PMEwald``: Ewald real space + smooth-PME
    reciprocal space + exclusion correction + self/charged-system terms,
    following NonbondedFullEwaldSystemForce's term structure."""
    keyword = "PMEwald"

    def __init__(self, system: GpuSystem, alpha: float, cutoff: float, order: int = 4,
                 grid=(64, 64, 64), real=True, reciprocal=True, correction=True,
                 exact_erf: bool = False, cellsize: float = 0.0):
        flags = (L.EWALD_REAL if real else 0) | (L.EWALD_RECIPROCAL if reciprocal else 0) | \
                (L.EWALD_CORRECTION if correction else 0)
        g = np.ascontiguousarray(np.asarray(grid, dtype=np.int32))
        fid = C.c_int()
        L.check(system.lib.pmgpu_force_pme_add(system.h, float(alpha), float(cutoff), int(order),
                                               L.ptr(g), flags, int(exact_erf), float(cellsize),
                                               C.byref(fid)))
        self.grid = tuple(int(x) for x in g)
        super().__init__(system, fid.value)


class GBForce(SystemForce):
    """``GBBornRadii`` + ``GBPartialSum`` + ``GBForce`` (OBC, vacuum, all pairs)
    evaluated as one term: the three reference passes run back to back on
    the device."""
    keyword = "GBForce"

    def __init__(self, system: GpuSystem, solute_dielec: float = 1.0,
                 solvent_dielec: float = 80.0):
        fid = C.c_int()
        L.check(system.lib.pmgpu_force_gb_add(system.h, float(solute_dielec),
                                              float(solvent_dielec), C.byref(fid)))
        super().__init__(system, fid.value)


class GBACEForce(SystemForce):
    """``GBACEForce`` (force/GB/GBACEForce.cpp): the ACE nonpolar term on the
    OBC Born radii, vacuum all pairs; with a GBForce in the same evaluation
    both share one Born-radius computation."""
    keyword = "GBACEForce"

    def __init__(self, system: GpuSystem, solvation_param: float = 2.26 / 418.4,
                 water_sphere_radius: float = 1.4):
        fid = C.c_int()
        L.check(system.lib.pmgpu_force_gbace_add(system.h, float(solvation_param),
                                                 float(water_sphere_radius), C.byref(fid)))
        super().__init__(system, fid.value)


class TorsionSystemForce(SystemForce):
    """``Dihedral`` and/or ``Improper`` (MTorsionSystemForce: cosine
    torsions for periodicity > 0, harmonic for periodicity 0)."""
    keyword = "Torsion"

    def __init__(self, system: GpuSystem, dihedrals: bool = True, impropers: bool = True):
        fid = C.c_int()
        L.check(system.lib.pmgpu_force_torsion_add(system.h, int(dihedrals), int(impropers),
                                                   C.byref(fid)))
        super().__init__(system, fid.value)


class BondedSystemForce(SystemForce):
    """``Bond`` and/or ``Angle`` (harmonic, with Urey-Bradley)."""
    keyword = "Bonded"

    def __init__(self, system: GpuSystem, bonds: bool = True, angles: bool = True):
        fid = C.c_int()
        L.check(system.lib.pmgpu_force_bonded_add(system.h, int(bonds), int(angles),
                                                  C.byref(fid)))
        super().__init__(system, fid.value)


class ForceFactory:
    """Parses ProtoMol ``.conf`` force lines into GPU forces.

    Grammar (factory/ForceFactory.cpp:133-200): keywords, ``-algorithm
    <Alg>``, one ``-switchingFunction <Sw>`` per potential in keyword order,
    and ``-<param> <value>`` pairs.  Parameters after a switching function
    belong to it; a trailing ``-cutoff`` belongs to the algorithm.  The GPU
    algorithms accept ProtoMol's names (``NonbondedCutoff``,
    ``NonbondedSimpleFull``, ``FullEwald``) with or without a ``GPU`` suffix,
    and ``PMEwald``."""

    def __init__(self, system: GpuSystem, cellsize: float = 0.0):
        self.system = system
        self.cellsize = cellsize
        self._born_radii = (3, 5.0)  # the last BornRadii line's -bornswitch, -cutoff

    @staticmethod
    def parse(line: str):
        toks = line.replace(",", " ").split()
        kws, i = [], 0
        while i < len(toks) and not toks[i].startswith("-"):
            kws.append(toks[i])
            i += 1
        alg, switches, params, cur = None, [], {}, None
        while i < len(toks):
            t = toks[i].lower()
            if t == "-algorithm":
                alg = toks[i + 1]
                i += 2
            elif t == "-switchingfunction":
                cur = {"kind": toks[i + 1]}
                switches.append(cur)
                i += 2
            elif t in ("-real", "-reciprocal", "-correction", "-exacterf"):
                params[t[1:]] = True
                i += 1
            elif t == "-gridsize":
                params["gridsize"] = tuple(int(x) for x in toks[i + 1:i + 4])
                i += 4
            elif t.startswith("-"):
                key = t[1:]
                val = float(toks[i + 1])
                target = cur if (cur is not None and key in ("cutoff", "switchon", "switchoff",
                                                               "n") and key not in cur) else params
                target[key] = val
                i += 2
            else:
                raise ValueError(f"cannot parse force line near '{toks[i]}': {line}")
        return kws, alg, switches, params

    def make(self, line: str) -> SystemForce:
        kws, alg, switches, p = self.parse(line)
        names = [k.lower() for k in kws]
        algn = re.sub("gpu$", "", (alg or "").lower())
        s = self.system
        if names and all(n in ("bond", "angle") for n in names):
            return BondedSystemForce(s, "bond" in names, "angle" in names)
        if names and all(n in ("dihedral", "improper") for n in names):
            return TorsionSystemForce(s, "dihedral" in names, "improper" in names)

        def term_switches(coulomb="coulomb"):
            sws = []
            for k, name in enumerate(names):
                sw = switches[k] if k < len(switches) else switches[-1]
                sws.append((name, _switch(sw["kind"], sw.get("cutoff", p.get("cutoff", 0.0)),
                                          sw.get("switchon", 0.0), sw.get("switchoff", 0.0),
                                          sw.get("n", 0.0))))
            lj = next((w for n, w in sws if n == "lennardjones"), None)
            co = next((w for n, w in sws if n == coulomb), None)
            return sws, lj, co

        if names and names[0] in ("bornradii", "bornself"):
            bsw = int(p.get("bornswitch", 3))
            cut = switches[0].get("cutoff", p.get("cutoff", 5.0)) if switches else \
                p.get("cutoff", 5.0)
            if names[0] == "bornradii":
                # its pass runs inside the BornSelf term, which must follow it
                self._born_radii = (bsw, cut)
                return _NoOpForce(s, "BornRadii")
            return BornSystemForce(s, self._born_radii[0], self._born_radii[1], bsw, cut,
                                   p.get("d", 80.0))
        if "coulombscpism" in names and algn in ("nonbondedcutoff", "nonbondedsimplefull"):
            if not switches:
                raise ValueError(f"CoulombSCPISM needs -switchingFunction: {line}")
            _, lj, co = term_switches(coulomb="coulombscpism")
            return ScpismSystemForce(s, lj, co, p.get("d", 80.0))
        if algn in ("nonbondedcutoff", "nonbondedfull"):
            if not switches:
                raise ValueError(f"{alg} needs -switchingFunction")
            sws, lj, co = term_switches()
            alg_cut = p.get("cutoff", max(w.cutoff for _, w in sws))
            cls = NonbondedCutoffSystemForce if algn == "nonbondedcutoff" else \
                NonbondedFullSystemForce
            return cls(s, lj, co, alg_cut, p.get("cellsize", self.cellsize))
        if algn in ("pmewald", "fullewald"):
            any_term = any(k in p for k in ("real", "reciprocal", "correction"))
            alpha = p["alpha"]
            rc = p.get("cutoff")
            if rc is None and "accuracy" in p:
                rc = math.sqrt(-math.log(p["accuracy"])) / alpha
            return PMEwaldSystemForce(
                s, alpha, rc or 0.0, int(p.get("order", 4)), p.get("gridsize", (64, 64, 64)),
                real=p.get("real", not any_term), reciprocal=p.get("reciprocal", not any_term),
                correction=p.get("correction", not any_term), exact_erf=p.get("exacterf", False),
                cellsize=self.cellsize)
        if algn == "nonbondedsimplefull":
            if "gbforce" in names:
                return GBForce(s, p.get("solutedielec", 1.0), p.get("solventdielec", 80.0))
            if "gbaceforce" in names:
                return GBACEForce(s, p.get("solvationparam", 2.26 / 418.4),
                                  p.get("watersphereradius", 1.4))
            if "gbbornradii" in names or "gbpartialsum" in names:
                return _NoOpForce(s, names[0])
            if s.periodic or (switches and any(sw["kind"].lower() != "universal"
                                               for sw in switches)):
                if switches:
                    _, lj, co = term_switches()
                else:
                    uni = _switch("Universal", 0.0)
                    lj = uni if "lennardjones" in names else None
                    co = uni if "coulomb" in names else None
                return NonbondedSimpleFullSwitchedForce(s, lj, co)
            return NonbondedSimpleFullSystemForce(s, "lennardjones" in names, "coulomb" in names)
        raise ValueError(f"no GPU force for: {line}")


class _NoOpForce:
    """GBBornRadii / GBPartialSum lines: their passes run inside the GPU
    GBForce term, which must follow them in the force list."""

    def __init__(self, system, name):
        self.system = system
        self.keyword = name
        self.id = -1

    def evaluate(self, positions, forces, energies, virial=False):
        return None


# ------------------------------------------------------------- integrators
class _Integrator:
    kind = L.INT_LEAPFROG

    def __init__(self, timestep: float, temperature: float = 0.0, gamma: float = 0.0,
                 seed: int = 0):
        self.p = L.Integrator(self.kind, float(timestep), float(temperature), float(gamma),
                              int(seed) & ((1 << 64) - 1))

    def run(self, system: GpuSystem, n_steps: int) -> None:
        """Integrator::run(n): all steps on the device."""
        L.check(system.lib.pmgpu_run(system.h, C.byref(self.p), int(n_steps)))

    def run_async(self, system: GpuSystem, n_steps: int) -> None:
        """Enqueue run(n) on the system's stream and return at once; finish
        with wait()."""
        L.check(system.lib.pmgpu_run_async(system.h, C.byref(self.p), int(n_steps)))

    @staticmethod
    def done(system: GpuSystem) -> bool:
        d = C.c_int()
        L.check(system.lib.pmgpu_run_query(system.h, C.byref(d)))
        return bool(d.value)

    @staticmethod
    def wait(system: GpuSystem) -> None:
        L.check(system.lib.pmgpu_run_wait(system.h))

    @staticmethod
    def discard(system: GpuSystem) -> None:
        """Wait for a pending run_async segment and undo it (the state at
        its start is restored)."""
        L.check(system.lib.pmgpu_run_discard(system.h))


class LeapfrogIntegrator(_Integrator):
    kind = L.INT_LEAPFROG


class LangevinLeapfrogIntegrator(_Integrator):
    kind = L.INT_LANGEVIN_LEAPFROG


class SystemEnsemble:
    """Resident systems advanced together (pmgpu_ensemble_*): every kernel
    of an MD step is one launch over all members, members with the same PME
    grid share one batched FFT, and segments replay as captured CUDA
    graphs.  A member's trajectory is bitwise the one it follows in any
    other ensemble with the same pair-kernel splits.  The members stay
    owned by the caller and must outlive the ensemble."""

    def __init__(self, members: list[GpuSystem]):
        if not members:
            raise ValueError("an ensemble needs members")
        self.lib = members[0].lib
        self.members = list(members)
        arr = (C.c_void_p * len(members))(*[m.h for m in members])
        h = C.c_void_p()
        L.check(self.lib.pmgpu_ensemble_create(arr, len(members), C.byref(h)))
        self.h = h

    def run(self, integrator: "_Integrator", n_steps: int) -> None:
        """integrator.run(member, n_steps) for every member at once."""
        L.check(self.lib.pmgpu_ensemble_run(self.h, C.byref(integrator.p), int(n_steps)))

    def set_splits(self, splits) -> None:
        a = np.ascontiguousarray(splits, dtype=np.int32)
        if a.shape != (len(self.members),):
            raise ValueError("one splits value per member")
        L.check(self.lib.pmgpu_ensemble_set_splits(self.h, L.ptr(a)))

    def time_pairs(self, splits, reps: int = 10) -> float:
        """Device ms of one force-only pair launch over all members with the
        given per-member splits (0: the member's current choice)."""
        a = np.ascontiguousarray(splits, dtype=np.int32)
        ms = C.c_double()
        L.check(self.lib.pmgpu_ensemble_time_pairs(self.h, L.ptr(a), int(reps), C.byref(ms)))
        return float(ms.value)

    def member(self, k: int) -> tuple[int, int]:
        """(i clusters, splits in use) of member k; (0, -1) for a member
        without the specialised force-only pair kernel."""
        c, sp = C.c_int(), C.c_int()
        L.check(self.lib.pmgpu_ensemble_member(self.h, int(k), C.byref(c), C.byref(sp)))
        return int(c.value), int(sp.value)

    def info(self) -> dict:
        i = L.EnsembleInfo()
        L.check(self.lib.pmgpu_ensemble_get_info(self.h, C.byref(i)))
        return {"members": i.members, "fft_buckets": i.fft_buckets, "kernels": i.kernels,
                "graph_replays": i.graph_replays, "steps": i.steps}

    def close(self) -> None:
        if self.h:
            L.check(self.lib.pmgpu_ensemble_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

