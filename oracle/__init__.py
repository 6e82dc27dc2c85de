"""FP64 CPU oracle for ProtoMol's nonbonded hot path -- TEST INFRASTRUCTURE.

This package is the checker the CUDA library is compared against.  Only the
test suite, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import it; the product (``protomol_b200``) never does.

* ``pmoracle.c`` -- C restatement (cells, pair enumeration, LJ/Coulomb with
  C1/C2/Cn/Cutoff/Universal switching, full Ewald real/reciprocal/correction,
  OBC GB, integrator updates), each function citing the ProtoMol file:line it
  follows.  Built to ``oracle/liboracle.so`` by :func:`build`.
* ``spme.py`` -- FP64 smooth-PME reciprocal restatement (numpy FFT).
* ``refdump.py`` -- reader for dumps written by ``oracle/_ref/pm_forcedump``
  (the unmodified ProtoMol library, built by ``oracle/ref.mk``).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

EXCL_NONE, EXCL_MODIFIED, EXCL_FULL = 0, 1, 2
SW_UNIVERSAL, SW_CUTOFF, SW_C1, SW_C2, SW_CN, SW_CMPCNCN = 0, 1, 2, 3, 4, 5
SW_COMPLEMENT = 16  # flag on C1 / C2 / Cn: ComplementSwitchingFunction of it
POT_COULOMB, POT_LJ, POT_SCPISM = 0, 1, 2
INV_TIMEFACTOR = 0.02045482828087295  # base/PMConstants.cpp:54
SQRTCOULOMBCONSTANT = 18.2226123264  # base/PMConstants.cpp:67
BOLTZMANN = 0.001987191  # base/PMConstants.cpp:70


def build(force: bool = False) -> str:
    """Compile the C restatement (gcc, FP64, no FMA contraction)."""
    src = os.path.join(HERE, "pmoracle.c")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.check_call(
            ["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-std=c99",
             "-D_GNU_SOURCE", "-o", LIB, src, "-lm"])
    return LIB


class _Switch(C.Structure):
    _fields_ = [("kind", C.c_int), ("cutoff", C.c_double), ("switchon", C.c_double),
                ("switchoff", C.c_double), ("order", C.c_double)]


class _System(C.Structure):
    _fields_ = [("n", C.c_int), ("pos", C.c_void_p), ("charge", C.c_void_p),
                ("type", C.c_void_p), ("molecule", C.c_void_p), ("ntypes", C.c_int),
                ("lj", C.c_void_p), ("nexcl", C.c_int), ("excl", C.c_void_p),
                ("excl_table_class", C.c_void_p),
                ("coulomb_scaling", C.c_double), ("periodic", C.c_int),
                ("box", C.c_double * 12)]


class _Ewald(C.Structure):
    _fields_ = [("alpha", C.c_double), ("accuracy", C.c_double), ("rc", C.c_double),
                ("kc", C.c_double), ("exact_erf", C.c_int)]


class _GB(C.Structure):
    _fields_ = [("vdwr", C.c_void_p), ("scale", C.c_void_p), ("offset", C.c_void_p),
                ("water", C.c_void_p), ("alpha_obc", C.c_double), ("beta_obc", C.c_double),
                ("gamma_obc", C.c_double), ("solute_dielec", C.c_double),
                ("solvent_dielec", C.c_double)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        _lib.orc_cutoff_pairs.restype = C.c_long
    return _lib


@dataclass
class Switch:
    """A ProtoMol switching function: kind in {Universal, Cutoff, C1, C2, Cn,
    CmpCnCn, ComplementC1, ComplementC2, ComplementCn}.  CmpCnCn takes
    switchon < switchoff < cutoff and the order."""
    kind: str = "Cutoff"
    cutoff: float = 0.0
    switchon: float = 0.0
    switchoff: float = 0.0
    order: float = 0.0

    def c(self) -> _Switch:
        name = self.kind.lower()
        comp = name.startswith("complement")
        if comp:
            name = name[len("complement"):]
        k = {"universal": SW_UNIVERSAL, "cutoff": SW_CUTOFF, "c1": SW_C1, "c2": SW_C2,
             "cn": SW_CN, "cmpcncn": SW_CMPCNCN, "complimentcncn": SW_CMPCNCN}[name]
        if comp:
            k |= SW_COMPLEMENT
        return _Switch(k, self.cutoff, self.switchon, self.switchoff, self.order)


@dataclass
class System:
    """A built ProtoMol topology plus positions, as flat FP64/int arrays."""
    pos: np.ndarray  # (n,3) float64
    charge: np.ndarray  # (n,) scaled charges
    type: np.ndarray  # (n,) int32
    molecule: np.ndarray  # (n,) int32
    lj: np.ndarray  # (T,T,4) A,B,A14,B14
    excl: np.ndarray  # (m,3) int32 a1<a2, class
    coulomb_scaling: float = 1.0
    periodic: bool = True
    box: np.ndarray = field(default_factory=lambda: np.zeros(12))
    mass: np.ndarray | None = None
    water: np.ndarray | None = None
    # GB atom parameters (topology/BuildTopology.cpp:824-884)
    gb_vdwr: np.ndarray | None = None
    gb_scale: np.ndarray | None = None
    gb_offset: np.ndarray | None = None
    gb_obc: tuple = (1.0, 0.8, 4.85)
    # class per exclusion-table entry as getTable() holds it (None: same as
    # excl[:, 2]); the Ewald correction term iterates the table
    excl_table_class: np.ndarray | None = None
    # SCPISM per-atom data (keys as pm_forcedump writes them: scp_sqrtalpha,
    # scp_alpha, scp_zeta, scp_eta, scp_c, scp_g, scp_hbond, scp_residue,
    # scp_name); None: no SCPISM parameters
    scpism: dict | None = None

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])

    def _keep(self):
        self._k = dict(
            pos=np.ascontiguousarray(self.pos, dtype=np.float64).reshape(-1),
            charge=np.ascontiguousarray(self.charge, dtype=np.float64),
            type=np.ascontiguousarray(self.type, dtype=np.int32),
            molecule=np.ascontiguousarray(self.molecule, dtype=np.int32),
            lj=np.ascontiguousarray(self.lj, dtype=np.float64).reshape(-1),
            excl=np.ascontiguousarray(self.excl, dtype=np.int32).reshape(-1)
            if len(self.excl) else np.zeros(3, np.int32),
        )
        if self.excl_table_class is not None and len(self.excl):
            self._k["tclass"] = np.ascontiguousarray(self.excl_table_class, dtype=np.int32)
        return self._k

    def c(self) -> _System:
        k = self._keep()
        s = _System()
        s.n = self.n
        s.pos = k["pos"].ctypes.data
        s.charge = k["charge"].ctypes.data
        s.type = k["type"].ctypes.data
        s.molecule = k["molecule"].ctypes.data
        s.ntypes = int(self.lj.shape[0])
        s.lj = k["lj"].ctypes.data
        s.nexcl = int(len(self.excl))
        s.excl = k["excl"].ctypes.data
        s.excl_table_class = k["tclass"].ctypes.data if "tclass" in k else None
        s.coulomb_scaling = float(self.coulomb_scaling)
        s.periodic = 1 if self.periodic else 0
        for i in range(12):
            s.box[i] = float(self.box[i])
        return s

    def with_positions(self, pos: np.ndarray) -> "System":
        import dataclasses
        return dataclasses.replace(self, pos=np.asarray(pos, dtype=np.float64).reshape(-1, 3))


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def cell_assign(sysm: System, cellsize: float):
    cs = sysm.c()
    cell = np.zeros((sysm.n, 3), np.int32)
    dims = np.zeros(3, np.int32)
    rc = lib().orc_cell_assign(C.byref(cs), C.c_double(cellsize), _ptr(cell), _ptr(dims))
    assert rc == 0
    return cell, dims


def cutoff_pairs(sysm: System, cellsize: float, alg_cutoff: float, pair_cutoff: float):
    cs = sysm.c()
    n = lib().orc_cutoff_pairs(C.byref(cs), C.c_double(cellsize), C.c_double(alg_cutoff),
                               C.c_double(pair_cutoff), None, C.c_long(0))
    out = np.zeros((max(n, 1), 3), np.int32)
    n2 = lib().orc_cutoff_pairs(C.byref(cs), C.c_double(cellsize), C.c_double(alg_cutoff),
                                C.c_double(pair_cutoff), _ptr(out), C.c_long(n))
    assert n2 == n
    return out[:n]


def cutoff_force(sysm: System, cellsize: float, alg_cutoff: float, terms):
    """terms: list of (potential 'LennardJones'|'Coulomb', Switch)."""
    cs = sysm.c()
    pots = np.array([POT_LJ if p.lower().startswith("lennard") else POT_COULOMB
                     for p, _ in terms], np.int32)
    sws = (_Switch * len(terms))(*[s.c() for _, s in terms])
    f = np.zeros((sysm.n, 3))
    e = np.zeros(2)
    v = np.zeros(9)
    rc = lib().orc_cutoff_force(C.byref(cs), C.c_double(cellsize), C.c_double(alg_cutoff),
                                len(terms), _ptr(pots), sws, _ptr(f), _ptr(e), _ptr(v))
    assert rc == 0
    return f, {"coulomb": e[0], "lj": e[1]}, v.reshape(3, 3)


def simplefull_force(sysm: System, potential: str, sw: Switch | None = None):
    cs = sysm.c()
    sw = sw or Switch("Universal")
    pot = POT_LJ if potential.lower().startswith("lennard") else POT_COULOMB
    s = sw.c()
    f = np.zeros((sysm.n, 3))
    e = np.zeros(2)
    v = np.zeros(9)
    rc = lib().orc_simplefull_force(C.byref(cs), pot, C.byref(s), _ptr(f), _ptr(e), _ptr(v))
    assert rc == 0
    return f, {"coulomb": e[0], "lj": e[1]}, v.reshape(3, 3)


def simplefull_force_n(sysm: System, terms):
    """NonbondedSimpleFull with OneAtomPair or OneAtomPairTwo: terms is a
    list of (potential 'LennardJones'|'Coulomb', Switch); vacuum, or the
    minimal image of a periodic box."""
    cs = sysm.c()
    pots = np.array([POT_LJ if p.lower().startswith("lennard") else POT_COULOMB
                     for p, _ in terms], np.int32)
    sws = (_Switch * len(terms))(*[s.c() for _, s in terms])
    f = np.zeros((sysm.n, 3))
    e = np.zeros(2)
    v = np.zeros(9)
    rc = lib().orc_simplefull_force_n(C.byref(cs), len(terms), _ptr(pots), sws, _ptr(f),
                                      _ptr(e), _ptr(v))
    assert rc == 0
    return f, {"coulomb": e[0], "lj": e[1]}, v.reshape(3, 3)


def full_force(sysm: System, potential: str, sw: Switch, alg_cutoff: float):
    """NonbondedFull (lattice sum) with OneAtomPairFull of one potential."""
    cs = sysm.c()
    pot = POT_LJ if potential.lower().startswith("lennard") else POT_COULOMB
    s = sw.c()
    f = np.zeros((sysm.n, 3))
    e = np.zeros(2)
    v = np.zeros(9)
    rc = lib().orc_full_force(C.byref(cs), pot, C.byref(s), C.c_double(alg_cutoff), _ptr(f),
                              _ptr(e), _ptr(v))
    assert rc == 0
    return f, {"coulomb": e[0], "lj": e[1]}, v.reshape(3, 3)


def torsion_force(sysm: System, atoms: np.ndarray, params: np.ndarray):
    """Torsion terms (4 atoms; k, periodicity, phase [rad]) ->
    (forces (n,3), energy, virial (3,3))."""
    cs = sysm.c()
    a = np.ascontiguousarray(atoms, dtype=np.int32).reshape(-1)
    p = np.ascontiguousarray(params, dtype=np.float64).reshape(-1)
    f = np.zeros((sysm.n, 3))
    e = C.c_double(0)
    v = np.zeros(9)
    assert lib().orc_torsion_force(C.byref(cs), len(a) // 4, _ptr(a), _ptr(p), _ptr(f),
                                   C.byref(e), _ptr(v)) == 0
    return f, e.value, v.reshape(3, 3)


def ewald_params(sysm: System, alpha: float, accuracy: float, exact_erf: bool = False):
    cs = sysm.c()
    e = _Ewald()
    lib().orc_ewald_setup(C.byref(cs), C.c_double(alpha), C.c_double(accuracy),
                          1 if exact_erf else 0, C.byref(e))
    return e


def ewald_real(sysm: System, ew: _Ewald, cellsize: float):
    cs = sysm.c()
    f = np.zeros((sysm.n, 3))
    e = C.c_double(0)
    v = np.zeros(9)
    assert lib().orc_ewald_real(C.byref(cs), C.byref(ew), C.c_double(cellsize), _ptr(f),
                                C.byref(e), _ptr(v)) == 0
    return f, e.value, v.reshape(3, 3)


def ewald_reciprocal(sysm: System, ew: _Ewald):
    cs = sysm.c()
    f = np.zeros((sysm.n, 3))
    e = C.c_double(0)
    v = np.zeros(9)
    assert lib().orc_ewald_reciprocal(C.byref(cs), C.byref(ew), _ptr(f), C.byref(e),
                                      _ptr(v)) == 0
    return f, e.value, v.reshape(3, 3)


def ewald_correction(sysm: System, ew: _Ewald):
    cs = sysm.c()
    f = np.zeros((sysm.n, 3))
    e = C.c_double(0)
    v = np.zeros(9)
    assert lib().orc_ewald_correction(C.byref(cs), C.byref(ew), _ptr(f), C.byref(e),
                                      _ptr(v)) == 0
    return f, e.value, v.reshape(3, 3)


def ewald_self(sysm: System, ew: _Ewald):
    cs = sysm.c()
    a, b = C.c_double(0), C.c_double(0)
    lib().orc_ewald_self(C.byref(cs), C.byref(ew), C.byref(a), C.byref(b))
    return a.value, b.value


def gb_force(sysm: System, solute_dielec: float = 1.0, solvent_dielec: float = 80.0):
    cs = sysm.c()
    vd = np.ascontiguousarray(sysm.gb_vdwr, np.float64)
    sc = np.ascontiguousarray(sysm.gb_scale, np.float64)
    of = np.ascontiguousarray(sysm.gb_offset, np.float64)
    wa = np.ascontiguousarray(sysm.water if sysm.water is not None else np.zeros(sysm.n),
                              np.int32)
    g = _GB(vd.ctypes.data, sc.ctypes.data, of.ctypes.data, wa.ctypes.data,
            sysm.gb_obc[0], sysm.gb_obc[1], sysm.gb_obc[2], solute_dielec, solvent_dielec)
    born = np.zeros(sysm.n)
    f = np.zeros((sysm.n, 3))
    e = C.c_double(0)
    assert lib().orc_gb_force(C.byref(cs), C.byref(g), _ptr(born), _ptr(f), C.byref(e)) == 0
    return f, e.value, born


def bonded_force(sysm: System, bonds=None, bond_params=None, angles=None, angle_params=None):
    """Harmonic bonds and Urey-Bradley angles -> (forces (n,3), {"bond": E,
    "angle": E}, virial (3,3))."""
    cs = sysm.c()
    f = np.zeros((sysm.n, 3))
    out, vt = {}, np.zeros(9)
    for key, atoms, prm, fn, w in (("bond", bonds, bond_params, lib().orc_bond_force, 2),
                                   ("angle", angles, angle_params, lib().orc_angle_force, 3)):
        if atoms is None or len(atoms) == 0:
            out[key] = 0.0
            continue
        a = np.ascontiguousarray(atoms, dtype=np.int32).reshape(-1)
        p = np.ascontiguousarray(prm, dtype=np.float64).reshape(-1)
        e = C.c_double(0)
        v = np.zeros(9)
        assert fn(C.byref(cs), len(a) // w, _ptr(a), _ptr(p), _ptr(f), C.byref(e), _ptr(v)) == 0
        out[key] = e.value
        vt += v
    return f, out, vt.reshape(3, 3)


ACE_SIGMA = 2.26 / 418.4  # GBACEForce -solvationparam default (GBACEForce.cpp:226)
ACE_RHO = 1.4             # -watersphereradius default (GBACEForce.cpp:229)


class _Scpism(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in ("sqrtalpha", "alpha", "zeta", "eta", "c", "g", "hbond",
                                           "residue", "name", "water")]


def _scpism(sysm: System):
    d = sysm.scpism
    keep = {k: np.ascontiguousarray(d["scp_" + k], dtype=np.float64)
            for k in ("sqrtalpha", "alpha", "zeta", "eta", "c", "g")}
    keep.update({k: np.ascontiguousarray(d["scp_" + k], dtype=np.int32)
                 for k in ("hbond", "residue", "name")})
    keep["water"] = np.ascontiguousarray(sysm.water if sysm.water is not None
                                         else np.zeros(sysm.n), dtype=np.int32)
    p = _Scpism(**{k: v.ctypes.data for k, v in keep.items()})
    return p, keep


def _pot(name: str) -> int:
    n = name.lower()
    if n.startswith("lennard"):
        return POT_LJ
    return POT_SCPISM if n == "coulombscpism" else POT_COULOMB


def scpism_pair_force(sysm: System, terms, D: float = 80.0):
    """LennardJones and/or CoulombSCPISM over every pair within the switch
    cutoffs: terms is a list of (potential, Switch)."""
    cs = sysm.c()
    p, keep = _scpism(sysm)
    pots = np.array([_pot(t) for t, _ in terms], np.int32)
    sws = (_Switch * len(terms))(*[w.c() for _, w in terms])
    f = np.zeros((sysm.n, 3))
    e = np.zeros(2)
    v = np.zeros(9)
    rc = lib().orc_scpism_pair_force(C.byref(cs), C.byref(p), C.c_double(D), len(terms),
                                     _ptr(pots), sws, _ptr(f), _ptr(e), _ptr(v))
    assert rc == 0
    return f, {"coulomb": e[0], "lj": e[1]}, v.reshape(3, 3)


def born_force(sysm: System, radii_switch: int = 3, radii_cutoff: float = 5.0,
               self_switch: int = 3, self_cutoff: float = 5.0, D: float = 80.0):
    """BornRadii then BornSelf: (forces, self energy, Born radii)."""
    cs = sysm.c()
    p, keep = _scpism(sysm)
    f = np.zeros((sysm.n, 3))
    e = np.zeros(2)
    v = np.zeros(9)
    born = np.zeros(sysm.n)
    rc = lib().orc_born_force(C.byref(cs), C.byref(p), int(radii_switch),
                              C.c_double(radii_cutoff), int(self_switch),
                              C.c_double(self_cutoff), C.c_double(D), _ptr(born), _ptr(f),
                              _ptr(e), _ptr(v))
    assert rc == 0
    return f, float(e[0]), born


def gbace_force(sysm: System, sigma: float = ACE_SIGMA, rho_s: float = ACE_RHO):
    """GBACEForce on the GBBornRadii radii -> (forces (n,3), energy)."""
    cs = sysm.c()
    vd = np.ascontiguousarray(sysm.gb_vdwr, np.float64)
    sc = np.ascontiguousarray(sysm.gb_scale, np.float64)
    of = np.ascontiguousarray(sysm.gb_offset, np.float64)
    wa = np.ascontiguousarray(sysm.water if sysm.water is not None else np.zeros(sysm.n),
                              np.int32)
    g = _GB(vd.ctypes.data, sc.ctypes.data, of.ctypes.data, wa.ctypes.data,
            sysm.gb_obc[0], sysm.gb_obc[1], sysm.gb_obc[2], 1.0, 80.0)
    f = np.zeros((sysm.n, 3))
    e = C.c_double(0)
    assert lib().orc_gbace_force(C.byref(cs), C.byref(g), C.c_double(sigma), C.c_double(rho_s),
                                 _ptr(f), C.byref(e)) == 0
    return f, e.value


def kick(mass, forces, h, vel):
    vel = np.ascontiguousarray(vel, np.float64).copy()
    lib().orc_kick(len(mass), _ptr(np.ascontiguousarray(mass, np.float64)),
                   _ptr(np.ascontiguousarray(forces, np.float64)), C.c_double(h), _ptr(vel))
    return vel


def drift(vel, h, pos):
    pos = np.ascontiguousarray(pos, np.float64).copy()
    lib().orc_drift(len(pos), _ptr(np.ascontiguousarray(vel, np.float64)), C.c_double(h),
                    _ptr(pos))
    return pos


def langevin_half_kick(mass, forces, timestep_fs, gamma_ps, temperature, gauss, vel):
    vel = np.ascontiguousarray(vel, np.float64).copy()
    lib().orc_langevin_half_kick(
        len(mass), _ptr(np.ascontiguousarray(mass, np.float64)),
        _ptr(np.ascontiguousarray(forces, np.float64)), C.c_double(timestep_fs),
        C.c_double(gamma_ps), C.c_double(temperature),
        _ptr(np.ascontiguousarray(gauss, np.float64)), _ptr(vel))
    return vel
