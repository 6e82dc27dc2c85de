"""Loading of the golden fixtures (tests/golden/*.npz, outputs of the
unmodified ProtoMol reference) into the two consumers: the FP64 oracle
(``oracle.System``) and the GPU path (``protomol_b200.GpuSystem``, which
reads a topology object by attribute)."""
from __future__ import annotations

import os
from types import SimpleNamespace

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name: str) -> dict:
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return {k: z[k] for k in z.files}


def topology(z: dict) -> SimpleNamespace:
    """Topology object for GpuSystem (and the oracle) from a fixture."""
    n = int(z["natoms"][0])
    nt = int(z["ntypes"][0])
    ex = z["exclusions"].reshape(-1, 3).astype(np.int32).copy()
    table_class = ex[:, 2].copy()
    if "exclusions_check" in z and len(ex):
        ex[:, 2] = z["exclusions_check"].astype(np.int32)
    t = SimpleNamespace(
        pos=z["positions"].reshape(n, 3).copy(), vel=z["velocities"].reshape(n, 3).copy(),
        charge=z["charge"].copy(), mass=z["mass"].copy(), type=z["type"].astype(np.int32),
        molecule=z["molecule"].astype(np.int32), lj=z["lj"].reshape(nt, nt, 4).copy(),
        exclusions=ex, exclusion_table_class=table_class,
        coulomb_scaling=float(z["coulomb_scaling"][0]), periodic=bool(int(z["periodic"][0])),
        box=z["box"].copy(), water=z["water"].astype(np.int32),
        bonds=z["bonds"].reshape(-1, 2).astype(np.int32) if "bonds" in z else np.zeros((0, 2), np.int32),
        bond_params=z["bond_params"].reshape(-1, 2) if "bond_params" in z else np.zeros((0, 2)),
        angles=z["angles"].reshape(-1, 3).astype(np.int32) if "angles" in z else np.zeros((0, 3), np.int32),
        angle_params=z["angle_params"].reshape(-1, 4) if "angle_params" in z else np.zeros((0, 4)))
    for kind in ("dihedral", "improper"):
        if kind + "s" in z and len(z[kind + "s"]):
            setattr(t, kind + "s", z[kind + "s"].reshape(-1, 4).astype(np.int32))
            setattr(t, kind + "_params", z[kind + "_params"].reshape(-1, 3).copy())
    if "gb_vdwr" in z:
        t.gb_vdwr = z["gb_vdwr"].copy()
        t.gb_scale = z["gb_scale"].copy()
        t.gb_offset = z["gb_offset"].copy()
        t.gb_obc = tuple(z["gb_obc"])
    if "scp_alpha" in z:
        t.scpism = {k: z[k].copy() for k in z if k.startswith("scp_")}
    return t


def oracle_system(z: dict):
    import oracle
    t = topology(z)
    s = oracle.System(pos=t.pos, charge=t.charge, type=t.type, molecule=t.molecule, lj=t.lj,
                      excl=t.exclusions, coulomb_scaling=t.coulomb_scaling,
                      periodic=t.periodic, box=t.box, mass=t.mass, water=t.water,
                      excl_table_class=t.exclusion_table_class)
    if hasattr(t, "gb_vdwr"):
        s.gb_vdwr, s.gb_scale, s.gb_offset, s.gb_obc = (t.gb_vdwr, t.gb_scale, t.gb_offset,
                                                         t.gb_obc)
    if hasattr(t, "scpism"):
        s.scpism = t.scpism
    return s


def forces(z: dict, k: int) -> np.ndarray:
    return z[f"forces_{k}"]


def energies(z: dict, k: int) -> np.ndarray:
    return z[f"energies_{k}"]


def rms_rel(a: np.ndarray, b: np.ndarray) -> float:
    """RMS relative force error: sqrt(sum |a-b|^2 / sum |b|^2)."""
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def parse_cutoff_def(d: str):
    """(potentials, switch dicts, algorithm cutoff) of a NonbondedCutoff,
    NonbondedFull or NonbondedSimpleFull line."""
    toks = d.split()
    pots = [t for t in toks if t in ("LennardJones", "Coulomb", "CoulombSCPISM")]
    sws, i, alg = [], 0, None
    while i < len(toks):
        if toks[i] == "-switchingFunction":
            sw = {"kind": toks[i + 1]}
            i += 2
            while i < len(toks) and toks[i] in ("-cutoff", "-switchon", "-switchoff", "-n") and \
                    toks[i][1:] not in sw:
                sw[toks[i][1:]] = float(toks[i + 1])
                i += 2
            sws.append(sw)
        elif toks[i] == "-cutoff":
            alg = float(toks[i + 1])
            i += 2
        else:
            i += 1
    if alg is None:
        alg = max(s.get("cutoff", 0.0) for s in sws)
    return pots, sws, alg
