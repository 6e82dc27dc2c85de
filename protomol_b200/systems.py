"""Seeded synthetic systems of the benchmark shapes, and writers of the
ProtoMol input files (PSF / PAR / XYZ / .conf) for the same systems, so the
reference CPU path can run the identical inputs.

* ``tip3p_box``: TIP3P water (O -0.834, H +0.417; CHARMM TIP3P LJ and
  bonded parameters: OT eps 0.1521, Rmin/2 1.7682; HT eps 0.046, Rmin/2
  0.2245; bond OT-HT k 450, r0 0.9572; angle HT-OT-HT k 55, 104.52 deg) on a
  cubic lattice with uniform jitter and random orientations, Maxwell-
  Boltzmann velocities.
* ``gb_polymer``: linear heteropolymer for the implicit-solvent (GB) form.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

SQRTCOULOMBCONSTANT = 18.2226123264  # base/PMConstants.cpp:67
BOLTZMANN = 0.001987191  # base/PMConstants.cpp:70

# CHARMM TIP3P parameters (epsilon as a positive well depth, Rmin/2 in A)
TIP3P = dict(q_o=-0.834, q_h=0.417, m_o=15.9994, m_h=1.008, eps_o=0.1521, rmin2_o=1.7682,
             eps_h=0.046, rmin2_h=0.2245, k_bond=450.0, r_oh=0.9572, k_angle=55.0,
             theta_hoh=104.52)


@dataclass
class MolecularSystem:
    """Topology arrays (what ProtoMol's GenericTopology holds for the
    nonbonded path) plus positions and velocities."""
    pos: np.ndarray                 # (n,3)
    vel: np.ndarray                 # (n,3)
    charge: np.ndarray              # scaled charges
    mass: np.ndarray
    type: np.ndarray                # int32 type index
    molecule: np.ndarray            # int32 molecule index
    type_names: list
    lj: np.ndarray                  # (T,T,4) A, B, A14, B14
    exclusions: np.ndarray          # (m,3) a1 < a2, class
    bonds: np.ndarray               # (nb,2)
    bond_params: np.ndarray         # (nb,2) k, r0
    angles: np.ndarray              # (na,3)
    angle_params: np.ndarray        # (na,4) k, theta0 [rad], k_ub, r_ub
    periodic: bool = True
    box: np.ndarray = field(default_factory=lambda: np.zeros(12))
    coulomb_scaling: float = 1.0
    water: np.ndarray | None = None
    gb_vdwr: np.ndarray | None = None
    gb_scale: np.ndarray | None = None
    gb_offset: np.ndarray | None = None
    gb_obc: tuple = (1.0, 0.8, 4.85)
    # torsions: (m,4) atoms and (m,3) k, periodicity, phase [rad]
    dihedrals: np.ndarray | None = None
    dihedral_params: np.ndarray | None = None
    impropers: np.ndarray | None = None
    improper_params: np.ndarray | None = None
    # PSF bookkeeping
    atom_names: list | None = None
    resnames: list | None = None
    raw_charge: np.ndarray | None = None
    eps: np.ndarray | None = None        # per type, for PAR
    rmin2: np.ndarray | None = None      # per type, for PAR

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])


def charmm_lj_table(eps: np.ndarray, rmin2: np.ndarray) -> np.ndarray:
    """CHARMM combination rule as BuildTopology builds the LJ table
    (topology/BuildTopology.cpp:662-672): r = s_i + s_j, e = sqrt(e_i e_j),
    A = r^12 e, B = 2 r^6 e (1-4 parameters equal the normal ones here)."""
    t = len(eps)
    lj = np.zeros((t, t, 4))
    for i in range(t):
        for j in range(t):
            r = rmin2[i] + rmin2[j]
            e = math.sqrt(eps[i] * eps[j])
            r6 = r ** 6
            A = r6 * r6 * e
            B = 2 * r6 * e
            lj[i, j] = (A, B, A, B)
    return lj


def _random_rotation(rng: np.random.Generator) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([
        [a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
        [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
        [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


def _random_rotations(rng: np.random.Generator, count: int) -> np.ndarray:
    """count rotation matrices from unit quaternions, (count, 3, 3)."""
    q = rng.normal(size=(count, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    a, b, c, d = q.T
    return np.stack([
        np.stack([a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)], -1),
        np.stack([2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)], -1),
        np.stack([2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d], -1)],
        1)


def mb_velocities(mass: np.ndarray, temperature: float, rng) -> np.ndarray:
    """Maxwell-Boltzmann velocities in ProtoMol units (A per internal time
    unit, so that 0.5 m v^2 is in kcal/mol), zero total momentum."""
    sig = np.sqrt(BOLTZMANN * temperature / mass)[:, None]
    v = rng.normal(size=(len(mass), 3)) * sig
    p = (v * mass[:, None]).sum(0) / mass.sum()
    return v - p


def tip3p_box(n_waters: int, edge: float, seed: int, jitter: float = 0.0,
              temperature: float = 300.0, lattice: int | None = None,
              origin: tuple = (0.0, 0.0, 0.0)) -> MolecularSystem:
    """n_waters TIP3P waters in a periodic cube of the given edge: lattice
    sites (spacing edge/lattice, a random subset if there are more sites
    than waters) plus U(-jitter, jitter) displacement, random orientations,
    rigid 0.9572 A / 104.52 deg geometry."""
    rng = np.random.default_rng(seed)
    if lattice is None:
        lattice = int(math.ceil(n_waters ** (1.0 / 3.0) - 1e-9))
    g = np.arange(lattice, dtype=np.float64)
    sites = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    if len(sites) < n_waters:
        raise ValueError("lattice too small")
    if len(sites) > n_waters:
        sites = sites[np.sort(rng.choice(len(sites), n_waters, replace=False))]
    spacing = edge / lattice
    centers = (sites + 0.5) * spacing - 0.5 * edge + np.asarray(origin)
    centers += rng.uniform(-jitter, jitter, size=centers.shape)
    p = TIP3P
    half = math.radians(p["theta_hoh"]) / 2
    local = np.array([[0.0, 0.0, 0.0],
                      [p["r_oh"] * math.sin(half), 0.0, p["r_oh"] * math.cos(half)],
                      [-p["r_oh"] * math.sin(half), 0.0, p["r_oh"] * math.cos(half)]])
    n = 3 * n_waters
    # one random rotation per water (the same draws, in the same order, as
    # n_waters calls of _random_rotation)
    R = _random_rotations(rng, n_waters)
    pos = (centers[:, None, :] + np.einsum("ak,wjk->waj", local, R)).reshape(n, 3)
    raw_q = np.tile([p["q_o"], p["q_h"], p["q_h"]], n_waters)
    mass = np.tile([p["m_o"], p["m_h"], p["m_h"]], n_waters)
    typ = np.tile(np.array([0, 1, 1], np.int32), n_waters)
    mol = np.repeat(np.arange(n_waters, dtype=np.int32), 3)
    eps = np.array([p["eps_o"], p["eps_h"]])
    rmin2 = np.array([p["rmin2_o"], p["rmin2_h"]])
    o = 3 * np.arange(n_waters)
    excl = np.stack([np.stack([o, o + 1, np.full_like(o, 2)], 1),
                     np.stack([o, o + 2, np.full_like(o, 2)], 1),
                     np.stack([o + 1, o + 2, np.full_like(o, 2)], 1)], 1).reshape(-1, 3)
    bonds = np.stack([np.stack([o, o + 1], 1), np.stack([o, o + 2], 1)], 1).reshape(-1, 2)
    bond_params = np.tile([p["k_bond"], p["r_oh"]], (len(bonds), 1))
    angles = np.stack([o + 1, o, o + 2], 1)
    angle_params = np.tile([p["k_angle"], math.radians(p["theta_hoh"]), 0.0, 0.0],
                           (len(angles), 1))
    box = np.array([edge, 0, 0, 0, edge, 0, 0, 0, edge, *origin], dtype=np.float64)
    vel = mb_velocities(mass, temperature, rng)
    return MolecularSystem(
        pos=pos, vel=vel, charge=raw_q * SQRTCOULOMBCONSTANT, mass=mass, type=typ,
        molecule=mol, type_names=["OT", "HT"], lj=charmm_lj_table(eps, rmin2),
        exclusions=excl.astype(np.int32), bonds=bonds.astype(np.int32),
        bond_params=bond_params, angles=angles.astype(np.int32), angle_params=angle_params,
        periodic=True, box=box, water=np.ones(n, np.int32),
        atom_names=["OH2", "H1", "H2"] * n_waters, resnames=["TIP3"] * n,
        raw_charge=raw_q, eps=eps, rmin2=rmin2)


def water_box_for_density(n_waters: int, density: float, seed: int, **kw) -> MolecularSystem:
    """Box edge set for a number density of waters per A^3."""
    edge = (n_waters / density) ** (1.0 / 3.0)
    return tip3p_box(n_waters, edge, seed, **kw)


def gb_polymer(n_atoms: int, seed: int, temperature: float = 300.0) -> MolecularSystem:
    """Linear heteropolymer (vacuum): random-walk chain with bond 1.53 A and
    ~109.5 deg angles that avoids close contacts, charges U[-0.5, 0.5]
    renormalised to net zero, LJ sigma U[3.0, 3.8] and eps U[0.05, 0.2],
    intrinsic Born radii U[1.2, 1.9], element letters cycling over
    C/N/O/H/S for the GB scaling factors."""
    rng = np.random.default_rng(seed)
    pos = np.zeros((n_atoms, 3))
    b = 1.53
    theta = math.radians(109.5)
    if n_atoms > 1:
        pos[1] = [b, 0, 0]
    if n_atoms > 2:
        pos[2] = pos[1] + b * np.array([-math.cos(theta), math.sin(theta), 0.0])
    for i in range(3, n_atoms):
        for _ in range(200):
            u = pos[i - 1] - pos[i - 2]
            u /= np.linalg.norm(u)
            # random direction at the tetrahedral angle to the previous bond
            t = rng.normal(size=3)
            t -= t.dot(u) * u
            t /= np.linalg.norm(t)
            d = -math.cos(theta) * u * -1.0
            d = math.cos(math.pi - theta) * u + math.sin(math.pi - theta) * t
            cand = pos[i - 1] + b * d
            if i < 4 or np.min(np.linalg.norm(pos[:i - 3] - cand, axis=1)) > 3.0:
                break
        pos[i] = cand
    pos -= pos.mean(0)
    q = rng.uniform(-0.5, 0.5, n_atoms)
    q -= q.mean()
    sigma = rng.uniform(3.0, 3.8, n_atoms)
    eps = rng.uniform(0.05, 0.2, n_atoms)
    rmin2 = sigma * 2 ** (1 / 6) / 2
    elem = np.array(list("CNOHS"))[np.arange(n_atoms) % 5]
    scale_by = {"H": 0.85, "C": 0.72, "N": 0.79, "O": 0.85, "P": 0.86, "S": 0.96}
    gb_scale = np.array([scale_by.get(e, 0.8) for e in elem])
    mass = np.array([{"C": 12.011, "N": 14.007, "O": 15.999, "H": 1.008,
                      "S": 32.06}[e] for e in elem])
    typ = np.arange(n_atoms, dtype=np.int32)
    lj = charmm_lj_table(eps, rmin2)
    bonds = np.stack([np.arange(n_atoms - 1), np.arange(1, n_atoms)], 1).astype(np.int32)
    bond_params = np.tile([300.0, 1.53], (len(bonds), 1))
    angles = np.stack([np.arange(n_atoms - 2), np.arange(1, n_atoms - 1),
                       np.arange(2, n_atoms)], 1).astype(np.int32)
    angle_params = np.tile([50.0, math.radians(109.5), 0.0, 0.0], (len(angles), 1))
    # periodic dihedrals n = 3, k = 0.2 kcal/mol, phase 0 along the backbone
    dih = np.stack([np.arange(n_atoms - 3), np.arange(1, n_atoms - 2),
                    np.arange(2, n_atoms - 1), np.arange(3, n_atoms)], 1).astype(np.int32)
    dih_params = np.tile([0.2, 3.0, 0.0], (len(dih), 1))
    # exclude scaled1-4: 1-2, 1-3 full; 1-4 modified
    ex = [(i, i + 1, 2) for i in range(n_atoms - 1)] + \
         [(i, i + 2, 2) for i in range(n_atoms - 2)] + \
         [(i, i + 3, 1) for i in range(n_atoms - 3)]
    vel = mb_velocities(mass, temperature, rng)
    return MolecularSystem(
        pos=pos, vel=vel, charge=q * SQRTCOULOMBCONSTANT, mass=mass, type=typ,
        molecule=np.zeros(n_atoms, np.int32), type_names=[f"{e}{i}" for i, e in enumerate(elem)],
        lj=lj, exclusions=np.array(ex, np.int32).reshape(-1, 3), bonds=bonds,
        bond_params=bond_params, angles=angles, angle_params=angle_params, periodic=False,
        box=np.zeros(12), water=np.zeros(n_atoms, np.int32),
        dihedrals=dih, dihedral_params=dih_params,
        gb_vdwr=rng.uniform(1.2, 1.9, n_atoms), gb_scale=gb_scale,
        gb_offset=np.full(n_atoms, 0.09), raw_charge=q, eps=eps, rmin2=rmin2,
        atom_names=[f"{e}{i % 100}" for i, e in enumerate(elem)], resnames=["POL"] * n_atoms)


# ---------------------------------------------------------------- writers
def write_psf(sysm: MolecularSystem, path: str) -> None:
    """X-PLOR/CHARMM PSF as ProtoMol's PSFReader tokenises it
    (io/PSFReader.cpp:115-200)."""
    n = sysm.n
    with open(path, "w") as f:
        f.write("PSF \n\n       1 !NTITLE\n REMARKS synthetic system\n\n")
        f.write(f"{n:8d} !NATOM\n")
        for i in range(n):
            res = int(sysm.molecule[i]) + 1
            f.write(f"{i + 1:8d} S{res % 10000:<4d} {res:4d} {sysm.resnames[i]:<4s} "
                    f"{sysm.atom_names[i]:<4s} {sysm.type_names[sysm.type[i]]:<4s} "
                    f"{sysm.raw_charge[i]:.17g} {sysm.mass[i]:.17g} 0\n")
        f.write(f"\n{len(sysm.bonds):8d} !NBOND: bonds\n")
        for k, (a, b) in enumerate(sysm.bonds):
            f.write(f"{a + 1:8d}{b + 1:8d}")
            if k % 4 == 3:
                f.write("\n")
        f.write(f"\n\n{len(sysm.angles):8d} !NTHETA: angles\n")
        for k, (a, b, c) in enumerate(sysm.angles):
            f.write(f"{a + 1:8d}{b + 1:8d}{c + 1:8d}")
            if k % 3 == 2:
                f.write("\n")
        for title, key in (("NPHI: dihedrals", "dihedrals"), ("NIMPHI: impropers", "impropers")):
            quads = getattr(sysm, key)
            quads = np.zeros((0, 4), np.int32) if quads is None else quads
            f.write(f"\n\n{len(quads):8d} !{title}\n")
            for k, q in enumerate(quads):
                f.write("".join(f"{a + 1:8d}" for a in q))
                if k % 2 == 1:
                    f.write("\n")
        f.write("\n\n       0 !NDON: donors\n\n\n       0 !NACC: acceptors\n\n\n"
                "       0 !NNB\n\n\n       0       0 !NGRP\n\n")


def write_par(sysm: MolecularSystem, path: str) -> None:
    """CHARMM PAR with the BONDS/ANGLES/NONBONDED sections the system uses."""
    tn = sysm.type_names
    with open(path, "w") as f:
        f.write("* synthetic parameters\n*\n\nBONDS\n")
        seen = set()
        for (a, b), (k, r0) in zip(sysm.bonds, sysm.bond_params):
            key = (tn[sysm.type[a]], tn[sysm.type[b]])
            if key in seen:
                continue
            seen.add(key)
            f.write(f"{key[0]:<6s} {key[1]:<6s} {k:.17g} {r0:.17g}\n")
        f.write("\nANGLES\n")
        seen = set()
        for (a, b, c), prm in zip(sysm.angles, sysm.angle_params):
            key = (tn[sysm.type[a]], tn[sysm.type[b]], tn[sysm.type[c]])
            if key in seen:
                continue
            seen.add(key)
            f.write(f"{key[0]:<6s} {key[1]:<6s} {key[2]:<6s} {prm[0]:.17g} "
                    f"{math.degrees(prm[1]):.17g}\n")
        for title, key in (("DIHEDRALS", "dihedral"), ("IMPROPER", "improper")):
            f.write(f"\n{title}\n")
            quads, prms = getattr(sysm, key + "s"), getattr(sysm, key + "_params")
            seen = set()
            for q, prm in zip(quads if quads is not None else [], prms if prms is not None else []):
                key4 = tuple(tn[sysm.type[a]] for a in q)
                if key4 in seen:
                    continue
                seen.add(key4)
                if title == "DIHEDRALS":
                    f.write(" ".join(f"{t:<6s}" for t in key4) +
                            f" {prm[0]:.17g} {int(prm[1])} {math.degrees(prm[2]):.17g}\n")
                else:
                    f.write(" ".join(f"{t:<6s}" for t in key4) +
                            f" {prm[0]:.17g} 0 {math.degrees(prm[2]):.17g}\n")
        f.write("\nNONBONDED nbxmod 5 atom cdiel shift vatom "
                "vdistance vswitch -\ncutnb 14.0 ctofnb 12.0 ctonnb 10.0 eps 1.0 e14fac 1.0 "
                "wmin 1.5\n\n")
        for t, name in enumerate(tn):
            f.write(f"{name:<6s} 0.000000 {-sysm.eps[t]:.17g} {sysm.rmin2[t]:.17g}\n")
        f.write("\nEND\n")


def write_xyz(arr: np.ndarray, names, path: str) -> None:
    with open(path, "w") as f:
        f.write(f"{len(arr)}\n!synthetic\n")
        for nm, (x, y, z) in zip(names, arr):
            f.write(f"{nm} {x:.17g} {y:.17g} {z:.17g}\n")


def write_protomol_inputs(sysm: MolecularSystem, directory: str, stem: str,
                          forces: list[str], integrator: str = "Leapfrog",
                          timestep: float = 0.5, numsteps: int = 0,
                          cellsize: float | None = None, extra: str = "",
                          outputs: bool = True, integrator_params: str = "",
                          outputfreq: int | None = None) -> str:
    """Write PSF/PAR/XYZ inputs and a .conf evaluating the given force lines
    with the given integrator; returns the conf path.  outputfreq defaults
    to numsteps (one output at the end)."""
    os.makedirs(directory, exist_ok=True)
    names = [sysm.type_names[t] for t in sysm.type]
    write_psf(sysm, os.path.join(directory, stem + ".psf"))
    write_par(sysm, os.path.join(directory, stem + ".par"))
    write_xyz(sysm.pos, names, os.path.join(directory, stem + ".pos.xyz"))
    write_xyz(sysm.vel, names, os.path.join(directory, stem + ".vel.xyz"))
    ofreq = outputfreq if outputfreq else max(1, numsteps)
    lines = [f"firststep 0", f"numsteps {numsteps}", f"outputfreq {ofreq}",
             "angularMomentum 0", "comMotion 0", "exclude scaled1-4", "seed 1234",
             f"posfile {stem}.pos.xyz", f"velfile {stem}.vel.xyz", f"psffile {stem}.psf",
             f"parfile {stem}.par", "temperature 300"]
    if outputs:
        lines += [f"XYZForceFile {stem}.out.forces", f"finXYZPosFile {stem}.out.pos",
                  f"finXYZVelFile {stem}.out.vel", f"allenergiesfile {stem}.out.energy"]
    if sysm.periodic:
        b = sysm.box
        lines += [f"cellBasisVector1 {b[0]:.17g} 0 0", f"cellBasisVector2 0 {b[4]:.17g} 0",
                  f"cellBasisVector3 0 0 {b[8]:.17g}",
                  f"cellorigin {b[9]:.17g} {b[10]:.17g} {b[11]:.17g}",
                  "boundaryConditions Periodic"]
    else:
        lines += ["boundaryConditions vacuum"]
    lines += ["cellManager Cubic", f"cellsize {cellsize if cellsize else 5.0}"]
    if extra:
        lines.append(extra)
    body = "\n".join(f"    force {fl}" for fl in forces)
    ip = f"    {integrator_params}\n" if integrator_params else ""
    lines.append(f"Integrator {{\n  level 0 {integrator} {{\n    timestep {timestep}\n{ip}{body}\n"
                 "  }\n}")
    conf = os.path.join(directory, stem + ".conf")
    with open(conf, "w") as f:
        f.write("\n".join(lines) + "\n")
    return conf
