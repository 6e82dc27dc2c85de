"""Regenerates the golden fixtures in this directory from the unmodified
ProtoMol reference (built by oracle/ref.mk into oracle/_ref/).

Each fixture is an .npz holding the topology ProtoMol built (charges, masses,
types, molecules, LJ table, exclusion table, box, GB atom parameters), the
positions, and the FP64 forces and ScalarStructure energies of each force
line, as written by oracle/_ref/pm_forcedump.  Inputs are the reference's own
test systems (its test/tests/*.conf data) and seeded synthetic systems from
protomol_b200.systems written out as PSF/PAR/XYZ.

    PROTOMOL_REF=<ProtoMol checkout> python tests/golden/make_golden.py [part]
"""
from __future__ import annotations

import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import refdump  # noqa: E402
from protomol_b200 import systems  # noqa: E402

def _ref_tests() -> str:
    """The reference's test inputs: $PROTOMOL_REF/test/tests, PROTOMOL_REF
    being the ProtoMol checkout (required; no default)."""
    ref = os.environ.get("PROTOMOL_REF")
    if not ref:
        raise SystemExit("set PROTOMOL_REF to the ProtoMol checkout")
    return os.path.join(ref, "test", "tests")


def save(name: str, d: dict, extra: dict | None = None) -> None:
    out = {}
    for k in ("natoms", "charge", "mass", "type", "molecule", "water", "lj", "ntypes",
              "scp_sqrtalpha", "scp_alpha", "scp_zeta", "scp_eta", "scp_c", "scp_g",
              "scp_hbond", "scp_residue", "scp_name",
              "exclusions", "exclusions_check", "coulomb_scaling", "periodic", "box",
              "positions", "velocities", "bonds", "bond_params", "angles", "angle_params",
              "dihedrals", "dihedral_params", "impropers", "improper_params",
              "gb_vdwr", "gb_scale", "gb_offset", "gb_obc"):
        if k in d:
            out[k] = np.asarray(d[k])
    defs, ids = [], []
    for k, f in enumerate(d["forces"]):
        out[f"forces_{k}"] = f["forces"]
        out[f"energies_{k}"] = f["energies"]
        defs.append(f["def"])
        ids.append(f.get("id", ""))
    out["defs"] = np.array(defs)
    out["ids"] = np.array(ids)
    if extra:
        out.update(extra)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print("wrote", name, d["natoms"][0], "atoms,", len(defs), "forces")


def reference_conf(conf: str, forces: list[str], steps: int = 0) -> dict:
    tmp = tempfile.mkdtemp()
    try:
        os.symlink(os.path.join(_ref_tests(), "data"), os.path.join(tmp, "data"))
        shutil.copy(os.path.join(_ref_tests(), conf), tmp)
        os.makedirs(os.path.join(tmp, "output"))
        return refdump.run(conf, os.path.join(tmp, "dump.txt"), forces, steps=steps, cwd=tmp)
    finally:
        shutil.rmtree(tmp)


def synthetic(sysm, stem: str, forces: list[str], cellsize: float, steps: int = 0,
              conf_forces=("Bond",), integrator="Leapfrog", timestep=0.5,
              integrator_params="") -> dict:
    tmp = tempfile.mkdtemp()
    try:
        conf = systems.write_protomol_inputs(sysm, tmp, stem, list(conf_forces),
                                             cellsize=cellsize, outputs=False,
                                             numsteps=max(steps, 20),
                                             integrator=integrator, timestep=timestep,
                                             integrator_params=integrator_params)
        return refdump.run(conf, os.path.join(tmp, "dump.txt"), forces, steps=steps, cwd=tmp)
    finally:
        shutil.rmtree(tmp)


def torsions() -> None:
    """The reference's GB test proteins through its Dihedral and Improper
    forces (periodic cosine torsions and harmonic impropers)."""
    for conf, name in (("www-fip35_FFAMBER_GB_LL.conf", "fip35_torsions"),
                       ("alanylalanine_FFAMBER_GB_LL.conf", "alanylalanine_torsions")):
        save(name, reference_conf(conf, ["Dihedral", "Improper"]))
    # the synthetic heteropolymer (n = 3 backbone dihedrals) through the
    # reference's PSF/PAR reader and its Dihedral/Bond/Angle forces
    poly = systems.gb_polymer(200, seed=3)
    save("polymer200_torsions", synthetic(poly, "poly", ["Dihedral", "Bond", "Angle"],
                                          cellsize=5.0), {"seed": np.array(3)})


def langevin_temperature() -> None:
    """The reference's LangevinLeapfrog thermostat on the 648-atom box with
    its MD forces (1 fs, 5/ps, 300 K): the mean kinetic temperature of steps
    1,000-3,000 (outputs every 20 steps), one run per random seed.  At 1 fs
    the stiff O-H bonds of flexible TIP3P leave the kinetic temperature a
    few per cent above the target in the reference's own integrator."""
    import subprocess
    c1 = systems.tip3p_box(216, 18.6, seed=1, lattice=6)
    md = ["LennardJones Coulomb -algorithm NonbondedCutoff -switchingFunction C2 -switchon 7 "
          "-cutoff 8 -switchingFunction C2 -switchon 7 -cutoff 8 -cutoff 8", "Bond", "Angle"]
    means = []
    seeds = [1234, 5, 6, 7]
    for seed in seeds:
        tmp = tempfile.mkdtemp()
        try:
            conf = systems.write_protomol_inputs(
                c1, tmp, "w", md, integrator="LangevinLeapfrog", timestep=1.0, numsteps=3000,
                cellsize=8.0, outputs=True, outputfreq=20,
                integrator_params=f"temperature 300 gamma 5 seed {seed}")
            text = open(conf).read().replace("seed 1234\n", f"seed {seed}\n", 1)
            open(conf, "w").write(text)
            subprocess.run([refdump.PROTOMOL, conf], cwd=tmp, check=True,
                           stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            rows = [[float(t[0])] + [float.fromhex(x) for x in t[1:]]
                    for t in (ln.split() for ln in open(os.path.join(tmp, "w.out.energy"))) if t]
            rows = np.array(rows)
            means.append(rows[rows[:, 0] > 1000.0, 4].mean())  # Temperature column
        finally:
            shutil.rmtree(tmp)
    np.savez_compressed(os.path.join(HERE, "c1_langevin_temperature.npz"),
                        seeds=np.array(seeds), mean_temperature=np.array(means))
    print("wrote c1_langevin_temperature", means)


def switch_variants() -> None:
    """The remaining switching functions and the lattice sum through the
    reference's own factory.  A 300-atom TIP3P box of 14.4 A (below twice
    the 8 A cutoff, so lattice images beyond the minimal one contribute):
    CmpCnCn on the cutoff path, NonbondedFull (lattice sum) with C1, C2, Cn
    and CmpCnCn, and the all-pairs path in a periodic box (minimal image)
    with C2, Cn and the Complement of C1, C2 and Cn.  The reference's
    vacuum GB protein (www-fip35): the all-pairs path with Complement
    switches."""
    small = systems.tip3p_box(100, 14.4, seed=5, lattice=5)
    d = synthetic(small, "small", [
        "Coulomb -algorithm NonbondedCutoff -switchingFunction ComplimentCnCn -switchon 2 "
        "-switchoff 4 -cutoff 6.5 -n 2 -cutoff 6.5",
        "LennardJones Coulomb -algorithm NonbondedCutoff -switchingFunction ComplimentCnCn "
        "-switchon 2 -switchoff 5 -cutoff 7 -n 3 -switchingFunction ComplimentCnCn "
        "-switchon 1 -switchoff 4 -cutoff 7 -n 4 -cutoff 7",
        "Coulomb -algorithm NonbondedFull -switchingFunction C1 -cutoff 8 -cutoff 8",
        "LennardJones -algorithm NonbondedFull -switchingFunction C2 -switchon 6 -cutoff 8 "
        "-cutoff 8",
        "Coulomb -algorithm NonbondedFull -switchingFunction Cn -n 3 -switchon 5 -cutoff 8 "
        "-cutoff 8",
        "LennardJones -algorithm NonbondedFull -switchingFunction ComplimentCnCn -switchon 2 "
        "-switchoff 5 -cutoff 8 -n 2 -cutoff 8",
        "LennardJones Coulomb -algorithm NonbondedSimpleFull -switchingFunction ComplementC2 "
        "-switchon 5 -cutoff 6 -switchingFunction ComplementC1 -cutoff 6",
        "Coulomb -algorithm NonbondedSimpleFull -switchingFunction ComplementCn -n 2 "
        "-switchon 4 -cutoff 6",
        "LennardJones -algorithm NonbondedSimpleFull -switchingFunction C2 -switchon 4 "
        "-cutoff 6",
        "LennardJones Coulomb -algorithm NonbondedSimpleFull -switchingFunction Cn -n 3 "
        "-switchon 4 -cutoff 6 -switchingFunction Cn -n 2 -switchon 3 -cutoff 6",
        "Bond"], cellsize=6.5)
    save("small_tip3p300_switches", d, {"seed": np.array(5)})
    d = reference_conf("www-fip35_FFAMBER_GB_LL.conf", [
        "Coulomb -algorithm NonbondedSimpleFull -switchingFunction ComplementC1 -cutoff 8",
        "LennardJones -algorithm NonbondedSimpleFull -switchingFunction ComplementCn -n 4 "
        "-switchon 6 -cutoff 9",
        "LennardJones Coulomb -algorithm NonbondedSimpleFull -switchingFunction ComplementC2 "
        "-switchon 7 -cutoff 9 -switchingFunction ComplementC1 -cutoff 9",
        "LennardJones Coulomb -algorithm NonbondedSimpleFull -switchingFunction C2 "
        "-switchon 7 -cutoff 9 -switchingFunction C1 -cutoff 9"])
    save("fip35_switches", d)


def scpism() -> None:
    """The reference's implicit-solvent (SCPISM) systems: its own force
    lines (LennardJones + CoulombSCPISM with Cn switching on NonbondedCutoff,
    BornRadii and BornSelf) and CoulombSCPISM with other switches and -D on
    the cutoff and all-pairs algorithms."""
    forces = [
        "LennardJones CoulombSCPISM -algorithm NonbondedCutoff -switchingFunction Cn -n 4 "
        "-switchon 8.0 -cutoff 20.0 -switchingFunction Cn -n 4 -switchon 8.0 -cutoff 20.0 "
        "-cutoff 20.0",
        "BornRadii -algorithm NonbondedCutoff -switchingFunction Cutoff -bornswitch 3 "
        "-cutoff 5 -cutoff 5",
        "BornSelf -algorithm NonbondedCutoff -switchingFunction Cutoff -bornswitch 3 "
        "-cutoff 5 -cutoff 5",
        "CoulombSCPISM -algorithm NonbondedCutoff -switchingFunction C2 -switchon 0 "
        "-cutoff 12 -cutoff 12 -D 60",
        "CoulombSCPISM -algorithm NonbondedSimpleFull -switchingFunction C1 -cutoff 15",
        "LennardJones CoulombSCPISM -algorithm NonbondedSimpleFull -switchingFunction C2 "
        "-switchon 6 -cutoff 14 -switchingFunction C1 -cutoff 14",
        "BornRadii -algorithm NonbondedCutoff -switchingFunction Cutoff -bornswitch 1 "
        "-cutoff 4 -cutoff 4",
        "BornSelf -algorithm NonbondedCutoff -switchingFunction Cutoff -bornswitch 2 "
        "-cutoff 4.5 -cutoff 4.5 -D 60"]
    save("alanine_scpism", reference_conf("alanine_CHARMM_IMPLICIT_LL.conf", forces))
    save("wwdomain_scpism", reference_conf("wwdomain_CHARMM_IMPLICIT_LL.conf", forces))


def main(which: str = "all") -> None:
    if which == "scpism":
        scpism()
        return
    if which == "switches":
        switch_variants()
        return
    if which == "torsions":
        torsions()
        return
    if which == "langevin":
        langevin_temperature()
        return
    if which == "gb":
        gb = ["GBBornRadii -algorithm NonbondedSimpleFull",
              "GBPartialSum -algorithm NonbondedSimpleFull",
              "GBForce -algorithm NonbondedSimpleFull -soluteDielec 1.0 -solventDielec 78.3",
              "LennardJones -algorithm NonbondedSimpleFull",
              "Coulomb -algorithm NonbondedSimpleFull",
              "GBACEForce -algorithm NonbondedSimpleFull"]
        save("fip35_gb", reference_conf("www-fip35_FFAMBER_GB_LL.conf", gb))
        save("alanylalanine_gb", reference_conf("alanylalanine_FFAMBER_GB_LL.conf", gb))
        return
    if which == "leapfrog100":
        md = ["LennardJones Coulomb -algorithm NonbondedCutoff -switchingFunction C2 -switchon 7 "
              "-cutoff 8 -switchingFunction C2 -switchon 7 -cutoff 8 -cutoff 8", "Bond", "Angle"]
        leapfrog100(systems.tip3p_box(216, 18.6, seed=1, lattice=6), md)
        return
    torsions()
    # 1. The reference's periodic water test (423 atoms, 28 A box).
    d = reference_conf("water_CHARMM_PERIODIC_L.conf", [
        "Coulomb -algorithm NonbondedCutoff -switchingFunction C1 -cutoff 6.5",
        "LennardJones -algorithm NonbondedCutoff -switchingFunction C2 -cutoff 6.5 -switchon 0.1",
        "Bond", "Angle",
        "Coulomb -algorithm FullEwald -real -alpha 0.35 -accuracy 0.0001",
        "Coulomb -algorithm FullEwald -reciprocal -alpha 0.35 -accuracy 0.0001",
        "Coulomb -algorithm FullEwald -correction -alpha 0.35 -accuracy 0.0001",
        "LennardJones Coulomb -algorithm NonbondedCutoff -switchingFunction Cn -n 4 "
        "-switchon 5 -cutoff 8 -switchingFunction Cn -n 3 -switchon 4 -cutoff 8 -cutoff 8",
    ])
    save("water423", d)
    # 2. The reference's GB tests (vacuum, GROMACS topologies).
    gb = ["GBBornRadii -algorithm NonbondedSimpleFull",
          "GBPartialSum -algorithm NonbondedSimpleFull",
          "GBForce -algorithm NonbondedSimpleFull -soluteDielec 1.0 -solventDielec 78.3",
          "LennardJones -algorithm NonbondedSimpleFull",
          "Coulomb -algorithm NonbondedSimpleFull",
          "GBACEForce -algorithm NonbondedSimpleFull"]
    save("fip35_gb", reference_conf("www-fip35_FFAMBER_GB_LL.conf", gb))
    save("alanylalanine_gb", reference_conf("alanylalanine_FFAMBER_GB_LL.conf", gb))
    # 3. Synthetic 648-atom TIP3P box (216 waters, 18.6 A): the small plain
    #    configuration, LJ + Coulomb C2 switching 7 -> 8 A.
    c1 = systems.tip3p_box(216, 18.6, seed=1, lattice=6)
    d = synthetic(c1, "c1", [
        "LennardJones Coulomb -algorithm NonbondedCutoff -switchingFunction C2 -switchon 7 "
        "-cutoff 8 -switchingFunction C2 -switchon 7 -cutoff 8 -cutoff 8",
        "Coulomb -algorithm NonbondedCutoff -switchingFunction C1 -cutoff 8",
        "LennardJones -algorithm NonbondedCutoff -switchingFunction Cn -n 2 -switchon 6 -cutoff 8",
        "LennardJones Coulomb -algorithm NonbondedCutoff -switchingFunction C2 -switchon 7 "
        "-cutoff 8 -switchingFunction C1 -cutoff 8 -cutoff 8",
        "Coulomb -algorithm FullEwald -real -alpha 0.35 -accuracy 0.0001",
        "Coulomb -algorithm FullEwald -reciprocal -alpha 0.35 -accuracy 0.0001",
        "Coulomb -algorithm FullEwald -correction -alpha 0.35 -accuracy 0.0001",
        "Bond", "Angle"], cellsize=8.0)
    save("c1_tip3p648", d, {"seed": np.array(1)})
    # 4. Trajectories of the same box through the reference's integrators:
    #    state after setup and after 20 steps.
    md = ["LennardJones Coulomb -algorithm NonbondedCutoff -switchingFunction C2 -switchon 7 "
          "-cutoff 8 -switchingFunction C2 -switchon 7 -cutoff 8 -cutoff 8", "Bond", "Angle"]
    for tag, integ, dt, prm in (("leapfrog", "Leapfrog", 0.5, ""),
                                ("langevin_t0", "LangevinLeapfrog", 1.0,
                                 "temperature 0 gamma 5 seed 1234")):
        d0 = synthetic(c1, "c1", ["Bond"], 8.0, 0, md, integ, dt, prm)
        d1 = synthetic(c1, "c1", ["Bond"], 8.0, 20, md, integ, dt, prm)
        save(f"c1_{tag}20", d0, {"positions_20": d1["positions"],
                                 "velocities_20": d1["velocities"],
                                 "timestep": np.array(dt), "md_forces": np.array(md)})
    leapfrog100(c1, md)
    langevin_temperature()


def leapfrog100(c1, md) -> None:
    """The small plain configuration as specified: 100 leapfrog steps of
    0.5 fs through the reference's own integrator, with the energies of
    every MD force term at EVERY step (pm_forcedump --steps k for k = 1..100,
    full precision) and the state at steps 25, 50, 75 and 100."""
    d0 = synthetic(c1, "c1", md, 8.0, 0, md, "Leapfrog", 0.5, "")
    per_step = np.zeros((101, 4))
    extra = {"timestep": np.array(0.5), "md_forces": np.array(md)}
    for k in range(0, 101):
        d = d0 if k == 0 else synthetic(c1, "c1", md, 8.0, k, md, "Leapfrog", 0.5, "")
        e = sum(f["energies"] for f in d["forces"])
        per_step[k] = e[[0, 1, 2, 3]]  # COULOMB, LENNARDJONES, BOND, ANGLE
        if k and k % 25 == 0:
            extra[f"positions_{k}"] = d["positions"]
            extra[f"velocities_{k}"] = d["velocities"]
    extra["energies_per_step"] = per_step
    save("c1_leapfrog100", d0, extra)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "all")
