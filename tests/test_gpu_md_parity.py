"""GPU parity of the kernels that MD steps run, at the benchmark
configurations.

The single evaluations in test_gpu_parity.py ask for energies, so they run
the generic pair kernel.  The inner steps of an MD run take the specialised
force-only FP32 kernels (LJ C2 + Ewald real space; LJ C2 + Coulomb C2/C1),
which a force-only evaluation (pmgpu_evaluate with no energy or virial
output) also runs.  The tests here pin those kernels, and whole MD runs,
against the FP64 oracle (itself pinned to the reference's outputs in
test_oracle_pins.py) and against the reference's own trajectories:

  * the 648-atom TIP3P box, leapfrog 0.5 fs x 100 steps, FP64 throughout,
    energies of every step and the state every 25 steps against the
    reference's run; in mixed precision the force-only forces at every
    step's positions against the oracle;
  * the 23,550-atom TIP3P box with PME (alpha 0.35, rc 9, order 4, 64^3),
    LJ C2 8 -> 9 A, bonds and angles, leapfrog 1 fs: forces and energies
    against the oracle at steps 0, 100 and 1,000;
  * the 2,000-atom GB heteropolymer with LangevinLeapfrog at 300 K: forces
    and energies against the oracle at steps 0 and 500.

Tolerances: RMS relative force error <= 1e-5 and energy relative error
<= 1e-6 (absolute floor 1e-4 kcal/mol) in mixed precision; FP64 runs
<= 1e-8 relative on energies and 1e-8 A on positions.
"""
import math

import numpy as np
import pytest

import fixtures as F
import oracle
from oracle import spme
from protomol_b200 import (ForceFactory, GpuSystem, LangevinLeapfrogIntegrator,
                           LeapfrogIntegrator, PMEwaldSystemForce, ScalarStructure, systems)
from protomol_b200._lib import PmgpuError

pytestmark = pytest.mark.gpu

RMS_MIXED = 1e-5
E_REL = 1e-6


def _energy_ok(got, want, rel=E_REL, floor=1e-4):
    return abs(got - want) <= max(rel * abs(want), floor)


def _ewald(s, alpha, rc, exact_erf=False):
    """FullEwald parameters at exactly rc (accuracy exp(-(alpha rc)^2))."""
    ew = oracle.ewald_params(s, alpha, math.exp(-(alpha * rc) ** 2), exact_erf)
    ew.rc = rc
    return ew


def _oracle_pme_md(s, topo, alpha, rc, order, K, lj_switchon):
    """Oracle forces and energies of the PME MD force set: LJ C2 cutoff,
    Ewald real + SPME reciprocal + exclusion correction + self terms,
    bonds and angles."""
    sw = oracle.Switch("C2", rc, lj_switchon)
    f, e, _ = oracle.cutoff_force(s, rc, rc, [("LennardJones", sw)])
    ew = _ewald(s, alpha, rc)
    fr, er, _ = oracle.ewald_real(s, ew, rc)
    fk, ek = spme.reciprocal(s.pos, s.charge, s.box, alpha, order, K)
    fc, ec, _ = oracle.ewald_correction(s, ew)
    es, eq = oracle.ewald_self(s, ew)
    fb, eb, _ = oracle.bonded_force(s, topo.bonds, topo.bond_params, topo.angles,
                                    topo.angle_params)
    return f + fr + fk + fc + fb, {"coulomb": er + ek + ec + es + eq, "lj": e["lj"],
                                   "bond": eb["bond"], "angle": eb["angle"]}


@pytest.mark.parametrize("name,rc,switchon", [("c1_tip3p648", 8.0, 7.0), ("water423", 6.5, 0.1)])
def test_force_only_lj_ewald_kernel_vs_oracle(ctx, name, rc, switchon):
    """LJ C2 + Ewald real space on one list, evaluated force-only: the
    specialised kernel the 23,550-atom benchmark's MD steps run, against
    the oracle's cutoff LJ and FullEwald real term, at the fixture's
    positions and after 20 LangevinLeapfrog steps at 300 K."""
    z = F.load(name)
    topo = F.topology(z)
    gs = GpuSystem(ctx, topo, "mixed")
    ff = ForceFactory(gs, rc)
    lj = ff.make(f"LennardJones -algorithm NonbondedCutoff -switchingFunction C2 "
                 f"-switchon {switchon} -cutoff {rc} -cutoff {rc}")
    PMEwaldSystemForce(gs, 0.35, rc, real=True, reciprocal=False, correction=False)
    sw = oracle.Switch("C2", rc, switchon)
    for stage in range(2):
        if stage:
            ff.make("Bond")
            ff.make("Angle")
            LangevinLeapfrogIntegrator(1.0, temperature=300.0, gamma=5.0, seed=3).run(gs, 20)
            for f in gs.forces[2:]:
                f.set_enabled(False)
        f_gpu = gs.evaluate_forces()
        assert lj.stats()["pair_kernel"] == "lj_c2+ewald"
        s = F.oracle_system(z).with_positions(gs.positions())
        fo, _, _ = oracle.cutoff_force(s, rc, rc, [("LennardJones", sw)])
        fr, _, _ = oracle.ewald_real(s, _ewald(s, 0.35, rc), rc)
        err = F.rms_rel(f_gpu, fo + fr)
        assert err <= RMS_MIXED, (stage, err)
    gs.close()


def test_c1_leapfrog100_fp64_every_step_vs_reference(ctx):
    """The small plain configuration as specified: 648-atom TIP3P box, LJ +
    Coulomb C2 7 -> 8 A, bonds, angles, leapfrog 0.5 fs, FP64 throughout,
    100 steps; the energies of every term at every step against the
    reference's own run, and positions and velocities at steps 25, 50, 75
    and 100."""
    z = F.load("c1_leapfrog100")
    topo = F.topology(z)
    gs = GpuSystem(ctx, topo, "double")
    ff = ForceFactory(gs, 8.0)
    for line in z["md_forces"]:
        ff.make(str(line))
    it = LeapfrogIntegrator(float(z["timestep"]))
    ref = z["energies_per_step"]
    e0, _ = gs.evaluate()
    assert np.abs(e0[:4] - ref[0]).max() <= 1e-8 * np.abs(ref[0]).max()
    worst = 0.0
    for k in range(1, 101):
        it.run(gs, 1)
        e, _ = gs.energies()
        d = np.abs(e[:4] - ref[k]).max() / np.abs(ref[k]).max()
        worst = max(worst, d)
        assert d <= 1e-8, (k, e[:4], ref[k])
        if k % 25 == 0:
            x, v = gs.positions(), gs.velocities()
            assert np.abs(x - z[f"positions_{k}"].reshape(-1, 3)).max() <= 1e-8, k
            vr = z[f"velocities_{k}"].reshape(-1, 3)
            assert np.abs(v - vr).max() <= 1e-8 * np.abs(vr).max(), k
    gs.close()


def test_c1_leapfrog100_mixed_forces_every_step_vs_oracle(ctx):
    """The same 100 steps in mixed precision: at every step's positions the
    force-only evaluation (the LJ C2 + Coulomb C2 kernel of the inner steps,
    plus bonds and angles) against the oracle's forces, and the step's
    energies against the oracle's at the same positions."""
    z = F.load("c1_leapfrog100")
    topo = F.topology(z)
    gs = GpuSystem(ctx, topo, "mixed")
    ff = ForceFactory(gs, 8.0)
    forces = [ff.make(str(line)) for line in z["md_forces"]]
    it = LeapfrogIntegrator(float(z["timestep"]))
    s0 = F.oracle_system(z)
    sw = oracle.Switch("C2", 8.0, 7.0)
    worst = 0.0
    for k in range(1, 101):
        it.run(gs, 1)
        e, _ = gs.energies()
        x = gs.positions()
        s = s0.with_positions(x)
        fo, eo, _ = oracle.cutoff_force(s, 8.0, 8.0, [("LennardJones", sw), ("Coulomb", sw)])
        fb, eb, _ = oracle.bonded_force(s, topo.bonds, topo.bond_params, topo.angles,
                                        topo.angle_params)
        for slot, want in ((0, eo["coulomb"]), (1, eo["lj"]), (2, eb["bond"]),
                           (3, eb["angle"])):
            assert _energy_ok(e[slot], want), (k, slot, e[slot], want)
        fg = gs.evaluate_forces()
        assert forces[0].stats()["pair_kernel"] == "lj_c2+coulomb_c2"
        err = F.rms_rel(fg, fo + fb)
        worst = max(worst, err)
        assert err <= RMS_MIXED, (k, err)
    # the mixed trajectory stays on the reference's within FP32 rounding
    # growth over 100 steps
    assert np.abs(gs.positions() - z["positions_100"].reshape(-1, 3)).max() <= 1e-3
    gs.close()


def _c2_system():
    return systems.tip3p_box(7850, 62.0, 2024, jitter=0.3, lattice=20)


def test_c2_configuration_vs_oracle_at_steps_0_100_1000(ctx):
    """The solvated benchmark system exactly as benched: 7,850 TIP3P waters
    (23,550 atoms) in a 62 A box, Ewald real 9 A + PME order 4 on 64^3
    (alpha 0.35) + exclusion correction, LJ C2 8 -> 9 A, bonds, angles,
    leapfrog 1 fs.  At steps 0, 100 and 1,000 of the device run, the
    force-only forces (the kernels the MD steps run) against the oracle at
    the device's positions, at RMS relative error <= 1e-5, and the FP64
    energies of an evaluation there against the oracle's at 1e-6."""
    sysm = _c2_system()
    gs = GpuSystem(ctx, sysm, "mixed")
    ff = ForceFactory(gs, 9.0)
    ff.make("Bond")
    ff.make("Angle")
    lj = ff.make("LennardJones -algorithm NonbondedCutoff -switchingFunction C2 -switchon 8.0 "
                 "-cutoff 9.0 -cutoff 9.0")
    ff.make("Coulomb -algorithm PMEwald -alpha 0.35 -cutoff 9.0 -order 4 -gridsize 64 64 64")
    it = LeapfrogIntegrator(1.0)
    s0 = oracle.System(pos=sysm.pos, charge=sysm.charge, type=sysm.type,
                       molecule=sysm.molecule, lj=sysm.lj, excl=sysm.exclusions,
                       periodic=True, box=sysm.box, mass=sysm.mass)
    done = 0
    for step in (0, 100, 1000):
        if step > done:
            it.run(gs, step - done)
            done = step
        x = gs.positions()
        fg = gs.evaluate_forces()
        assert lj.stats()["pair_kernel"] == "lj_c2+ewald"
        s = s0.with_positions(x)
        fo, eo = _oracle_pme_md(s, sysm, 0.35, 9.0, 4, 64, 8.0)
        err = F.rms_rel(fg, fo)
        assert err <= RMS_MIXED, (step, err)
        e, _ = gs.evaluate()
        for slot, key in ((0, "coulomb"), (1, "lj"), (2, "bond"), (3, "angle")):
            assert _energy_ok(e[slot], eo[key]), (step, key, e[slot], eo[key])
    gs.close()


def test_gb_polymer2000_vs_oracle_at_steps_0_and_500(ctx):
    """The implicit-solvent configuration: 2,000-atom heteropolymer, GB OBC2
    (solvent 78.5) + LJ + Coulomb all pairs, bonds, angles, dihedrals;
    forces (force-only) and energies against the oracle at the start and
    after 500 LangevinLeapfrog steps (1 fs, 5/ps, 300 K)."""
    sm = systems.gb_polymer(2000, 3)
    gs = GpuSystem(ctx, sm, "mixed")
    ff = ForceFactory(gs)
    for line in ("GBBornRadii -algorithm NonbondedSimpleFull",
                 "GBPartialSum -algorithm NonbondedSimpleFull",
                 "GBForce -algorithm NonbondedSimpleFull -soluteDielec 1.0 -solventDielec 78.5",
                 "LennardJones -algorithm NonbondedSimpleFull",
                 "Coulomb -algorithm NonbondedSimpleFull", "Bond", "Angle", "Dihedral"):
        ff.make(line)
    for step in (0, 500):
        if step:
            LangevinLeapfrogIntegrator(1.0, 300.0, 5.0, seed=3).run(gs, step)
        x = gs.positions()
        fg = gs.evaluate_forces()
        s = oracle.System(pos=x, charge=sm.charge, type=sm.type, molecule=sm.molecule,
                          lj=sm.lj, excl=sm.exclusions, periodic=False, box=sm.box,
                          mass=sm.mass, water=sm.water, gb_vdwr=sm.gb_vdwr,
                          gb_scale=sm.gb_scale, gb_offset=sm.gb_offset, gb_obc=sm.gb_obc)
        fgb, egb, _ = oracle.gb_force(s, 1.0, 78.5)
        flj, elj, _ = oracle.simplefull_force(s, "LennardJones")
        fco, eco, _ = oracle.simplefull_force(s, "Coulomb")
        fb, eb, _ = oracle.bonded_force(s, sm.bonds, sm.bond_params, sm.angles, sm.angle_params)
        ft, et, _ = oracle.torsion_force(s, sm.dihedrals, sm.dihedral_params)
        err = F.rms_rel(fg, fgb + flj + fco + fb + ft)
        assert err <= RMS_MIXED, (step, err)
        e, _ = gs.evaluate()
        for slot, want in ((0, egb + eco["coulomb"]), (1, elj["lj"]), (2, eb["bond"]),
                           (3, eb["angle"]), (4, et)):
            assert _energy_ok(e[slot], want), (step, slot, e[slot], want)
    gs.close()


@pytest.mark.parametrize("precision,tol", [("mixed", RMS_MIXED), ("double", 1e-8)])
def test_cutoff_switch_on_the_cutoff_path_vs_oracle(ctx, precision, tol):
    """The Cutoff switching function (a step at the cutoff,
    switch/CutoffSwitchingFunction.h:41-44) on LJ and Coulomb cutoff
    forces, alone and beside a C2 term (OneAtomPairTwo then switches both),
    against the oracle.  Universal is not a cutoff switch: ProtoMol's
    factory registers it for NonbondedCutoff only with the tabulated LJ
    force (module/NonbondedCutoffForceModule.cpp:55-96), and the GPU path
    rejects it on a cutoff force with an argument error."""
    z = F.load("c1_tip3p648")
    topo = F.topology(z)
    gs = GpuSystem(ctx, topo, precision)
    ff = ForceFactory(gs, 8.0)
    s = F.oracle_system(z)
    cut = oracle.Switch("Cutoff", 8.0)
    c2 = oracle.Switch("C2", 8.0, 7.0)
    for line, terms in (
            ("LennardJones Coulomb -algorithm NonbondedCutoff -switchingFunction Cutoff -cutoff 8 "
             "-switchingFunction Cutoff -cutoff 8 -cutoff 8",
             [("LennardJones", cut), ("Coulomb", cut)]),
            ("LennardJones Coulomb -algorithm NonbondedCutoff -switchingFunction C2 -switchon 7 "
             "-cutoff 8 -switchingFunction Cutoff -cutoff 8 -cutoff 8",
             [("LennardJones", c2), ("Coulomb", cut)]),
            ("Coulomb -algorithm NonbondedCutoff -switchingFunction Cutoff -cutoff 8",
             [("Coulomb", cut)])):
        force = ff.make(line)
        f = np.zeros_like(topo.pos)
        e = ScalarStructure()
        force.evaluate(topo.pos, f, e)
        fo, eo, _ = oracle.cutoff_force(s, 8.0, 8.0, terms)
        assert F.rms_rel(f, fo) <= tol, (line, F.rms_rel(f, fo))
        assert _energy_ok(e[0], eo["coulomb"]), line
        assert _energy_ok(e[1], eo["lj"]), line
        force.set_enabled(False)
    with pytest.raises(PmgpuError):
        ff.make("LennardJones -algorithm NonbondedCutoff -switchingFunction Universal -cutoff 8")
    gs.close()
