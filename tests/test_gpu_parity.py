"""GPU parity: the CUDA path (libpmgpu through the C ABI) against the
ProtoMol reference's own outputs (golden fixtures) and the FP64 oracle.

Tolerances (stated per the FP32-pair / FP64-accumulate design):
  * mixed precision: RMS relative force error <= 1e-5 per force term,
    energy relative error <= 1e-6 (abs floor 1e-4 kcal/mol);
  * double precision ("FP64 throughout"): RMS relative force error <= 1e-8;
  * the cutoff pair set and the cell assignment are bit-exact.
"""
import numpy as np
import pytest

import fixtures as F
import oracle
from protomol_b200 import (ForceFactory, GpuSystem, LangevinLeapfrogIntegrator,
                           LeapfrogIntegrator, PMEwaldSystemForce, ScalarStructure)

pytestmark = pytest.mark.gpu

RMS_MIXED = 1e-5
RMS_DOUBLE = 1e-8
E_REL = 1e-6


def _energy_ok(got, want, rel=E_REL, floor=1e-4):
    return abs(got - want) <= max(rel * abs(want), floor)


def _eval(force, topo):
    f = np.zeros((topo.pos.shape[0], 3))
    e = ScalarStructure()
    force.evaluate(topo.pos, f, e, virial=True)
    return f, e


@pytest.mark.parametrize("precision,tol", [("mixed", RMS_MIXED), ("double", RMS_DOUBLE)])
@pytest.mark.parametrize("name,cellsize", [("water423", 6.5), ("c1_tip3p648", 8.0)])
def test_cutoff_forces_vs_reference(ctx, name, cellsize, precision, tol):
    z = F.load(name)
    topo = F.topology(z)
    gs = GpuSystem(ctx, topo, precision)
    ff = ForceFactory(gs, cellsize)
    n = 0
    for k, d in enumerate(z["defs"]):
        d = str(d)
        if "NonbondedCutoff" not in d:
            continue
        force = ff.make(d)
        f, e = _eval(force, topo)
        ref_f, ref_e = F.forces(z, k), F.energies(z, k)
        err = F.rms_rel(f, ref_f)
        assert err <= tol, (d, err)
        assert _energy_ok(e[0], ref_e[0]), (d, e[0], ref_e[0])
        assert _energy_ok(e[1], ref_e[1]), (d, e[1], ref_e[1])
        vir_err = np.abs(e[7:16] - ref_e[7:16]).max() / max(np.abs(ref_e[7:16]).max(), 1)
        assert vir_err <= 1e-5, (d, vir_err)
        n += 1
    assert n >= 3
    gs.close()


@pytest.mark.parametrize("name,cellsize", [("water423", 6.5), ("c1_tip3p648", 8.0)])
def test_pair_set_and_cells_bit_exact(ctx, name, cellsize):
    z = F.load(name)
    topo = F.topology(z)
    s = F.oracle_system(z)
    gs = GpuSystem(ctx, topo, "mixed")
    rc = 8.0 if name.startswith("c1") else 6.5
    line = (f"LennardJones Coulomb -algorithm NonbondedCutoff -switchingFunction C2 -switchon "
            f"{rc - 1} -cutoff {rc} -switchingFunction C1 -cutoff {rc} -cutoff {rc}")
    force = ForceFactory(gs, cellsize).make(line)
    got = force.pair_set()
    want = oracle.cutoff_pairs(s, cellsize, rc, rc)[:, :2]
    got = np.unique(np.sort(got, axis=1), axis=0)
    want = np.unique(np.sort(want, axis=1), axis=0)
    assert got.shape == want.shape
    assert np.array_equal(got, want)
    cells, dims = gs.cell_assign(cellsize)
    ocells, odims = oracle.cell_assign(s, cellsize)
    assert tuple(dims) == tuple(odims)
    assert np.array_equal(cells, ocells)
    gs.close()


@pytest.mark.parametrize("precision,tol", [("mixed", RMS_MIXED), ("double", RMS_DOUBLE)])
@pytest.mark.parametrize("name", ["water423", "c1_tip3p648"])
def test_ewald_real_and_correction_vs_reference(ctx, name, precision, tol):
    z = F.load(name)
    topo = F.topology(z)
    gs = GpuSystem(ctx, topo, precision)
    alpha = 0.35
    rc = np.sqrt(-np.log(1e-4)) / alpha  # Rc of FullEwald -accuracy 1e-4
    k_real = [k for k, d in enumerate(z["defs"]) if "FullEwald -real" in str(d)][0]
    k_corr = [k for k, d in enumerate(z["defs"]) if "FullEwald -correction" in str(d)][0]
    real = PMEwaldSystemForce(gs, alpha, rc, real=True, reciprocal=False, correction=False)
    corr = PMEwaldSystemForce(gs, alpha, rc, real=False, reciprocal=False, correction=True)
    f, e = _eval(real, topo)
    assert F.rms_rel(f, F.forces(z, k_real)) <= tol
    assert _energy_ok(e[0], F.energies(z, k_real)[0])
    f, e = _eval(corr, topo)
    assert F.rms_rel(f, F.forces(z, k_corr)) <= 1e-10  # FP64 kernel
    assert _energy_ok(e[0], F.energies(z, k_corr)[0], rel=1e-10, floor=1e-8)
    gs.close()


@pytest.mark.parametrize("name", ["water423", "c1_tip3p648"])
def test_pme_reciprocal_vs_spme_restatement_and_full_ewald(ctx, name):
    from oracle import spme
    z = F.load(name)
    topo = F.topology(z)
    gs = GpuSystem(ctx, topo, "mixed")
    L = topo.box[0]
    for order, K in ((4, 32), (6, 48)):
        rec = PMEwaldSystemForce(gs, 0.35, 0.0, order=order, grid=(K, K, K), real=False,
                                 reciprocal=True, correction=False)
        f, e = _eval(rec, topo)
        fo, eo = spme.reciprocal(topo.pos, topo.charge, L, 0.35, order, K)
        # matched grid, order and alpha: FP32 FFT/B-spline vs FP64 restatement
        assert F.rms_rel(f, fo) <= 1e-5, (order, K, F.rms_rel(f, fo))
        assert _energy_ok(e[0], eo, rel=1e-5)
        rec.set_enabled(False)
    # Converged PME approaches the reference's full Ewald k-sum (its
    # algorithm, via the reference-pinned oracle, at accuracy 1e-14 so the
    # k-sphere truncation is below FP32 resolution).
    s = F.oracle_system(z)
    fk, ek, _ = oracle.ewald_reciprocal(s, oracle.ewald_params(s, 0.35, 1e-14))
    rec = PMEwaldSystemForce(gs, 0.35, 0.0, order=8, grid=(64, 64, 64), real=False,
                             reciprocal=True, correction=False)
    f, e = _eval(rec, topo)
    assert F.rms_rel(f, fk) <= 1e-5, F.rms_rel(f, fk)
    assert _energy_ok(e[0], ek, rel=1e-5)
    gs.close()


@pytest.mark.parametrize("precision,tol", [("mixed", RMS_MIXED), ("double", RMS_DOUBLE)])
@pytest.mark.parametrize("name", ["fip35_gb", "alanylalanine_gb"])
def test_gb_and_simplefull_vs_reference(ctx, name, precision, tol):
    z = F.load(name)
    topo = F.topology(z)
    gs = GpuSystem(ctx, topo, precision)
    ff = ForceFactory(gs)
    gb = ff.make("GBForce -algorithm NonbondedSimpleFull -soluteDielec 1.0 -solventDielec 78.3")
    f, e = _eval(gb, topo)
    assert F.rms_rel(f, F.forces(z, 2)) <= tol, F.rms_rel(f, F.forces(z, 2))
    assert _energy_ok(e[0], F.energies(z, 2)[0])
    for k, line, slot in ((3, "LennardJones -algorithm NonbondedSimpleFull", 1),
                          (4, "Coulomb -algorithm NonbondedSimpleFull", 0)):
        fc = ff.make(line)
        f, e = _eval(fc, topo)
        assert F.rms_rel(f, F.forces(z, k)) <= tol, line
        assert _energy_ok(e[slot], F.energies(z, k)[slot])
    gs.close()


def test_bonded_vs_reference(ctx):
    z = F.load("water423")
    topo = F.topology(z)
    gs = GpuSystem(ctx, topo, "mixed")
    ff = ForceFactory(gs)
    for k, line, slot in ((2, "Bond", 2), (3, "Angle", 3)):
        f, e = _eval(ff.make(line), topo)
        assert F.rms_rel(f, F.forces(z, k)) <= 1e-10
        assert _energy_ok(e[slot], F.energies(z, k)[slot], rel=1e-10, floor=1e-8)
    gs.close()


@pytest.mark.parametrize("precision,tol", [("double", 1e-8), ("mixed", 2e-4)])
@pytest.mark.parametrize("tag,integ", [("leapfrog", "leapfrog"), ("langevin_t0", "langevin")])
def test_trajectory_vs_reference(ctx, tag, integ, precision, tol):
    """20 steps of the device integrator against the reference's own
    Leapfrog / LangevinLeapfrog (temperature 0, so the noise term is zero)."""
    z = F.load(f"c1_{tag}20")
    topo = F.topology(z)
    gs = GpuSystem(ctx, topo, precision)
    ff = ForceFactory(gs, 8.0)
    for line in z["md_forces"]:
        ff.make(str(line))
    dt = float(z["timestep"])
    it = LeapfrogIntegrator(dt) if integ == "leapfrog" else \
        LangevinLeapfrogIntegrator(dt, temperature=0.0, gamma=5.0, seed=1234)
    it.run(gs, 20)
    x = gs.positions()
    v = gs.velocities()
    dx = np.abs(x - z["positions_20"].reshape(-1, 3)).max()
    dv = np.abs(v - z["velocities_20"].reshape(-1, 3)).max() / np.abs(z["velocities_20"]).max()
    assert dx <= tol, dx
    assert dv <= 10 * tol, dv
    gs.close()


def test_run_segmentation_invariance(ctx):
    """run(20) equals run(7) + run(13) bit for bit (forces stay resident
    between calls as ProtoMol keeps myForces; fixed-point sums)."""
    z = F.load("c1_leapfrog20")
    out = []
    for split in ((20,), (7, 13)):
        topo = F.topology(z)
        gs = GpuSystem(ctx, topo, "mixed")
        ff = ForceFactory(gs, 8.0)
        for line in z["md_forces"]:
            ff.make(str(line))
        it = LangevinLeapfrogIntegrator(1.0, temperature=300.0, gamma=5.0, seed=99)
        for n in split:
            it.run(gs, n)
        out.append((gs.positions(), gs.velocities()))
        gs.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


def test_graph_replay_equals_eager(ctx):
    """Inner steps replayed from captured CUDA graphs give bit-identical
    trajectories to eager launches (profiling on forces the eager path)."""
    z = F.load("c1_leapfrog20")
    out = []
    for eager in (True, False):
        topo = F.topology(z)
        gs = GpuSystem(ctx, topo, "mixed")
        ff = ForceFactory(gs, 8.0)
        for line in z["md_forces"]:
            ff.make(str(line))
        gs.profile(enable=eager)
        LangevinLeapfrogIntegrator(1.0, temperature=300.0, gamma=5.0, seed=7).run(gs, 25)
        out.append((gs.positions(), gs.velocities(), gs.energies()[0]))
        gs.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][2], out[1][2])


@pytest.mark.parametrize("name", ["fip35_torsions", "alanylalanine_torsions", "polymer200_torsions"])
def test_torsions_vs_reference(ctx, name):
    """Dihedral force (FP64 kernel) against the reference's own output."""
    z = F.load(name)
    topo = F.topology(z)
    gs = GpuSystem(ctx, topo, "mixed")
    f, e = _eval(ForceFactory(gs).make("Dihedral"), topo)
    # FP64 arithmetic; the int64 fixed-point force sums resolve 2^-32
    # kcal/mol/A, about 1e-9 of these small torsion forces
    assert F.rms_rel(f, F.forces(z, 0)) <= 1e-8
    assert _energy_ok(e[4], F.energies(z, 0)[4], rel=1e-10, floor=1e-8)
    gs.close()


def test_list_follows_uploaded_positions(ctx):
    """The pair list is rebuilt whenever the positions handed in lie more
    than half the skin from those of the last build, so evaluations at
    configurations handed in between calls (the whole box shifted by
    1-1.5 A, which changes the periodic images of atoms near the faces, and
    every molecule moved by 0.05-0.2 A) still match the oracle at each
    configuration."""
    z = F.load("c1_tip3p648")
    topo = F.topology(z)
    gs = GpuSystem(ctx, topo, "mixed")
    ff = ForceFactory(gs, 8.0)
    line = ("LennardJones Coulomb -algorithm NonbondedCutoff -switchingFunction C2 "
            "-switchon 7 -cutoff 8 -switchingFunction C2 -switchon 7 -cutoff 8 -cutoff 8")
    force = ff.make(line)
    terms = [("LennardJones", oracle.Switch("C2", 8.0, 7.0)),
             ("Coulomb", oracle.Switch("C2", 8.0, 7.0))]
    rng = np.random.default_rng(5)
    pos = topo.pos.copy()
    mol = topo.molecule
    for k in range(4):
        if k:
            shift = rng.normal(size=3)
            pos += shift / np.linalg.norm(shift) * rng.uniform(1.0, 1.5)
            for m in np.unique(mol):
                v = rng.normal(size=3)
                pos[mol == m] += v / np.linalg.norm(v) * rng.uniform(0.05, 0.2)
        f = np.zeros_like(pos)
        e = ScalarStructure()
        force.evaluate(pos, f, e)
        s = F.oracle_system(z)
        s.pos = pos.copy()
        fo, eo, _ = oracle.cutoff_force(s, 8.0, 8.0, terms)
        err = F.rms_rel(f, fo)
        assert err <= RMS_MIXED, (k, err)
    assert force.stats()["list_builds"] >= 4
    gs.close()


@pytest.mark.parametrize("table", ["charmm_rule", "nbfix"])
def test_polymer_all_pairs_vs_oracle(ctx, table):
    """GB, LJ and Coulomb all pairs of a 700-atom heteropolymer (one LJ type
    per atom) in the mixed FP32 form against the FP64 oracle.  Its table
    follows the CHARMM rule, so the LJ pass computes (A, B) from per-type
    parameters; "nbfix" scales the (A, B) of one off-diagonal pair in every
    seventh row, which the rule cannot express, so the pass reads the table."""
    import oracle
    from protomol_b200 import systems
    sm = systems.gb_polymer(700, seed=5)
    if table == "nbfix":
        lj = sm.lj.copy()
        nt = lj.shape[0]
        for t in range(0, nt, 7):
            u = (13 * t + 5) % nt
            if u != t:
                lj[t, u, :2] *= 1.25
                lj[u, t, :2] = lj[t, u, :2]
        sm.lj = lj
    s = oracle.System(pos=sm.pos, charge=sm.charge, type=sm.type, molecule=sm.molecule,
                      lj=sm.lj, excl=sm.exclusions, periodic=False, box=sm.box, mass=sm.mass,
                      water=sm.water, gb_vdwr=sm.gb_vdwr, gb_scale=sm.gb_scale,
                      gb_offset=sm.gb_offset, gb_obc=sm.gb_obc)
    gs = GpuSystem(ctx, sm, "mixed")
    ff = ForceFactory(gs)
    rf, re, _ = oracle.gb_force(s, 1.0, 78.5)
    f, e = _eval(ff.make("GBForce -algorithm NonbondedSimpleFull -soluteDielec 1.0 "
                         "-solventDielec 78.5"), sm)
    assert F.rms_rel(f, rf) <= RMS_MIXED, F.rms_rel(f, rf)
    assert _energy_ok(e[0], re)
    for line, pot, slot, key in (("LennardJones -algorithm NonbondedSimpleFull", "LennardJones",
                                  1, "lj"),
                                 ("Coulomb -algorithm NonbondedSimpleFull", "Coulomb", 0,
                                  "coulomb")):
        rf, re, rv = oracle.simplefull_force(s, pot)
        f, e = _eval(ff.make(line), sm)
        assert F.rms_rel(f, rf) <= RMS_MIXED, (line, F.rms_rel(f, rf))
        assert _energy_ok(e[slot], re[key]), (line, e[slot], re[key])
        vir_err = np.abs(e[7:16] - rv.ravel()).max() / max(np.abs(rv).max(), 1)
        assert vir_err <= 1e-5, (line, vir_err)
    gs.close()


@pytest.mark.parametrize("n", [1, 2, 3, 31, 33, 65])
def test_all_pairs_small_and_ragged_sizes(ctx, n):
    """The half-pair tile sweeps at sizes below one tile, at a tile and a
    bit, and with a ragged last tile: GB, LJ and Coulomb of a short polymer
    (its exclusions fall on the diagonal and first off-diagonal tiles)
    against the FP64 oracle."""
    import oracle
    from protomol_b200 import systems
    sm = systems.gb_polymer(n, seed=7)
    s = oracle.System(pos=sm.pos, charge=sm.charge, type=sm.type, molecule=sm.molecule,
                      lj=sm.lj, excl=sm.exclusions, periodic=False, box=sm.box, mass=sm.mass,
                      water=sm.water, gb_vdwr=sm.gb_vdwr, gb_scale=sm.gb_scale,
                      gb_offset=sm.gb_offset, gb_obc=sm.gb_obc)
    gs = GpuSystem(ctx, sm, "mixed")
    ff = ForceFactory(gs)
    rf, re, _ = oracle.gb_force(s, 1.0, 78.5)
    f, e = _eval(ff.make("GBForce -algorithm NonbondedSimpleFull -soluteDielec 1.0 "
                         "-solventDielec 78.5"), sm)
    if n > 1:
        assert F.rms_rel(f, rf) <= RMS_MIXED, F.rms_rel(f, rf)
    else:
        assert np.abs(f).max() == 0.0
    assert _energy_ok(e[0], re)
    for line, pot, slot, key in (("LennardJones -algorithm NonbondedSimpleFull", "LennardJones",
                                  1, "lj"),
                                 ("Coulomb -algorithm NonbondedSimpleFull", "Coulomb", 0,
                                  "coulomb")):
        rf, re, _ = oracle.simplefull_force(s, pot)
        f, e = _eval(ff.make(line), sm)
        if np.abs(rf).max() > 0:
            assert F.rms_rel(f, rf) <= RMS_MIXED, (line, F.rms_rel(f, rf))
        else:
            assert np.abs(f).max() == 0.0, line
        assert _energy_ok(e[slot], re[key]), (line, e[slot], re[key])
    gs.close()


def test_polymer_leapfrog_force_only_steps_vs_oracle(ctx):
    """Ten leapfrog steps of a 300-atom polymer under GB + LJ + Coulomb all
    pairs: the inner MD steps take the force-only kernels (no energies),
    which the single evaluations above never run; the trajectory is
    integrated on the host with the FP64 oracle's forces beside it
    (LeapfrogIntegrator.cpp:33-104: half kick, drift, forces, half kick)."""
    import oracle
    from protomol_b200 import systems
    sm = systems.gb_polymer(300, seed=21)
    lines = ["GBBornRadii -algorithm NonbondedSimpleFull",
             "GBPartialSum -algorithm NonbondedSimpleFull",
             "GBForce -algorithm NonbondedSimpleFull -soluteDielec 1.0 -solventDielec 78.5",
             "LennardJones -algorithm NonbondedSimpleFull",
             "Coulomb -algorithm NonbondedSimpleFull"]
    gs = GpuSystem(ctx, sm, "mixed")
    ff = ForceFactory(gs)
    for line in lines:
        ff.make(line)
    steps, dt = 10, 1.0
    LeapfrogIntegrator(dt).run(gs, steps)
    x_gpu, v_gpu = gs.positions(), gs.velocities()
    gs.close()

    def forces(pos):
        s = oracle.System(pos=pos, charge=sm.charge, type=sm.type, molecule=sm.molecule,
                          lj=sm.lj, excl=sm.exclusions, periodic=False, box=sm.box,
                          mass=sm.mass, water=sm.water, gb_vdwr=sm.gb_vdwr,
                          gb_scale=sm.gb_scale, gb_offset=sm.gb_offset, gb_obc=sm.gb_obc)
        return (oracle.gb_force(s, 1.0, 78.5)[0] + oracle.simplefull_force(s, "LennardJones")[0]
                + oracle.simplefull_force(s, "Coulomb")[0])

    h = dt * oracle.INV_TIMEFACTOR
    x, v = sm.pos.copy(), sm.vel.copy()
    f = forces(x)
    for _ in range(steps):
        v = oracle.kick(sm.mass, f, 0.5 * h, v)
        x = oracle.drift(v, h, x)
        f = forces(x)
        v = oracle.kick(sm.mass, f, 0.5 * h, v)
    assert np.abs(x_gpu - x).max() <= 1e-6, np.abs(x_gpu - x).max()
    assert np.abs(v_gpu - v).max() / np.abs(v).max() <= 1e-5


@pytest.mark.parametrize("precision,tol", [("mixed", RMS_MIXED), ("double", RMS_DOUBLE)])
@pytest.mark.parametrize("name", ["fip35_gb", "alanylalanine_gb"])
def test_gbace_vs_reference(ctx, name, precision, tol):
    """GBACEForce (ACE nonpolar term on the OBC Born radii) alone and
    evaluated together with GBForce (one shared Born-radius chain) against
    the reference's own forces and energies."""
    z = F.load(name)
    topo = F.topology(z)
    k_ace = [k for k, d in enumerate(z["defs"]) if str(d).startswith("GBACEForce")][0]
    gs = GpuSystem(ctx, topo, precision)
    ff = ForceFactory(gs)
    ace = ff.make("GBACEForce -algorithm NonbondedSimpleFull")
    f, e = _eval(ace, topo)
    ref = F.forces(z, k_ace)
    # the ACE forces of the 32-atom dipeptide are ~1e-3 kcal/mol/A, where
    # the int64 fixed-point sums (2^-32 per unit) leave ~1e-9 absolute:
    # an RMS floor of 1e-9 kcal/mol/A below the relative tolerance
    rms_ref = float(np.sqrt((ref ** 2).mean()))
    tol = max(tol, 1e-9 / rms_ref)
    assert F.rms_rel(f, ref) <= tol, F.rms_rel(f, ref)
    assert _energy_ok(e[0], F.energies(z, k_ace)[0], floor=1e-6)
    gb = ff.make("GBForce -algorithm NonbondedSimpleFull -soluteDielec 1.0 -solventDielec 78.3")
    en, _ = gs.evaluate()
    both = F.forces(z, 2) + ref
    assert F.rms_rel(gs.forces_total(), both) <= tol
    assert _energy_ok(en[0], F.energies(z, 2)[0] + F.energies(z, k_ace)[0])
    fo = gs.evaluate_forces()  # the force-only form of the MD steps
    assert F.rms_rel(fo, both) <= tol
    gs.close()


def test_gbace_polymer_vs_oracle(ctx):
    """GBACE on a 700-atom heteropolymer (mixed precision) against the FP64
    oracle, alone and beside GBForce."""
    import oracle
    from protomol_b200 import systems
    sm = systems.gb_polymer(700, seed=9)
    s = oracle.System(pos=sm.pos, charge=sm.charge, type=sm.type, molecule=sm.molecule,
                      lj=sm.lj, excl=sm.exclusions, periodic=False, box=sm.box, mass=sm.mass,
                      water=sm.water, gb_vdwr=sm.gb_vdwr, gb_scale=sm.gb_scale,
                      gb_offset=sm.gb_offset, gb_obc=sm.gb_obc)
    fa, ea = oracle.gbace_force(s)
    fg, eg, _ = oracle.gb_force(s, 1.0, 78.5)
    gs = GpuSystem(ctx, sm, "mixed")
    ff = ForceFactory(gs)
    ace = ff.make("GBACEForce -algorithm NonbondedSimpleFull")
    f, e = _eval(ace, sm)
    assert F.rms_rel(f, fa) <= RMS_MIXED, F.rms_rel(f, fa)
    assert _energy_ok(e[0], ea, floor=1e-6)
    ff.make("GBForce -algorithm NonbondedSimpleFull -soluteDielec 1.0 -solventDielec 78.5")
    assert F.rms_rel(gs.evaluate_forces(), fa + fg) <= RMS_MIXED
    en, _ = gs.evaluate()
    assert _energy_ok(en[0], ea + eg)
    gs.close()
