"""GPU parity of the remaining switching functions and of the lattice sum
against the reference's own outputs (tests/golden, made by
tests/golden/make_golden.py through ProtoMol's factory):

  * CmpCnCn (switch/CmpCnCnSwitchingFunction.h) on the cutoff path, one
    and two terms;
  * NonbondedFull (force/nonbonded/NonbondedFullSystemForce.h with
    OneAtomPairFull) with C1, C2, Cn and CmpCnCn in a 14.4 A box, below
    twice the 8 A cutoff, so images beyond the minimal one contribute;
  * NonbondedSimpleFull with C2, Cn and the Complement of C1, C2 and Cn
    (switch/ComplementSwitchingFunction.h), periodic (minimal image) and in
    vacuum on the reference's www-fip35 protein.

Tolerances as the other parity tests: mixed precision RMS relative force
error <= 1e-5 and energy relative error <= 1e-6 (absolute floor 1e-4
kcal/mol); double precision 1e-8.
"""
import numpy as np
import pytest

import fixtures as F
import oracle
from protomol_b200 import ForceFactory, GpuSystem, LeapfrogIntegrator, ScalarStructure
from protomol_b200._lib import PmgpuError

pytestmark = pytest.mark.gpu

E_REL = 1e-6


def _energy_ok(got, want, rel=E_REL, floor=1e-4):
    return abs(got - want) <= max(rel * abs(want), floor)


# forces are summed in 64-bit fixed point, 2^-32 kcal/mol/A per unit: for
# terms whose forces are small (the far-pair Complement terms, ~1e-2) a few
# units of that resolution exceed 1e-8 relative
FIXED_QUANTUM = 2.0 ** -32


def _forces_ok(f, ref, tol):
    return F.rms_rel(f, ref) <= tol or np.abs(f - ref).max() <= 4 * FIXED_QUANTUM


@pytest.mark.parametrize("name", ["small_tip3p300_switches", "fip35_switches"])
@pytest.mark.parametrize("precision,tol", [("mixed", 1e-5), ("double", 1e-8)])
def test_switch_variants_and_lattice_sum_vs_reference(ctx, name, precision, tol):
    z = F.load(name)
    topo = F.topology(z)
    gs = GpuSystem(ctx, topo, precision)
    ff = ForceFactory(gs, 6.5)
    seen = 0
    for k, d in enumerate(z["defs"]):
        d = str(d)
        if "-algorithm" not in d:
            continue
        force = ff.make(d)
        ref_f, ref_e = F.forces(z, k), F.energies(z, k)
        f = np.zeros_like(topo.pos)
        e = ScalarStructure()
        force.evaluate(topo.pos, f, e, virial=True)
        assert _forces_ok(f, ref_f, tol), (d, F.rms_rel(f, ref_f), np.abs(f - ref_f).max())
        assert _energy_ok(e[0], ref_e[0], rel=min(E_REL, tol)), (d, e[0], ref_e[0])
        assert _energy_ok(e[1], ref_e[1], rel=min(E_REL, tol)), (d, e[1], ref_e[1])
        vir = np.asarray(e[7:16])
        vtol = (1e-5 if precision == "mixed" else 1e-8) * max(1.0, np.abs(ref_e[7:16]).max())
        assert np.abs(vir - ref_e[7:16]).max() <= vtol, (d, vir, ref_e[7:16])
        # the force-only evaluation (the kernels of an inner MD step)
        f2 = np.zeros_like(topo.pos)
        force.evaluate(topo.pos, f2, None)
        assert _forces_ok(f2, ref_f, tol), (d, "force-only", F.rms_rel(f2, ref_f))
        force.set_enabled(False)
        seen += 1
    assert seen == (4 if name == "fip35_switches" else 10)
    gs.close()


@pytest.mark.parametrize("precision,tol", [("mixed", 1e-5), ("double", 1e-8)])
def test_lattice_sum_md_forces_vs_oracle(ctx, precision, tol):
    """20 leapfrog steps of the 14.4 A box with NonbondedFull LJ C2 and
    Coulomb C1 (8 A) plus bonds and angles: the forces of a force-only
    evaluation at the final positions against the oracle's lattice sum."""
    z = F.load("small_tip3p300_switches")
    topo = F.topology(z)
    gs = GpuSystem(ctx, topo, precision)
    ff = ForceFactory(gs, 6.5)
    lj = ff.make("LennardJones -algorithm NonbondedFull -switchingFunction C2 -switchon 6 "
                 "-cutoff 8 -cutoff 8")
    co = ff.make("Coulomb -algorithm NonbondedFull -switchingFunction C1 -cutoff 8 -cutoff 8")
    ff.make("Bond")
    ff.make("Angle")
    gs.set_positions(topo.pos)
    gs.set_velocities(np.zeros_like(topo.pos))
    LeapfrogIntegrator(0.5).run(gs, 20)
    pos = gs.positions()
    assert np.abs(pos - topo.pos).max() > 1e-4  # the atoms moved
    s = F.oracle_system(z).with_positions(pos)
    fo = np.zeros_like(pos)
    eo = {"lj": 0.0, "coulomb": 0.0}
    for force, pot, sw in ((lj, "LennardJones", oracle.Switch("C2", 8.0, 6.0)),
                           (co, "Coulomb", oracle.Switch("C1", 8.0))):
        fk, ek, _ = oracle.full_force(s, pot, sw, 8.0)
        fo += fk
        eo["lj"] += ek["lj"]
        eo["coulomb"] += ek["coulomb"]
    f = np.zeros_like(pos)
    e = ScalarStructure()
    lj.evaluate(pos, f, e)
    co.evaluate(pos, f, e)
    assert F.rms_rel(f, fo) <= tol, F.rms_rel(f, fo)
    assert _energy_ok(e[0], eo["coulomb"], rel=min(E_REL, tol))
    assert _energy_ok(e[1], eo["lj"], rel=min(E_REL, tol))
    gs.close()


def test_switch_variant_argument_errors(ctx):
    """The factory's rules, as ProtoMol's: a Complement switch only on the
    all-pairs path, the lattice sum only in a periodic box, CmpCnCn with
    switchon < switchoff <= cutoff."""
    z = F.load("small_tip3p300_switches")
    gs = GpuSystem(ctx, F.topology(z), "mixed")
    ff = ForceFactory(gs, 6.5)
    with pytest.raises(PmgpuError):
        ff.make("Coulomb -algorithm NonbondedCutoff -switchingFunction ComplementC1 -cutoff 6")
    with pytest.raises(PmgpuError):
        ff.make("Coulomb -algorithm NonbondedCutoff -switchingFunction ComplimentCnCn "
                "-switchon 4 -switchoff 3 -cutoff 6 -n 2 -cutoff 6")
    gs.close()
    v = F.load("fip35_switches")
    gv = GpuSystem(ctx, F.topology(v), "mixed")
    with pytest.raises(PmgpuError):
        ForceFactory(gv, 8.0).make("Coulomb -algorithm NonbondedFull -switchingFunction C1 "
                                   "-cutoff 8 -cutoff 8")
    gv.close()
