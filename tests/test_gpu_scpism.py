"""GPU parity of the SCPISM implicit-solvent forces against the reference's
own outputs on its implicit-solvent test systems (alanine dipeptide and the
WW domain, tests/golden made by tests/golden/make_golden.py):
LennardJones + CoulombSCPISM with Cn switching at 20 A on NonbondedCutoff
(the reference's own force line), CoulombSCPISM with C1/C2 switches and
another -D on the cutoff and all-pairs algorithms, and the BornRadii +
BornSelf chain with three Born switches.  Both precisions compute these
terms in FP64: forces within 1e-8 relative (or a few units of the 2^-32
fixed-point force resolution), energies within 1e-8 relative."""
import numpy as np
import pytest

import fixtures as F
import oracle
from protomol_b200 import ForceFactory, GpuSystem, LeapfrogIntegrator, ScalarStructure
from protomol_b200._lib import PmgpuError

pytestmark = pytest.mark.gpu

TOL = 1e-8


def _forces_ok(f, ref):
    return F.rms_rel(f, ref) <= TOL or np.abs(f - ref).max() <= 4 * 2.0 ** -32


def _param(line, key, default):
    toks = line.split()
    return float(toks[toks.index(key) + 1]) if key in toks else default


@pytest.mark.parametrize("name", ["alanine_scpism", "wwdomain_scpism"])
@pytest.mark.parametrize("precision", ["mixed", "double"])
def test_scpism_forces_vs_reference(ctx, name, precision):
    z = F.load(name)
    topo = F.topology(z)
    gs = GpuSystem(ctx, topo, precision)
    ff = ForceFactory(gs, 5.0)
    seen = 0
    for k, d in enumerate(z["defs"]):
        d = str(d)
        force = ff.make(d)
        if d.startswith("BornRadii"):
            continue  # its pass runs inside the BornSelf term that follows
        ref_f, ref_e = F.forces(z, k), F.energies(z, k)
        f = np.zeros_like(topo.pos)
        e = ScalarStructure()
        force.evaluate(topo.pos, f, e, virial=True)
        assert _forces_ok(f, ref_f), (d, F.rms_rel(f, ref_f), np.abs(f - ref_f).max())
        for slot in (0, 1):
            assert abs(e[slot] - ref_e[slot]) <= TOL * max(1.0, abs(ref_e[slot])), (d, slot)
        f2 = np.zeros_like(topo.pos)
        force.evaluate(topo.pos, f2, None)  # force-only
        assert _forces_ok(f2, ref_f), (d, "force-only")
        force.set_enabled(False)
        seen += 1
    assert seen == 6
    gs.close()


def test_scpism_md_forces_vs_oracle(ctx):
    """The reference conf's force set on the WW domain (LJ + CoulombSCPISM
    Cn 20 A, BornRadii + BornSelf, bonds, angles, torsions), 10 leapfrog
    steps of 0.25 fs from rest on the device; at the final positions the
    SCPISM and Born forces of a force-only evaluation against the oracle."""
    z = F.load("wwdomain_scpism")
    topo = F.topology(z)
    gs = GpuSystem(ctx, topo, "mixed")
    ff = ForceFactory(gs, 5.0)
    defs = [str(d) for d in z["defs"]][:3]
    forces = [ff.make(d) for d in defs]
    for line in ("Bond", "Angle", "Dihedral Improper"):
        ff.make(line)
    gs.set_velocities(np.zeros_like(topo.pos))
    LeapfrogIntegrator(0.25).run(gs, 10)
    x = gs.positions()
    assert np.abs(x - topo.pos).max() > 1e-5
    s = F.oracle_system(z).with_positions(x)
    sw = oracle.Switch("Cn", 20.0, 8.0, 0.0, 4.0)
    fo, _, _ = oracle.scpism_pair_force(s, [("LennardJones", sw), ("CoulombSCPISM", sw)], 80.0)
    fb, _, _ = oracle.born_force(s, 3, 5.0, 3, 5.0, 80.0)
    f = np.zeros_like(x)
    forces[0].evaluate(x, f, None)
    assert F.rms_rel(f, fo) <= TOL, F.rms_rel(f, fo)
    f = np.zeros_like(x)
    forces[2].evaluate(x, f, None)
    assert _forces_ok(f, fb), F.rms_rel(f, fb)
    gs.close()


def test_scpism_needs_its_parameters(ctx):
    """Without SCPISM data the SCPISM forces are refused, as the
    reference reports "requires SCPISM parameters"."""
    z = F.load("c1_tip3p648")
    gs = GpuSystem(ctx, F.topology(z), "mixed")
    ff = ForceFactory(gs, 8.0)
    with pytest.raises(PmgpuError):
        ff.make("CoulombSCPISM -algorithm NonbondedCutoff -switchingFunction C2 -switchon 0 "
                "-cutoff 8 -cutoff 8")
    with pytest.raises(PmgpuError):
        ff.make("BornSelf -algorithm NonbondedCutoff -switchingFunction Cutoff -cutoff 5 "
                "-cutoff 5")
    gs.close()
