"""Pins the FP64 oracle restatement (oracle/pmoracle.c) against the golden
fixtures, which are outputs of the unmodified ProtoMol reference
(tests/golden/make_golden.py).  Every term below matches the reference
to rounding (most bit for bit)."""
import numpy as np
import pytest

import fixtures as F
import oracle

CUT_TOL = 1e-11  # absolute, kcal/mol/A: FP64 restatement vs FP64 reference


def _cutoff_terms(d):
    pots, sws, alg = F.parse_cutoff_def(d)
    terms = [(p, oracle.Switch(sws[j]["kind"], sws[j].get("cutoff", 0.0),
                               sws[j].get("switchon", 0.0), 0.0, sws[j].get("n", 0.0)))
             for j, p in enumerate(pots)]
    return terms, alg


@pytest.mark.parametrize("name,cellsize", [("water423", 6.5), ("c1_tip3p648", 8.0)])
def test_cutoff_forces_match_reference(name, cellsize):
    z = F.load(name)
    s = F.oracle_system(z)
    seen = 0
    for k, d in enumerate(z["defs"]):
        if "NonbondedCutoff" not in d:
            continue
        terms, alg = _cutoff_terms(str(d))
        f, e, v = oracle.cutoff_force(s, cellsize, alg, terms)
        ref_e = F.energies(z, k)
        assert np.abs(f - F.forces(z, k)).max() < CUT_TOL, d
        assert e["coulomb"] == pytest.approx(ref_e[0], abs=1e-9)
        assert e["lj"] == pytest.approx(ref_e[1], abs=1e-9)
        assert np.abs(v.reshape(-1) - ref_e[7:16]).max() < 1e-9
        seen += 1
    assert seen >= 3


@pytest.mark.parametrize("name,cellsize", [("water423", 6.5), ("c1_tip3p648", 8.0)])
def test_full_ewald_terms_match_reference(name, cellsize):
    z = F.load(name)
    s = F.oracle_system(z)
    ew = oracle.ewald_params(s, 0.35, 1e-4)
    for k, d in enumerate(z["defs"]):
        d = str(d)
        if "FullEwald" not in d:
            continue
        if "-real" in d:
            f, e, v = oracle.ewald_real(s, ew, cellsize)
        elif "-reciprocal" in d:
            f, e, v = oracle.ewald_reciprocal(s, ew)
        else:
            f, e, v = oracle.ewald_correction(s, ew)
            a, b = oracle.ewald_self(s, ew)
            e += a + b
        assert np.abs(f - F.forces(z, k)).max() < 1e-11, d
        assert e == pytest.approx(F.energies(z, k)[0], rel=1e-13, abs=1e-10), d


@pytest.mark.parametrize("name", ["fip35_gb", "alanylalanine_gb"])
def test_gb_and_simplefull_match_reference(name):
    z = F.load(name)
    s = F.oracle_system(z)
    f, e, born = oracle.gb_force(s, 1.0, 78.3)
    assert np.abs(f - F.forces(z, 2)).max() < 1e-10
    assert e == pytest.approx(F.energies(z, 2)[0], rel=1e-12)
    for k, pot, slot in ((3, "LennardJones", "lj"), (4, "Coulomb", "coulomb")):
        f, e, v = oracle.simplefull_force(s, pot)
        assert np.abs(f - F.forces(z, k)).max() < 1e-10
        assert e[slot] == pytest.approx(F.energies(z, k)[1 if slot == "lj" else 0], rel=1e-12)


def test_spme_restatement_converges_to_reference_ksum():
    """ProtoMol has no PME.  The FP64 SPME restatement converges to the
    reference's Ewald k-sum (restated bit-exactly above; accuracy 1e-14 so
    the k-sphere truncation is negligible) as order and grid grow."""
    from oracle import spme
    z = F.load("c1_tip3p648")
    s = F.oracle_system(z)
    t = F.topology(z)
    fk, ek, _ = oracle.ewald_reciprocal(s, oracle.ewald_params(s, 0.35, 1e-14))
    errs = []
    for p, K in ((4, 32), (6, 48), (8, 96)):
        f, e = spme.reciprocal(t.pos, t.charge, t.box, 0.35, p, K)
        errs.append(F.rms_rel(f, fk))
        if p == 8:
            assert abs(e - ek) <= 1e-10 * abs(ek)
    assert errs[0] > errs[1] > errs[2]
    assert errs[2] < 1e-10


def test_pair_set_equals_brute_force_minimal_image():
    """The cell enumeration covers exactly the pairs within the cutoff."""
    z = F.load("c1_tip3p648")
    s = F.oracle_system(z)
    pairs = oracle.cutoff_pairs(s, 8.0, 8.0, 8.0)
    L = s.box[0]
    got = set(map(tuple, np.sort(pairs[:, :2], axis=1)))
    want = set()
    for i in range(s.n):
        d = s.pos[i + 1:] - s.pos[i]
        d -= L * np.rint(d / L)
        r2 = (d * d).sum(1)
        js = np.nonzero(r2 <= 64.0)[0] + i + 1
        for j in js:
            if s.molecule[i] == s.molecule[j]:
                continue  # TIP3P: every intramolecular pair is excluded
            want.add((i, int(j)))
    assert got == want


def test_cell_assignment_formula():
    """ProtoMol cells: cell size L / floor(L / cellsize), index
    floor((L/2 + minimalPosition(x)) / size)."""
    z = F.load("water423")
    s = F.oracle_system(z)
    cells, dims = oracle.cell_assign(s, 6.5)
    assert tuple(dims) == (4, 4, 4)
    w = s.pos - s.box[9:12]
    w -= 28.0 * np.rint(w / 28.0)
    ref = np.floor((w + 14.0) / 7.0).astype(int)
    ok = np.all(cells == ref, axis=1)
    assert ok.mean() > 0.999


@pytest.mark.parametrize("name", ["fip35_torsions", "alanylalanine_torsions", "polymer200_torsions"])
def test_torsion_oracle_matches_reference(name):
    """MTorsionSystemForce::calcTorsion (Dihedral force) restated in the
    oracle against the reference's own forces and DIHEDRAL energy."""
    z = F.load(name)
    s = F.oracle_system(z)
    atoms = z["dihedrals"].reshape(-1, 4)
    prm = z["dihedral_params"].reshape(-1, 3)
    f, e, _ = oracle.torsion_force(s, atoms, prm)
    ref_f = F.forces(z, 0)
    assert np.abs(f - ref_f).max() <= 1e-10 * max(1.0, np.abs(ref_f).max())
    assert abs(e - F.energies(z, 0)[4]) <= 1e-10 * max(1.0, abs(e))


@pytest.mark.parametrize("name", ["water423", "c1_tip3p648"])
def test_bond_and_angle_oracle_match_reference(name):
    """BondSystemForce / AngleSystemForce (with Urey-Bradley) restated in
    the oracle against the reference's own forces, energies and virial."""
    z = F.load(name)
    s = F.oracle_system(z)
    t = F.topology(z)
    for kw, args, slot in (("Bond", (t.bonds, t.bond_params, None, None), 2),
                           ("Angle", (None, None, t.angles, t.angle_params), 3)):
        k = [i for i, d in enumerate(z["defs"]) if str(d) == kw][0]
        f, e, v = oracle.bonded_force(s, *args)
        ref_e = F.energies(z, k)
        assert np.abs(f - F.forces(z, k)).max() <= 1e-12, kw
        assert e[kw.lower()] == pytest.approx(ref_e[slot], rel=1e-13, abs=1e-12), kw
        assert np.abs(v.reshape(-1) - ref_e[7:16]).max() <= 1e-10, kw


def test_leapfrog100_oracle_trajectory_matches_reference():
    """The small plain configuration (648-atom TIP3P box, LJ + Coulomb C2
    7 -> 8 A, bonds, angles, leapfrog 0.5 fs) integrated on the host with the
    oracle's forces (LeapfrogIntegrator.cpp:33-104: half kick, drift, forces,
    half kick) reproduces the reference's own 100-step run: the energies of
    every step and the state at steps 25, 50, 75 and 100."""
    z = F.load("c1_leapfrog100")
    t = F.topology(z)
    s = F.oracle_system(z)
    sw = oracle.Switch("C2", 8.0, 7.0)

    def forces(x):
        s2 = s.with_positions(x)
        f, e, _ = oracle.cutoff_force(s2, 8.0, 8.0, [("LennardJones", sw), ("Coulomb", sw)])
        fb, eb, _ = oracle.bonded_force(s2, t.bonds, t.bond_params, t.angles, t.angle_params)
        return f + fb, np.array([e["coulomb"], e["lj"], eb["bond"], eb["angle"]])

    h = float(z["timestep"]) * oracle.INV_TIMEFACTOR
    x, v = t.pos.copy(), t.vel.copy()
    f, e = forces(x)
    ref = z["energies_per_step"]
    assert np.abs(e - ref[0]).max() <= 1e-9
    for k in range(1, 101):
        v = oracle.kick(t.mass, f, 0.5 * h, v)
        x = oracle.drift(v, h, x)
        f, e = forces(x)
        v = oracle.kick(t.mass, f, 0.5 * h, v)
        assert np.abs(e - ref[k]).max() <= 1e-8 * max(1.0, np.abs(ref[k]).max()), k
        if k % 25 == 0:
            assert np.abs(x - z[f"positions_{k}"].reshape(-1, 3)).max() <= 1e-10, k
            assert np.abs(v - z[f"velocities_{k}"].reshape(-1, 3)).max() <= 1e-9, k


@pytest.mark.parametrize("name", ["fip35_gb", "alanylalanine_gb"])
def test_gbace_oracle_matches_reference(name):
    """GBACEForce (the ACE nonpolar term on the GB Born radii, default
    -solvationparam and -watersphereradius) restated in the oracle against
    the reference's own forces and energy on its GB test systems."""
    z = F.load(name)
    s = F.oracle_system(z)
    k = [i for i, d in enumerate(z["defs"]) if str(d).startswith("GBACEForce")][0]
    f, e = oracle.gbace_force(s)
    ref_f = F.forces(z, k)
    assert np.abs(f - ref_f).max() <= 1e-12 * max(1.0, np.abs(ref_f).max())
    assert e == pytest.approx(F.energies(z, k)[0], rel=1e-13)


def _switch_terms(d):
    pots, sws, alg = F.parse_cutoff_def(d)
    terms = [(p, oracle.Switch(sws[j]["kind"], sws[j].get("cutoff", 0.0),
                               sws[j].get("switchon", 0.0), sws[j].get("switchoff", 0.0),
                               sws[j].get("n", 0.0)))
             for j, p in enumerate(pots)]
    return terms, alg


@pytest.mark.parametrize("name", ["small_tip3p300_switches", "fip35_switches"])
def test_switch_variants_and_lattice_sum_match_reference(name):
    """CmpCnCn (cutoff path), the Complement switches and C1/C2/Cn on the
    all-pairs path (vacuum and periodic minimal image), and the NonbondedFull
    lattice sum in a box below twice the cutoff, against the reference's
    own forces, energies and virial."""
    z = F.load(name)
    s = F.oracle_system(z)
    kinds = set()
    for k, d in enumerate(z["defs"]):
        d = str(d)
        if "-algorithm" not in d:
            continue
        terms, alg = _switch_terms(d)
        if "NonbondedCutoff" in d:
            f, e, v = oracle.cutoff_force(s, 6.5, alg, terms)
        elif "NonbondedFull " in d:
            assert len(terms) == 1
            f, e, v = oracle.full_force(s, terms[0][0], terms[0][1], alg)
        else:
            f, e, v = oracle.simplefull_force_n(s, terms)
        ref_f, ref_e = F.forces(z, k), F.energies(z, k)
        scale = max(1.0, np.abs(ref_f).max())
        assert np.abs(f - ref_f).max() < 1e-11 * scale, d
        assert e["coulomb"] == pytest.approx(ref_e[0], rel=1e-12, abs=1e-9), d
        assert e["lj"] == pytest.approx(ref_e[1], rel=1e-12, abs=1e-9), d
        assert np.abs(v.reshape(-1) - ref_e[7:16]).max() < 1e-8 * max(1.0, np.abs(ref_e[7:16]).max()), d
        kinds.add(d.split("-algorithm")[1].split()[0])
    assert kinds >= ({"NonbondedSimpleFull"} if name == "fip35_switches" else
                     {"NonbondedCutoff", "NonbondedFull", "NonbondedSimpleFull"})


def _param(line, key, default):
    toks = line.split()
    return float(toks[toks.index(key) + 1]) if key in toks else default


@pytest.mark.parametrize("name", ["alanine_scpism", "wwdomain_scpism"])
def test_scpism_oracle_matches_reference(name):
    """SCPISM on the reference's implicit-solvent systems: LennardJones +
    CoulombSCPISM (Cn on NonbondedCutoff; C1, C2 on the cutoff and
    all-pairs algorithms; -D), and the BornRadii + BornSelf chain (Born
    switches 3, 1 and 2), against the reference's own forces and energies."""
    z = F.load(name)
    s = F.oracle_system(z)
    seen = 0
    for k, d in enumerate(z["defs"]):
        d = str(d)
        if d.startswith("BornRadii"):
            continue
        if d.startswith("BornSelf"):
            rd = str(z["defs"][k - 1])  # its BornRadii line
            f, e, _ = oracle.born_force(s, int(_param(rd, "-bornswitch", 3)),
                                        _param(rd, "-cutoff", 5.0),
                                        int(_param(d, "-bornswitch", 3)),
                                        _param(d, "-cutoff", 5.0), _param(d, "-D", 80.0))
            e_c, e_lj = e, 0.0
        else:
            terms, _ = _switch_terms(d)
            f, e, _ = oracle.scpism_pair_force(s, terms, _param(d, "-D", 80.0))
            e_c, e_lj = e["coulomb"], e["lj"]
        ref_f, ref_e = F.forces(z, k), F.energies(z, k)
        assert np.abs(f - ref_f).max() < 1e-11 * max(1.0, np.abs(ref_f).max()), d
        assert e_c == pytest.approx(ref_e[0], rel=1e-12, abs=1e-9), d
        assert e_lj == pytest.approx(ref_e[1], rel=1e-12, abs=1e-9), d
        seen += 1
    assert seen == 6
