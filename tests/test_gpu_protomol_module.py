"""The drop-in, end to end: ProtoMol's own driver with the GPU module
(protomol_b200/protomol_module, built into oracle/_ref/protomol_gpu by its
Makefile) runs the same .conf as the stock binary with the force lines
switched to the GPU algorithms (the reference's force grammar, the
algorithm name carrying a GPU suffix) and, where asked, the device-resident
integrators (LeapfrogGPU, LangevinLeapfrogGPU).  Trajectories and the
energies written at every output step agree with the stock run."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from protomol_b200 import systems

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CPU = os.path.join(ROOT, "oracle", "_ref", "protomol")
GPU = os.path.join(ROOT, "oracle", "_ref", "protomol_gpu")
needs_bins = pytest.mark.skipif(not (os.path.exists(CPU) and os.path.exists(GPU)),
                                reason="reference binaries not built")

C2C2 = ("-switchingFunction C2 -switchon 7 -cutoff 8 -switchingFunction C2 -switchon 7 "
        "-cutoff 8 -cutoff 8")


def _read_xyz(path):
    """ProtoMol's finXYZPosFile: the atom count, then one line per atom
    (name, x, y, z) with no comment line."""
    with open(path) as fh:
        lines = fh.read().split("\n")
    n = int(lines[0])
    return np.array([[float(v) for v in ln.split()[1:4]] for ln in lines[1:1 + n]])


def _read_energies(path):
    """allenergiesfile rows: time, then hexadecimal floats in the columns of
    the .header file (E_potential, E_kinetic, E_total, ...)."""
    rows = []
    with open(path) as fh:
        for line in fh:
            toks = line.split()
            if toks:
                rows.append([float(toks[0])] + [float.fromhex(t) for t in toks[1:]])
    return np.array(rows)


def _run(binary, sysm, forces, steps, workdir, integrator="Leapfrog", timestep=0.5,
         params="", extra="", outputfreq=None, cellsize=8.0):
    conf = systems.write_protomol_inputs(sysm, workdir, "w", forces, integrator=integrator,
                                         timestep=timestep, numsteps=steps, cellsize=cellsize,
                                         outputs=True, integrator_params=params, extra=extra,
                                         outputfreq=outputfreq)
    out = subprocess.run([binary, conf], cwd=workdir, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    pos = _read_xyz(os.path.join(workdir, "w.out.pos"))
    energy = _read_energies(os.path.join(workdir, "w.out.energy"))
    return pos, energy


def _both(sysm, cpu_forces, gpu_forces, steps, **kw):
    gpu_integ = kw.pop("gpu_integrator", None)
    with tempfile.TemporaryDirectory() as a, tempfile.TemporaryDirectory() as b:
        pc, ec = _run(CPU, sysm, cpu_forces, steps, a, **kw)
        if gpu_integ:
            kw["integrator"] = gpu_integ
        pg, eg = _run(GPU, sysm, gpu_forces, steps, b, **kw)
    return pc, ec, pg, eg


@needs_bins
def test_cpu_integrator_with_gpu_cutoff_forces_reference_grammar():
    """The reference's own force line, -algorithm NonbondedCutoffGPU, under
    the stock Leapfrog (positions up, forces down every step)."""
    sysm = systems.tip3p_box(216, 18.6, seed=1, lattice=6)
    pc, ec, pg, eg = _both(
        sysm, [f"LennardJones Coulomb -algorithm NonbondedCutoff {C2C2}", "Bond", "Angle"],
        [f"LennardJones Coulomb -algorithm NonbondedCutoffGPU {C2C2}", "Bond", "Angle"], 20)
    # FP32 pair arithmetic (RMS relative force error ~1e-6) over 20 steps of
    # 0.5 fs: positions agree to ~1e-6 A, far below the 1e-3 A of thermal
    # motion per step
    assert np.abs(pc - pg).max() < 1e-5, np.abs(pc - pg).max()
    for c in (1, 3):  # E_potential, E_total of the last output line
        assert abs(ec[-1, c] - eg[-1, c]) <= 1e-5 * abs(ec[-1, c]), (c, ec[-1], eg[-1])


@needs_bins
def test_leapfrog_gpu_100_steps_outputs_every_10():
    """LeapfrogGPU, 100 steps of 0.5 fs with an output every 10 steps: the
    device integrator runs each 10-step chunk on the device and writes
    positions, velocities and energies back only at the outputs; every
    output row (E_potential, E_kinetic, E_total) and the final positions
    match the stock Leapfrog with CPU forces.  Bond and Angle are the CPU
    force lines, which the device integrator maps to its bonded terms."""
    sysm = systems.tip3p_box(216, 18.6, seed=1, lattice=6)
    pc, ec, pg, eg = _both(
        sysm, [f"LennardJones Coulomb -algorithm NonbondedCutoff {C2C2}", "Bond", "Angle"],
        [f"LennardJones Coulomb -algorithm NonbondedCutoffGPU {C2C2}", "Bond", "Angle"], 100,
        outputfreq=10, gpu_integrator="LeapfrogGPU")
    assert ec.shape == eg.shape and ec.shape[0] == 11, (ec.shape, eg.shape)
    assert np.array_equal(ec[:, 0], eg[:, 0])  # output times
    for c in (1, 2, 3):
        err = np.abs(ec[:, c] - eg[:, c]) / np.abs(ec[:, c]).max()
        assert err.max() <= 1e-5, (c, err)
    # FP32 pair forces (RMS relative error ~1e-6 per step) drift apart from
    # the FP64 run through the water's chaotic dynamics: ~5e-4 A after 100
    # steps, the bound the FP64 oracle comparison of the same run uses
    assert np.abs(pc - pg).max() < 1e-3, np.abs(pc - pg).max()


@needs_bins
def test_cn_switching_through_the_module():
    """Cn switching (the reference's Cn/Cn line) on the GPU cutoff force."""
    sysm = systems.tip3p_box(216, 18.6, seed=1, lattice=6)
    cn = ("-switchingFunction Cn -n 4 -switchon 5 -cutoff 8 -switchingFunction Cn -n 3 "
          "-switchon 4 -cutoff 8 -cutoff 8")
    pc, ec, pg, eg = _both(
        sysm, [f"LennardJones Coulomb -algorithm NonbondedCutoff {cn}", "Bond", "Angle"],
        [f"LennardJones Coulomb -algorithm NonbondedCutoffGPU {cn}", "Bond", "Angle"], 10)
    assert np.abs(pc - pg).max() < 1e-5, np.abs(pc - pg).max()  # FP32 forces, as above
    for c in (1, 3):
        assert abs(ec[-1, c] - eg[-1, c]) <= 1e-5 * abs(ec[-1, c]), (c, ec[-1], eg[-1])


@needs_bins
def test_cpu_integrator_with_gpu_pme_matches_full_ewald():
    sysm = systems.tip3p_box(216, 18.6, seed=1, lattice=6)
    # FullEwald at accuracy 1e-8 (real-space cutoff sqrt(-ln acc)/alpha =
    # 12.3 A, several images in this 18.6 A box) against PME at the same
    # alpha and cutoff, order 8 on 48^3: both converged to ~1e-7
    alpha, acc = 0.35, 1e-8
    rc = float(np.sqrt(-np.log(acc)) / alpha)
    pc, ec, pg, eg = _both(
        sysm, [f"Coulomb -algorithm FullEwald -real -reciprocal -correction -alpha {alpha} "
               f"-accuracy {acc:.17g}", "Bond", "Angle"],
        [f"Coulomb -algorithm PMEwaldGPU -alpha {alpha} -cutoff {rc:.17g} -order 8 "
         f"-gridsize 48", "Bond", "Angle"], 10)
    assert np.abs(pc - pg).max() < 1e-5, np.abs(pc - pg).max()  # FP32 forces, as above
    for c in (1, 3):
        assert abs(ec[-1, c] - eg[-1, c]) <= 1e-4 * abs(ec[-1, c]), (c, ec[-1], eg[-1])


@needs_bins
def test_lattice_sum_cmpcncn_and_complement_through_the_module():
    """The remaining algorithm and switches through ProtoMol's factory: the
    NonbondedFull lattice sum (C1 Coulomb, C2 LJ) in a 14.4 A box below
    twice its 8 A cutoff, CmpCnCn on NonbondedCutoff and the Complement
    switches on the periodic all-pairs form, under the stock Leapfrog
    against the stock binary with the CPU forces."""
    sysm = systems.tip3p_box(100, 14.4, seed=5, lattice=5)
    lines = [
        "Coulomb -algorithm {full} -switchingFunction C1 -cutoff 8 -cutoff 8",
        "LennardJones -algorithm {full} -switchingFunction C2 -switchon 6 -cutoff 8 -cutoff 8",
        "LennardJones Coulomb -algorithm {cut} -switchingFunction ComplimentCnCn -switchon 2 "
        "-switchoff 5 -cutoff 6.5 -n 3 -switchingFunction ComplimentCnCn -switchon 1 "
        "-switchoff 4 -cutoff 6.5 -n 2 -cutoff 6.5",
        "LennardJones Coulomb -algorithm {sf} -switchingFunction ComplementC2 -switchon 5 "
        "-cutoff 6 -switchingFunction ComplementC1 -cutoff 6",
        "Bond", "Angle"]
    cpu = [ln.format(full="NonbondedFull", cut="NonbondedCutoff", sf="NonbondedSimpleFull")
           for ln in lines]
    gpu = [ln.format(full="NonbondedFullGPU", cut="NonbondedCutoffGPU",
                     sf="NonbondedSimpleFullGPU") for ln in lines]
    pc, ec, pg, eg = _both(sysm, cpu, gpu, 10, cellsize=6.5)
    assert np.abs(pc - pg).max() < 1e-5, np.abs(pc - pg).max()  # FP32 forces, as above
    for c in (1, 3):
        assert abs(ec[-1, c] - eg[-1, c]) <= 1e-5 * abs(ec[-1, c]), (c, ec[-1], eg[-1])


def _gb_polymer(n, seed):
    """A GB heteropolymer as ProtoMol's PSF/PAR path builds it: the reader
    takes each type's GB radius from its PAR Rmin/2 (topology/
    BuildTopology.cpp:608, :881), so the polymer's radii are set to that."""
    sm = systems.gb_polymer(n, seed)
    sm.gb_vdwr = sm.rmin2[sm.type].copy()
    return sm


@needs_bins
@pytest.mark.parametrize("obc", [2, 1])
def test_langevin_gpu_gb_polymer_matches_stock(obc):
    """GBBornRadii / GBPartialSum / GBForce / GBACEForce, LJ and Coulomb as
    NonbondedSimpleFullGPU with CPU Bond, Angle and Dihedral, under
    LangevinLeapfrogGPU at temperature 0 (no noise, so the run is
    deterministic) against the stock LangevinLeapfrog with the CPU forces;
    doGBSAObc 1 and 2 set different OBC constants in the topology, which
    the module reads from there."""
    sm = _gb_polymer(300, 5)
    gb = ["GBBornRadii -algorithm {a}", "GBPartialSum -algorithm {a}",
          "GBForce -algorithm {a} -soluteDielec 1 -solventDielec 78.5",
          "GBACEForce -algorithm {a}",
          "LennardJones -algorithm {a}", "Coulomb -algorithm {a}"]
    bonded = ["Bond", "Angle", "Dihedral"]
    pc, ec, pg, eg = _both(
        sm, [g.format(a="NonbondedSimpleFull") for g in gb] + bonded,
        [g.format(a="NonbondedSimpleFullGPU") for g in gb] + bonded, 20,
        integrator="LangevinLeapfrog", gpu_integrator="LangevinLeapfrogGPU", timestep=1.0,
        params="temperature 0 gamma 5 seed 1234", extra=f"doGBSAObc {obc}", outputfreq=10,
        cellsize=5.0)
    assert ec.shape == eg.shape == (3, ec.shape[1]), (ec.shape, eg.shape)
    for c in (1, 3):
        err = np.abs(ec[:, c] - eg[:, c]) / np.abs(ec[:, c]).max()
        assert err.max() <= 1e-5, (c, err)
    assert np.abs(pc - pg).max() < 1e-5, np.abs(pc - pg).max()
