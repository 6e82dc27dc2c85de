"""The drop-in, end to end: ProtoMol's own driver with the GPU force module
(protomol_b200/protomol_module, built into oracle/_ref/protomol_gpu by
oracle/ref.mk) runs the same .conf as the stock binary with the nonbonded
force lines switched to the GPU algorithms; trajectories and energies agree."""
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


def _run(binary, sysm, forces, steps, workdir):
    conf = systems.write_protomol_inputs(sysm, workdir, "w", forces, integrator="Leapfrog",
                                         timestep=0.5, numsteps=steps, cellsize=8.0,
                                         outputs=True)
    out = subprocess.run([binary, conf], cwd=workdir, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    pos = _read_xyz(os.path.join(workdir, "w.out.pos"))
    energy = _read_energies(os.path.join(workdir, "w.out.energy"))
    return pos, energy


@pytest.mark.skipif(not (os.path.exists(CPU) and os.path.exists(GPU)),
                    reason="reference binaries not built (make -f oracle/ref.mk)")
def test_protomol_driver_with_gpu_forces_matches_cpu():
    sysm = systems.tip3p_box(216, 18.6, seed=1, lattice=6)
    cpu_forces = ["LennardJones Coulomb -algorithm NonbondedCutoff -switchingFunction C2 "
                  "-switchon 7 -cutoff 8 -switchingFunction C2 -switchon 7 -cutoff 8 -cutoff 8",
                  "Bond", "Angle"]
    gpu_forces = ["LennardJones Coulomb -algorithm NonbondedCutoffGPU -cutoff 8 "
                  "-ljswitch C2 -ljswitchon 7 -coulombswitch C2 -coulombswitchon 7",
                  "Bond", "Angle"]
    with tempfile.TemporaryDirectory() as a, tempfile.TemporaryDirectory() as b:
        pc, ec = _run(CPU, sysm, cpu_forces, 20, a)
        pg, eg = _run(GPU, sysm, gpu_forces, 20, b)
    # FP32 pair arithmetic (RMS relative force error ~1e-6) over 20 steps of
    # 0.5 fs: positions agree far below the 1e-3 A of thermal motion per step
    assert np.abs(pc - pg).max() < 1e-6, np.abs(pc - pg).max()
    # E_potential (column 1) and E_total (column 3) of the last output line
    for c in (1, 3):
        assert abs(ec[-1, c] - eg[-1, c]) <= 1e-5 * abs(ec[-1, c]), (c, ec[-1], eg[-1])


@pytest.mark.skipif(not (os.path.exists(CPU) and os.path.exists(GPU)),
                    reason="reference binaries not built (make -f oracle/ref.mk)")
def test_protomol_driver_with_gpu_pme_matches_full_ewald():
    sysm = systems.tip3p_box(216, 18.6, seed=1, lattice=6)
    # FullEwald at accuracy 1e-8 (real-space cutoff sqrt(-ln acc)/alpha =
    # 12.3 A, several images in this 18.6 A box) against PME at the same
    # alpha and cutoff, order 8 on 48^3: both converged to ~1e-7
    alpha, acc = 0.35, 1e-8
    rc = float(np.sqrt(-np.log(acc)) / alpha)
    cpu_forces = [f"Coulomb -algorithm FullEwald -real -reciprocal -correction -alpha {alpha} "
                  f"-accuracy {acc:.17g}", "Bond", "Angle"]
    gpu_forces = [f"Coulomb -algorithm PMEwaldGPU -alpha {alpha} -cutoff {rc:.17g} -order 8 "
                  f"-gridsize 48", "Bond", "Angle"]
    with tempfile.TemporaryDirectory() as a, tempfile.TemporaryDirectory() as b:
        pc, ec = _run(CPU, sysm, cpu_forces, 10, a)
        pg, eg = _run(GPU, sysm, gpu_forces, 10, b)
    assert np.abs(pc - pg).max() < 1e-6, np.abs(pc - pg).max()
    for c in (1, 3):
        assert abs(ec[-1, c] - eg[-1, c]) <= 1e-4 * abs(ec[-1, c]), (c, ec[-1], eg[-1])
