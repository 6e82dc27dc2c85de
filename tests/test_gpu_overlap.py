"""A segment started ahead and undone (pmgpu_run_discard), and the device
integrators' overlap of ProtoMol's output writing with the next segment:
a discard restores the state the segment started from, and ProtoMol runs
with and without the overlap write the same outputs (bit for bit when every
guess of the next segment is right, as a restart from the same state when
some are discarded)."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import fixtures as F
from protomol_b200 import ForceFactory, GpuSystem, LangevinLeapfrogIntegrator, systems

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GPU = os.path.join(ROOT, "oracle", "_ref", "protomol_gpu")
needs_bin = pytest.mark.skipif(not os.path.exists(GPU), reason="module binary not built")

C2C2 = ("-switchingFunction C2 -switchon 7 -cutoff 8 -switchingFunction C2 -switchon 7 "
        "-cutoff 8 -cutoff 8")


def _c1(ctx):
    z = F.load("c1_leapfrog100")
    gs = GpuSystem(ctx, F.topology(z), "mixed")
    ff = ForceFactory(gs, 8.0)
    for line in z["md_forces"]:
        ff.make(str(line))
    return gs


def test_discard_restores_the_segment_start(ctx):
    """LangevinLeapfrog at 300 K, whose noise is keyed by the step counter:
    10 steps, a 20-step segment started and discarded, 10 more steps.  Right
    after the discard positions, velocities and forces are those before the
    segment, bit for bit; the continuation follows the run that never
    started it (a wrong step counter would change every kick's noise by
    about 1e-2 A/ps; a fresh pair list may only move the last bits)."""
    out = []
    for speculate in (False, True):
        gs = _c1(ctx)
        it = LangevinLeapfrogIntegrator(1.0, 300.0, 5.0, seed=7)
        it.run(gs, 10)
        if speculate:
            x0, v0, f0 = gs.positions(), gs.velocities(), gs.forces_total()
            it.run_async(gs, 20)
            it.discard(gs)
            assert np.array_equal(gs.positions(), x0)
            assert np.array_equal(gs.velocities(), v0)
            assert np.array_equal(gs.forces_total(), f0)
        it.run(gs, 10)
        out.append((gs.positions(), gs.velocities()))
        gs.close()
    assert np.abs(out[0][0] - out[1][0]).max() < 1e-9
    assert np.abs(out[0][1] - out[1][1]).max() < 1e-7


def test_discard_without_pending_segment_is_a_no_op(ctx):
    gs = _c1(ctx)
    x0 = gs.positions()
    LangevinLeapfrogIntegrator.discard(gs)
    assert np.array_equal(gs.positions(), x0)
    gs.close()


def _module_run(workdir, overlap, extra=""):
    sysm = systems.tip3p_box(216, 18.6, seed=1, lattice=6)
    conf = systems.write_protomol_inputs(
        sysm, workdir, "w", [f"LennardJones Coulomb -algorithm NonbondedCutoffGPU {C2C2}",
                             "Bond", "Angle"],
        integrator="LangevinLeapfrogGPU", timestep=0.5, numsteps=100, cellsize=8.0,
        outputs=True, integrator_params="temperature 300 gamma 5 seed 1234", extra=extra,
        outputfreq=10)
    env = dict(os.environ, PMGPU_OVERLAP="1" if overlap else "0")
    out = subprocess.run([GPU, conf], cwd=workdir, capture_output=True, text=True,
                         timeout=600, env=env)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    # every keyword is ProtoMol's (an unknown one is only reported)
    assert "not recognized" not in out.stdout + out.stderr
    res = {}
    for name in ("w.out.energy", "w.out.pos", "w.out.vel", "w.out.forces"):
        with open(os.path.join(workdir, name)) as fh:
            res[name] = fh.read()
    return res


@needs_bin
def test_overlapped_outputs_equal_plain_outputs():
    """LangevinLeapfrogGPU, 100 steps with an output every 10: every next
    segment is guessed right, so the files are identical with and without
    the overlap."""
    with tempfile.TemporaryDirectory() as a, tempfile.TemporaryDirectory() as b:
        plain = _module_run(a, False)
        over = _module_run(b, True)
    for name in plain:
        assert plain[name] == over[name], name


def _numbers(text):
    vals = []
    for tok in text.split():
        try:
            vals.append(float.fromhex(tok) if "0x" in tok else float(tok))
        except ValueError:
            pass
    return np.array(vals)


@needs_bin
def test_overlap_with_discarded_guesses():
    """Forces written every 15 steps beside the outputs every 10: ProtoMol
    asks for 10, 5, 5, 10, ... steps, so some started segments are
    discarded and rerun from the restored state; the outputs agree with the
    plain run to the last bits."""
    extra = "XYZForceFileOutputFreq 15"
    with tempfile.TemporaryDirectory() as a, tempfile.TemporaryDirectory() as b:
        plain = _module_run(a, False, extra)
        over = _module_run(b, True, extra)
    for name in plain:
        p, o = _numbers(plain[name]), _numbers(over[name])
        assert p.shape == o.shape, name
        assert np.abs(p - o).max() <= 1e-8 * max(1.0, np.abs(p).max()), name
