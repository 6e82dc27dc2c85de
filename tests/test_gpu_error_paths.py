"""Error paths and the Langevin thermostat, on the GPU without any device
fault: a pair list whose capacity is too small for the system (the build
flags the overflow, the host grows the list and repeats the segment), column
buckets too small for the atoms binned into a column (the same growth), a
non-finite position handed in from the host (refused before any upload),
and the statistics of the Langevin noise (Philox4x32-10 + Box-Muller)
through the integrator."""
import numpy as np
import pytest

import fixtures as F
from protomol_b200 import (ForceFactory, GpuSystem, LangevinLeapfrogIntegrator,
                           LeapfrogIntegrator, PmgpuError, systems)
from protomol_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _c1(ctx, precision="mixed"):
    z = F.load("c1_leapfrog100")
    topo = F.topology(z)
    gs = GpuSystem(ctx, topo, precision)
    ff = ForceFactory(gs, 8.0)
    for line in z["md_forces"]:
        ff.make(str(line))
    return gs


def test_list_overflow_retry_is_bit_identical(ctx):
    """A list fixed at one tile per row overflows on its first build; the
    segment is repeated with the grown list and the trajectory equals, bit
    for bit, the run whose list never overflowed (fixed-point force sums and
    the same tile order per row)."""
    out = []
    for cap in (None, 1):
        gs = _c1(ctx)
        if cap:
            gs.set_list_capacity(cap)
        LangevinLeapfrogIntegrator(1.0, 300.0, 5.0, seed=11).run(gs, 30)
        out.append((gs.positions(), gs.velocities(), gs.energies()[0]))
        assert gs.forces[0].stats()["list_entries"] > 0
        gs.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][2], out[1][2])


def test_list_overflow_in_single_evaluation(ctx):
    """The same growth path in a single evaluation: the forces equal those
    of an unconstrained list."""
    gs = _c1(ctx)
    e0, _ = gs.evaluate()
    f0 = gs.forces_total()
    gs.set_list_capacity(1)
    e1, _ = gs.evaluate()
    assert np.array_equal(f0, gs.forces_total())
    assert np.array_equal(e0, e1)
    gs.close()


def test_column_bucket_overflow_retry_is_bit_identical(ctx):
    """Column buckets fixed at 32 atoms overflow on the first build (the
    648-atom box bins about 40 atoms into each of its 16 columns); the
    buckets grow to the fullest column's count, the segment is repeated and
    the trajectory equals, bit for bit, the run whose buckets never
    overflowed."""
    out = []
    for cap in (None, 32):
        gs = _c1(ctx)
        if cap:
            gs.set_column_capacity(cap)
        LangevinLeapfrogIntegrator(1.0, 300.0, 5.0, seed=11).run(gs, 30)
        out.append((gs.positions(), gs.velocities(), gs.energies()[0]))
        assert gs.forces[0].stats()["list_entries"] > 0
        gs.close()
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)


def test_column_bucket_overflow_in_single_evaluation(ctx):
    gs = _c1(ctx)
    e0, _ = gs.evaluate()
    f0 = gs.forces_total()
    gs.set_column_capacity(32)
    e1, _ = gs.evaluate()
    assert np.array_equal(f0, gs.forces_total())
    assert np.array_equal(e0, e1)
    gs.close()


def test_non_finite_positions_are_refused(ctx):
    gs = _c1(ctx)
    x = gs.positions()
    bad = x.copy()
    bad[17, 1] = np.nan
    with pytest.raises(PmgpuError) as ei:
        gs.set_positions(bad)
    assert ei.value.code == L.ERR_NAN
    bad[17, 1] = np.inf
    with pytest.raises(PmgpuError):
        gs.set_positions(bad)
    # the resident state is untouched and usable
    assert np.array_equal(gs.positions(), x)
    LeapfrogIntegrator(0.5).run(gs, 2)
    assert np.all(np.isfinite(gs.positions()))
    gs.close()


def _temperature(vel, mass):
    """Instantaneous temperature 2 KE / (3 N k_B) (no constraints)."""
    return float((mass[:, None] * vel ** 2).sum() / (3 * len(mass) * 0.001987191))


def test_langevin_noise_statistics_without_forces(ctx):
    """With no force terms LangevinLeapfrog is an Ornstein-Uhlenbeck process
    per velocity component; from rest its stationary distribution is
    Gaussian with mean 0 and variance k_B T / m.  Over 1,296 atoms x 3
    components x 40 samples (spaced by the 1 / gamma relaxation time) the
    scaled velocities have mean 0 and variance 1, and skewness and excess
    kurtosis near 0."""
    sm = systems.tip3p_box(432, 23.5, seed=4, lattice=8)
    sm.vel = np.zeros_like(sm.vel)
    gs = GpuSystem(ctx, sm, "mixed")  # no forces added
    T = 300.0
    it = LangevinLeapfrogIntegrator(1.0, temperature=T, gamma=50.0, seed=2024)
    it.run(gs, 200)  # ten relaxation times (1 / gamma = 20 fs)
    u = []
    for _ in range(40):
        it.run(gs, 20)
        v = gs.velocities()
        u.append(v / np.sqrt(0.001987191 * T / sm.mass[:, None]))
    u = np.concatenate([a.ravel() for a in u])
    m = len(u)
    # bounds of six standard errors, the successive samples being
    # correlated (exp(-1) apart) and so worth about half as many
    assert abs(u.mean()) <= 6 / np.sqrt(m), u.mean()
    assert abs(u.var() - 1.0) <= 6 * np.sqrt(2 / m), u.var()
    assert abs(((u - u.mean()) ** 3).mean()) <= 6 * np.sqrt(6 / m)
    assert abs(((u - u.mean()) ** 4).mean() / u.var() ** 2 - 3.0) <= 8 * np.sqrt(24 / m)
    gs.close()


def test_langevin_thermostat_matches_reference(ctx):
    """The 648-atom TIP3P box with all its forces under LangevinLeapfrog
    (1 fs, 5/ps, 300 K): after 1,000 steps of equilibration the average
    kinetic temperature over the next 2,000 steps matches the reference's
    own LangevinLeapfrog on the same system (tests/golden/
    c1_langevin_temperature.npz, four seeds: 311-316 K; at 1 fs the stiff
    O-H bonds of flexible water leave the kinetic temperature a few per cent
    above the target in both).  The bound, 10 K, is about three times the
    combined scatter of such 2,000-step means."""
    ref = np.load(F.GOLDEN + "/c1_langevin_temperature.npz")["mean_temperature"]
    gs = _c1(ctx)
    mass = F.topology(F.load("c1_leapfrog100")).mass
    it = LangevinLeapfrogIntegrator(1.0, temperature=300.0, gamma=5.0, seed=77)
    it.run(gs, 1000)
    temps = []
    for _ in range(100):
        it.run(gs, 20)
        temps.append(_temperature(gs.velocities(), mass))
    t = float(np.mean(temps))
    assert abs(t - float(ref.mean())) <= 10.0, (t, ref)
    assert t > 300.0  # the integrator's bias has the reference's sign
    gs.close()
