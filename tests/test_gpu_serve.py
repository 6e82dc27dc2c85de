"""Batched / served forms on the GPU: results in the mix equal results
alone (bit for bit), and small boxes (edges below twice the cutoff, where
the real-space sum sees several images) agree with the oracle."""
import numpy as np
import pytest

import fixtures as F
import oracle
from oracle import spme
from protomol_b200 import ForceFactory, GpuSystem, PMEwaldSystemForce, ScalarStructure, serve
from protomol_b200 import systems

pytestmark = pytest.mark.gpu


def _mix():
    reqs = [serve.Request(rid=0, n_waters=120, seed=11, steps=40),
            serve.Request(rid=1, n_waters=400, seed=12, kind="evaluate", steps=0),
            serve.Request(rid=2, n_waters=900, seed=13, steps=30, integrator="leapfrog"),
            serve.Request(rid=3, n_waters=250, seed=14, steps=25),
            serve.Request(rid=4, n_waters=600, seed=15, kind="evaluate", steps=0),
            serve.Request(rid=5, n_waters=150, seed=16, steps=60)]
    return reqs


def test_served_results_equal_alone(ctx):
    alone = [serve.execute(ctx, r) for r in _mix()]
    mixed = _mix()
    stats = serve.Server(ctx, slots=4).run(mixed, realtime=False)
    assert stats["failed"] == 0
    assert stats["peak_in_flight"] >= 2
    for a, m in zip(alone, sorted(mixed, key=lambda r: r.rid)):
        assert np.array_equal(a.energies, m.energies), a.rid
        if a.kind == "evaluate":
            assert np.array_equal(a.forces, m.forces), a.rid
        else:
            assert np.array_equal(a.positions, m.positions), a.rid


def test_reused_shells_give_the_results_of_new_systems(ctx):
    """Requests on boxes of one shape (different seeds) run one after the
    other in shells from the pool: new positions, velocities and step
    counter, every list built afresh; each result equals the request run
    in a new system, bit for bit (Langevin noise included)."""
    shapes = [(250, "segment", 30), (250, "evaluate", 0), (250, "segment", 30),
              (400, "segment", 20), (400, "segment", 20), (250, "evaluate", 0)]

    def reqs():
        return [serve.Request(rid=k, n_waters=nw, seed=40 + k, kind=kind, steps=st)
                for k, (nw, kind, st) in enumerate(shapes)]

    alone = [serve.execute(ctx, r) for r in reqs()]
    srv = serve.Server(ctx, slots=1)
    pooled = reqs()
    stats = srv.run(pooled, realtime=False)
    srv.close()
    assert stats["failed"] == 0 and stats["shells_reused"] >= 3, stats
    for a, m in zip(alone, sorted(pooled, key=lambda r: r.rid)):
        assert np.array_equal(a.energies, m.energies), a.rid
        if a.kind == "evaluate":
            assert np.array_equal(a.forces, m.forces), a.rid
        else:
            assert np.array_equal(a.positions, m.positions), a.rid


def test_admission_respects_memory_budget(ctx):
    srv = serve.Server(ctx, slots=8)
    reqs = _mix()
    # a budget that holds the largest request alone: requests are admitted
    # only while their footprints fit beside the ones in flight
    fps = sorted(r.footprint() for r in reqs)
    srv.budget = fps[-1]
    stats = srv.run(reqs, realtime=False)
    assert stats["failed"] == 0
    assert stats["peak_footprint_bytes"] <= srv.budget
    assert stats["peak_in_flight"] < len(reqs)


def _oracle_system(sm):
    return oracle.System(pos=sm.pos, charge=sm.charge, type=sm.type, molecule=sm.molecule,
                         lj=sm.lj, excl=sm.exclusions.astype(np.int32),
                         coulomb_scaling=sm.coulomb_scaling, periodic=True, box=sm.box,
                         mass=sm.mass)


def _eval(force, n, pos):
    f = np.zeros((n, 3))
    e = ScalarStructure()
    force.evaluate(pos, f, e)
    return f, e


def test_small_box_vs_oracle(ctx):
    """180 waters at liquid density: edge 17.5 A, below twice the 9 A
    cutoff.  LJ (minimal image only), Ewald real space (every image inside
    the cutoff) and PME against the oracle."""
    sm = systems.water_box_for_density(180, serve.WATER_DENSITY, 5, jitter=0.2)
    L = sm.box[0]
    assert 9.0 < L < 18.0
    n = sm.pos.shape[0]
    s = _oracle_system(sm)
    gs = GpuSystem(ctx, sm, "mixed")
    ff = ForceFactory(gs, 9.0)
    lj = ff.make("LennardJones -algorithm NonbondedCutoff -switchingFunction C2 -switchon 8 "
                 "-cutoff 9 -cutoff 9")
    f, e = _eval(lj, n, sm.pos)
    fo, eo, _ = oracle.cutoff_force(s, 9.0, 9.0, [("LennardJones", oracle.Switch("C2", 9.0, 8.0))])
    assert F.rms_rel(f, fo) <= 1e-5, F.rms_rel(f, fo)
    assert abs(e[1] - eo["lj"]) <= 1e-6 * abs(eo["lj"]) + 1e-4
    lj.set_enabled(False)
    alpha = 0.35
    acc = float(np.exp(-(alpha * 9.0) ** 2))
    ew = oracle.ewald_params(s, alpha, acc)
    real = PMEwaldSystemForce(gs, alpha, 9.0, real=True, reciprocal=False, correction=False)
    f, e = _eval(real, n, sm.pos)
    fo, eo = oracle.ewald_real(s, ew, 9.0)[:2]
    assert F.rms_rel(f, fo) <= 1e-5, F.rms_rel(f, fo)
    assert abs(e[0] - eo) <= 1e-6 * abs(eo) + 1e-4
    real.set_enabled(False)
    K = serve.fft_size(int(np.ceil(L)))
    rec = PMEwaldSystemForce(gs, alpha, 0.0, order=4, grid=(K, K, K), real=False,
                             reciprocal=True, correction=False)
    f, e = _eval(rec, n, sm.pos)
    fo, eo = spme.reciprocal(sm.pos, sm.charge, L, alpha, 4, K)
    assert F.rms_rel(f, fo) <= 1e-5, F.rms_rel(f, fo)
    assert abs(e[0] - eo) <= 1e-5 * abs(eo)
    gs.close()
