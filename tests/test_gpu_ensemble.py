"""The batched ensemble (pmgpu_ensemble_*): every kernel of an MD step is one
launch over all member boxes, members with the same PME grid share one
batched FFT, each segment replays as one CUDA graph.

A member's launches compute exactly what its own launches compute, in
64-bit fixed-point sums, so its trajectory does not depend on the other
members: alone or in a batch, bit for bit, at the same pair-kernel splits.
The boxes below cover both pair-kernel paths (the 120-water box is smaller
than twice the 9 A cutoff and takes the generic minimal-image kernel, the
rest the specialised force-only kernel) and a shared FFT bucket (the two
260-water boxes)."""
import numpy as np
import pytest

from protomol_b200 import serve, tuner
from protomol_b200.engine import (LangevinLeapfrogIntegrator, LeapfrogIntegrator,
                                  SystemEnsemble)

pytestmark = pytest.mark.gpu

SIZES = (120, 260, 260, 400, 700)


def _request(k, nw, integrator="leapfrog"):
    return serve.Request(rid=k, n_waters=nw, seed=31 + k, steps=20, integrator=integrator)


def _members(ctx, sizes=SIZES):
    return [serve.build(ctx, _request(k, nw)) for k, nw in enumerate(sizes)]


def _state(gs):
    return gs.positions(), gs.velocities(), gs.energies()[0]


def _same(a, b):
    return all(np.array_equal(x, y) for x, y in zip(a, b))


def _pair_force(gs):
    return next(f for f in gs.forces if f.stats()["list_entries"] > 0)


def _close(members, ens=None):
    if ens is not None:
        ens.close()
    for gs in members:
        gs.close()


@pytest.mark.parametrize("integ", ["leapfrog", "langevin"])
def test_member_alone_equals_member_in_batch(ctx, integ):
    it = (LeapfrogIntegrator(1.0) if integ == "leapfrog" else
          LangevinLeapfrogIntegrator(1.0, 300.0, 5.0, seed=77))
    ms = _members(ctx)
    ens = SystemEnsemble(ms)
    splits = [ens.member(k)[1] for k in range(len(ms))]
    ens.run(it, 20)
    ens.run(it, 7)  # a second segment (another graph) continues the first
    batched = [_state(gs) for gs in ms]
    info = ens.info()
    assert info["members"] == len(ms) and info["steps"] == 7
    assert info["fft_buckets"] == 4
    _close(ms, ens)
    for k in (0, 1, 4):
        gs = serve.build(ctx, _request(k, SIZES[k]))  # member k's request
        one = SystemEnsemble([gs])
        one.set_splits([max(0, splits[k])])
        one.run(it, 20)
        one.run(it, 7)
        assert _same(_state(gs), batched[k]), k
        _close([gs], one)


def test_ensemble_matches_single_system_runs(ctx):
    """Every member's own pmgpu_run (its own launches, its own FFT plan)
    against the ensemble: the trajectories agree to FP32 rounding of the
    FFT (the batched plan may order its arithmetic differently); the pair
    kernels, the list and the update are the same code."""
    it = LeapfrogIntegrator(1.0)
    ms = _members(ctx)
    ens = SystemEnsemble(ms)
    ens.run(it, 20)
    batched = [_state(gs) for gs in ms]
    _close(ms, ens)
    ms = _members(ctx)
    for k, gs in enumerate(ms):
        it.run(gs, 20)
        x, v, e = _state(gs)
        assert np.abs(x - batched[k][0]).max() <= 1e-6, k
        assert np.abs(e - batched[k][2]).max() <= 1e-6 * np.abs(e).max(), k
    _close(ms)


def test_launches_per_step_do_not_grow_with_members(ctx):
    it = LeapfrogIntegrator(1.0)
    per_step = []
    for sizes in ((120, 400), (120, 260, 260, 400, 700, 300, 500, 150)):
        ms = _members(ctx, sizes)
        ens = SystemEnsemble(ms)
        ens.run(it, 10)
        info = ens.info()
        assert info["graph_replays"] == 1  # the whole 10-step segment
        per_step.append(info["kernels"])
        _close(ms, ens)
    assert per_step[0] == per_step[1], per_step


def test_overflow_inside_a_segment_is_retried_bit_identically(ctx):
    """A member's list rows limited to one tile: the first rebuild inside
    the segment overflows, its list grows, every member goes back to the
    segment start with its list built again there, and the segment runs
    again; the trajectories equal those of a run that never overflowed."""
    it = LeapfrogIntegrator(1.0)
    out = []
    for limit in (None, 1):
        ms = _members(ctx)
        for gs in ms:
            # hot boxes: the lists are rebuilt within the segment
            gs.set_velocities(gs.velocities() * 3.0)
            gs.evaluate()
        if limit:
            ms[3].limit_list_rows(limit)
            cap0 = _pair_force(ms[3]).stats()["list_capacity"]
        ens = SystemEnsemble(ms)
        ens.run(it, 40)
        out.append([_state(gs) for gs in ms])
        if limit:
            st = _pair_force(ms[3]).stats()
            assert st["list_capacity"] > cap0 and st["list_builds"] >= 1, (st, cap0)
        _close(ms, ens)
    for k in range(len(SIZES)):
        assert _same(out[0][k], out[1][k]), k


def test_tuned_splits_are_cached_and_reproducible(ctx, tmp_path):
    path = str(tmp_path / "splits.json")
    it = LeapfrogIntegrator(1.0)
    runs = []
    for attempt in range(2):
        ms = _members(ctx)
        ens = SystemEnsemble(ms)
        tn = tuner.SplitTuner(path, key="lj_c2+ewald", reps=3)
        splits = tn.apply(ens)
        if attempt == 0:
            assert tn.timings > 0 and tn.table
        else:
            assert tn.timings == 0  # the cache answered
        ens.run(it, 10)
        runs.append((splits, [_state(gs) for gs in ms]))
        _close(ms, ens)
    assert runs[0][0] == runs[1][0]
    for a, b in zip(runs[0][1], runs[1][1]):
        assert _same(a, b)
