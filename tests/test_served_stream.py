"""Host side of the batched and served forms (no device needed): the seeded
request stream (log-uniform atom counts, the evaluation/segment mix,
Poisson arrivals), the ensemble's box shapes and PME grids, the per-system
footprint that admission compares with free device memory, and the
latency/throughput summary."""
import math

import numpy as np
import pytest

from protomol_b200 import serve


def _smooth(m):
    for p in (2, 3, 5):
        while m % p == 0:
            m //= p
    return m == 1


@pytest.mark.parametrize("n", [1, 7, 13, 31, 37, 62, 97, 121, 250])
def test_fft_size_is_the_next_5_smooth_length(n):
    g = serve.fft_size(n)
    assert g >= n and _smooth(g)
    assert not any(_smooth(m) for m in range(n, g))


def test_request_stream_shape():
    """2,000 requests as configured: 500-50,000 atoms log-uniform (rounded
    to whole waters), 30 % single evaluations, Poisson arrivals."""
    rate = 20.0
    reqs = serve.request_stream(2000, 7, rate_per_s=rate)
    again = serve.request_stream(2000, 7, rate_per_s=rate)
    assert [(r.n_waters, r.kind, r.seed, r.arrival) for r in reqs] == \
        [(r.n_waters, r.kind, r.seed, r.arrival) for r in again]
    atoms = np.array([r.n_atoms for r in reqs])
    assert atoms.min() >= 500 - 1 and atoms.max() <= 50000 + 1
    # log-uniform: the log of the count is uniform, so its median sits at
    # the geometric mean and each decade holds half the requests
    logs = np.log(atoms)
    assert abs(np.median(logs) - 0.5 * (math.log(500) + math.log(50000))) < 0.15
    assert abs(np.mean(atoms < 5000) - 0.5) < 0.05
    ev = np.mean([r.kind == "evaluate" for r in reqs])
    assert abs(ev - 0.3) < 0.04
    assert all(r.steps == (0 if r.kind == "evaluate" else 1000) for r in reqs)
    t = np.array([r.arrival for r in reqs])
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert np.all(gaps >= 0)
    # exponential gaps: mean 1/rate, standard deviation equal to the mean
    assert abs(gaps.mean() * rate - 1.0) < 0.08
    assert abs(gaps.std() / gaps.mean() - 1.0) < 0.1
    assert all(r.arrival == 0.0 for r in serve.request_stream(10, 3))


def test_ensemble_boxes_and_grids():
    """256 boxes of 100-1,000 waters at 0.0334 waters/A^3: edges 14.4-31.0
    A, PME grids of at most 1 A spacing with 2^a 3^b 5^c points."""
    boxes = serve.ensemble(256, 11)
    assert len(boxes) == 256
    nw = np.array([b.n_waters for b in boxes])
    assert nw.min() >= 100 and nw.max() <= 1000
    for b in boxes:
        assert 14.3 < b.edge < 31.1
        assert b.grid >= b.edge / serve.SPACING and _smooth(b.grid)
        assert b.kind == "segment" and b.steps == 50 and b.integrator == "leapfrog"
    assert np.mean([b.edge < 18.0 for b in boxes]) > 0.15  # multi-image real space


def test_footprint_grows_with_the_system():
    """Admission compares this estimate with free device memory: it must grow
    with the atom count and stay within a sane range per atom."""
    small = serve.Request(rid=0, n_waters=200, seed=1)
    large = serve.Request(rid=1, n_waters=16000, seed=1)
    fs, fl = small.footprint(), large.footprint()
    assert 0 < fs < fl
    assert 1e3 < fl / large.n_atoms < 1e5  # bytes per atom


def test_summary_statistics():
    reqs = []
    for k in range(100):
        r = serve.Request(rid=k, n_waters=100, seed=k, kind="segment", steps=1000,
                          arrival=float(k))
        r.t_done = r.arrival + 0.01 * (k + 1)  # latencies 0.01 .. 1.00 s
        reqs.append(r)
    bad = serve.Request(rid=100, n_waters=100, seed=0, arrival=0.0)
    bad.error = "refused"
    s = serve.summarize(reqs + [bad], wall=10.0, slots=4, peak=3)
    assert s["requests"] == 101 and s["failed"] == 1
    assert s["p50_latency_s"] == pytest.approx(np.percentile(0.01 * np.arange(1, 101), 50))
    assert s["p99_latency_s"] == pytest.approx(np.percentile(0.01 * np.arange(1, 101), 99))
    # 100 segments of 1,000 fs steps in 10 s: 1e-4 ns per second
    assert s["ns_per_day"] == pytest.approx(100 * 1000 * 1e-6 * 86400 / 10.0)
    assert s["atom_steps_per_s"] == pytest.approx(100 * 300 * 1000 / 10.0)
