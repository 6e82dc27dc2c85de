"""The pair-kernel split autotuner's table logic on the CPU: size buckets,
the deterministic choice, coordinate descent over the buckets present, the
JSON cache (a second tuner answers from it without timing anything)."""
import json

from protomol_b200 import tuner


def test_buckets_are_floor_log2_of_clusters():
    assert [tuner.bucket(c) for c in (1, 2, 3, 4, 7, 8, 300, 511, 512)] == \
        [0, 1, 1, 2, 2, 3, 8, 8, 9]
    assert tuner.bucket(0) == 0


def test_choice_is_the_fastest_and_ties_go_to_fewer_splits():
    assert tuner.choose({1: 3.0, 2: 1.0, 4: 2.0}) == 2
    assert tuner.choose({8: 1.0, 2: 1.0, 4: 1.0}) == 2


def _model(clusters, splits):
    """A fake launch time: each member wants its own best splits (4 for the
    small ones, 2 for the large) and pays for the distance from it."""
    t = 0.0
    for c, s in zip(clusters, splits):
        want = 4 if c < 64 else 2
        s = s or 8
        t += c * (1.0 + abs(s - want))
    return t


def test_tune_picks_each_buckets_optimum_and_caches(tmp_path):
    path = str(tmp_path / "t.json")
    clusters = [40, 40, 50, 300, 310, 0]  # the last: no specialised kernel
    tn = tuner.SplitTuner(path, key="k", candidates=(1, 2, 4, 8))
    calls = []
    table = tn.tune(clusters, lambda sp: calls.append(list(sp)) or _model(clusters, sp))
    assert table == {5: 4, 8: 2}
    assert len(calls) == 2 * 4 and tn.timings == 8
    # the largest bucket first, the others held at their current values
    assert calls[0] == [0, 0, 0, 1, 1, 0]
    assert tn.splits_for(clusters) == [4, 4, 4, 2, 2, 0]
    with open(path) as fh:
        assert json.load(fh) == {"k": {"5": 4, "8": 2}}
    again = tuner.SplitTuner(path, key="k")
    assert again.tune(clusters, lambda sp: 1 / 0) == table and again.timings == 0
    # a new bucket is timed, the cached ones are not
    more = clusters + [1000]
    assert again.tune(more, lambda sp: _model(more, sp))[9] == 2
    assert again.timings == len(tuner.CANDIDATES)
    other = tuner.SplitTuner(path, key="other")
    assert other.table == {}


def test_apply_sets_the_ensemble_splits(tmp_path):
    class FakeEnsemble:
        def __init__(self):
            self.members = [None] * 3
            self.set = None

        def member(self, k):
            return ([20, 200, 0][k], 8)

        def time_pairs(self, splits, reps):
            return _model([20, 200, 0], splits)

        def set_splits(self, splits):
            self.set = list(splits)

    fe = FakeEnsemble()
    tn = tuner.SplitTuner(str(tmp_path / "a.json"), candidates=(2, 4))
    assert tn.apply(fe) == [4, 2, 0] and fe.set == [4, 2, 0]
