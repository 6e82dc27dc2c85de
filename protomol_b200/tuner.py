"""Autotuner of the batched force-only pair kernel's splits.

The force-only pair kernel divides the tiles of each 8-atom i cluster over
`splits` warps.  One system alone wants many splits to fill the 148 SMs; in
a batched launch over many systems the others fill the device and fewer
splits save the per-warp set-up and the end-of-row reduction.  The best
value depends on the system's size and on the launch it shares, so the
tuner picks one value per size bucket (bucket = floor(log2(i clusters)))
by timing the whole batched launch (coordinate descent over the buckets,
largest first, the other buckets held at their current values).

The table is cached (a JSON file keyed by device name and kernel form), so
a later process takes the same splits without timing anything: results of
a run depend on the splits through FP32 rounding only, and a cached table
makes them reproducible bit for bit.  Choices are deterministic for given
timings (the fastest; ties go to fewer splits).  No counterpart in the
reference, which has no GPU path.
"""
from __future__ import annotations

import json
import math
import os
from typing import Callable, Sequence

CANDIDATES = (1, 2, 3, 4, 6, 8, 12, 16)


def bucket(clusters: int) -> int:
    """Size bucket of a system with `clusters` 8-atom i clusters."""
    return int(math.floor(math.log2(max(1, int(clusters)))))


def choose(times: dict[int, float]) -> int:
    """The candidate with the least time; ties go to fewer splits."""
    return min(times, key=lambda c: (times[c], c))


class SplitTuner:
    def __init__(self, path: str | None = None, key: str = "default",
                 candidates: Sequence[int] = CANDIDATES, reps: int = 10):
        self.path = path
        self.key = key
        self.candidates = tuple(sorted(set(int(c) for c in candidates)))
        self.reps = reps
        self.table: dict[int, int] = {}
        self.timings = 0  # timed launches so far (0 when the cache answered)
        if path and os.path.exists(path):
            self.load()

    # ---- persistence ---------------------------------------------------
    def load(self) -> None:
        with open(self.path) as fh:
            data = json.load(fh)
        entry = data.get(self.key, {})
        self.table = {int(b): int(s) for b, s in entry.items()}

    def save(self) -> None:
        if not self.path:
            return
        data = {}
        if os.path.exists(self.path):
            with open(self.path) as fh:
                data = json.load(fh)
        data[self.key] = {str(b): s for b, s in sorted(self.table.items())}
        tmp = self.path + ".tmp"
        with open(tmp, "w") as fh:
            json.dump(data, fh, indent=1, sort_keys=True)
        os.replace(tmp, self.path)

    # ---- tuning --------------------------------------------------------
    def splits_for(self, clusters: Sequence[int]) -> list[int]:
        """Per-member splits from the table (0: the member's own choice;
        members with no clusters have no specialised kernel)."""
        return [self.table.get(bucket(c), 0) if c > 0 else 0 for c in clusters]

    def tune(self, clusters: Sequence[int], time_fn: Callable[[list[int]], float]) -> dict:
        """Fills the table for the buckets of `clusters` it lacks, timing
        time_fn(per-member splits) -> ms; returns the table."""
        present = sorted({bucket(c) for c in clusters if c > 0}, reverse=True)
        missing = [b for b in present if b not in self.table]
        if not missing:
            return dict(self.table)
        current = self.splits_for(clusters)
        for b in missing:
            times = {}
            for cand in self.candidates:
                trial = [cand if (c > 0 and bucket(c) == b) else s
                         for c, s in zip(clusters, current)]
                times[cand] = float(time_fn(trial))
                self.timings += 1
            best = choose(times)
            self.table[b] = best
            current = [best if (c > 0 and bucket(c) == b) else s
                       for c, s in zip(clusters, current)]
        self.save()
        return dict(self.table)

    def apply(self, ensemble) -> list[int]:
        """Tunes (where the table lacks a bucket) and sets the splits of an
        engine.SystemEnsemble; returns the per-member splits."""
        clusters = [ensemble.member(k)[0] for k in range(len(ensemble.members))]
        self.tune(clusters, lambda sp: ensemble.time_pairs(sp, self.reps))
        splits = self.splits_for(clusters)
        ensemble.set_splits(splits)
        return splits
