"""The pipelined-launch tuner's host logic (no GPU): candidate space, analytic features, corpus
plan, hold-out split, and the tuner's choices with scripted timings."""

import math

import numpy as np
import pytest

from threadcoarsenedstencilgenerator_b200 import pipetune as P
from threadcoarsenedstencilgenerator_b200.spec import StencilSpec


def test_candidates_respect_the_kernel_limits():
    for base in P.sample_problems(40):
        cands = P.candidates(base)
        assert cands, base
        vec = 16 // base.itemsize
        for cx, cy, bx, by, ch in cands:
            tx = bx * cx
            assert tx % vec == 0 and tx + 2 * base.range + vec <= 256
            if base.dimension == 3:
                assert 64 <= bx * by <= 1024 and ch in (2, 3)
            else:
                assert by == 1 and cy == 1 and ch in (1, 2)
        assert len(set(cands)) == len(cands)


def test_features_are_analytic_and_finite():
    base = StencilSpec(dimension=3, neighbourhood="Star", coefficients="Variable", range=4)
    grid = P.corpus_grid(base)
    X = np.stack([P.features(base, grid, c) for c in P.candidates(base)])
    assert X.shape[1] == len(P.PIPE_FEATURES)
    assert np.all(np.isfinite(X))
    # the tuned launch of the 512^3 workload (2x4 coarsening, 64x4 block, 3 planes) is in the space
    assert (2, 4, 64, 4, 3) in P.candidates(base)
    f = dict(zip(P.PIPE_FEATURES, P.features(base, (512, 512, 512), (2, 4, 64, 4, 3))))
    assert f["log_tile_x"] == 7 and f["log_tile_y"] == 4 and f["chunk"] == 3
    assert math.isclose(f["loads_per_lup"], (8 + 8 * 6) / 8)


def test_corpus_plan_and_holdout_are_seeded():
    a, b = P.corpus_plan(12, 10), P.corpus_plan(12, 10)
    assert [(p, c) for p, _, _, c in a] == [(p, c) for p, _, _, c in b]
    hold = P.holdout_ids(40)
    assert hold == P.holdout_ids(40) and len(hold) == 8
    pids = np.array([0, 1, hold[0], 2])
    h, mask = P.split(pids, 40)
    assert h == hold and list(mask) == [p not in hold for p in pids]


class _FakeModel:
    """Predicts a fixed ordering: log throughput = -(index in the candidate list) * slope."""

    def __init__(self, slope=0.01, in_domain=True):
        self.slope, self._in = slope, in_domain

    def predict(self, X):
        return -self.slope * np.arange(len(X), dtype=np.float32)

    def in_domain(self, X):
        return self._in


@pytest.mark.parametrize("scenario", ["agrees", "disagrees", "outside"])
def test_tuner_times_top_k_or_falls_back(monkeypatch, scenario):
    base = StencilSpec(dimension=3, neighbourhood="Star", coefficients="Jacobi", range=2)
    cands = P.candidates(base)
    timings = {c: 100.0 - 0.1 * i for i, c in enumerate(cands)}  # best first, as the model predicts
    if scenario == "disagrees":
        timings[cands[3]] = 300.0  # a much faster candidate the model ranks 4th: large prediction error
    timed = []

    def fake_time(b, grid, cand, mask, bufs, sweeps=3):
        timed.append(cand)
        return timings[cand]

    monkeypatch.setattr(P, "time_candidate", fake_time)
    model = _FakeModel(in_domain=scenario != "outside")
    r = P.PipeTuner(model, top_k=5).tune(base, (100, 100, 100))
    if scenario == "agrees":
        assert not r.fell_back and r.timed == 5 and r.candidate == cands[0] and len(timed) == 5
    else:
        assert r.fell_back and len(timed) == 5 * (scenario == "disagrees") + len(cands)
        assert r.candidate == max(timings, key=timings.get)
