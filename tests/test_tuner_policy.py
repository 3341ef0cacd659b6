"""The learned tuner's decisions, on the CPU with scripted timings and predictions.

Autotuner.tune ranks the candidates with the model, times the top 5 and keeps the best unless the
measured log-throughput differences disagree with the predicted ones by more than the tolerance;
then it times the same 5 again over twice the sweeps, keeps each block's faster timing (noise
only slows a run down), and only if the disagreement stays does it run the exhaustive sweep.  The
feature, timing and model calls are replaced here, so no GPU is needed.
"""

import math

import numpy as np
import pytest

from threadcoarsenedstencilgenerator_b200 import autotune as A

BLOCKS = [(32 * (i + 1), 1, 1) for i in range(12)]


class FakeModel:
    def __init__(self, pred, in_domain=True):
        self.pred = np.asarray(pred, dtype=np.float64)
        self._in = in_domain

    def predict(self, X):
        return self.pred[: len(X)]

    def in_domain(self, X):
        return self._in


class FakeSpec:
    dimension = 2


class FakeStencil:
    spec = FakeSpec()


@pytest.fixture
def timings(monkeypatch):
    """Script time_block: glups[block] for 2-sweep timings, glups4[block] for the re-timings."""
    calls = []
    state = {"glups": {}, "glups4": {}}

    def time_block(st, geom, x, y, block, sweeps=2):
        calls.append((tuple(block), sweeps))
        table = state["glups4"] if sweeps > 2 and state["glups4"] else state["glups"]
        return table.get(tuple(block))

    def exhaustive(st, geom, x, y, blocks, sweeps=2):
        return [(tuple(b), state["glups"][tuple(b)]) for b in blocks if tuple(b) in state["glups"]]

    monkeypatch.setattr(A, "candidate_blocks", lambda dim: list(BLOCKS))
    monkeypatch.setattr(A, "candidate_features", lambda st, geom, blocks: (list(blocks), np.zeros((len(blocks), 3))))
    monkeypatch.setattr(A, "time_block", time_block)
    monkeypatch.setattr(A, "exhaustive", exhaustive)
    return state, calls


def _pred_from(glups):
    """Predictions that agree exactly with the timings (log throughput, any offset)."""
    return [math.log(glups[b]) + 0.3 for b in BLOCKS]


def test_no_model_runs_the_sweep(timings):
    state, calls = timings
    state["glups"] = {b: 10.0 + i for i, b in enumerate(BLOCKS)}
    r = A.Autotuner(None).tune(FakeStencil(), None, None, None)
    assert r.fell_back and r.reason == "no model" and r.block == BLOCKS[-1] and r.timed == len(BLOCKS)


def test_consistent_model_times_its_top_5_only(timings):
    state, calls = timings
    state["glups"] = {b: 10.0 + i for i, b in enumerate(BLOCKS)}
    r = A.Autotuner(FakeModel(_pred_from(state["glups"]))).tune(FakeStencil(), None, None, None)
    assert not r.fell_back and r.timed == 5 and r.block == BLOCKS[-1]
    assert [c[0] for c in calls] == BLOCKS[::-1][:5]  # in predicted order
    assert r.model_error == pytest.approx(0.0, abs=1e-12)


def test_out_of_domain_runs_the_sweep(timings):
    state, calls = timings
    state["glups"] = {b: 10.0 for b in BLOCKS}
    r = A.Autotuner(FakeModel(_pred_from(state["glups"]), in_domain=False)).tune(FakeStencil(), None, None, None)
    assert r.fell_back and "outside" in r.reason


def test_noisy_timing_is_timed_again_before_falling_back(timings):
    state, calls = timings
    state["glups"] = {b: 10.0 + i for i, b in enumerate(BLOCKS)}
    pred = _pred_from(state["glups"])
    noisy = dict(state["glups"])
    noisy[BLOCKS[-2]] = 2.0  # one 2-sweep timing far off
    state["glups"], state["glups4"] = noisy, {b: 10.0 + i for i, b in enumerate(BLOCKS)}
    r = A.Autotuner(FakeModel(pred)).tune(FakeStencil(), None, None, None)
    assert not r.fell_back and r.block == BLOCKS[-1]
    assert sum(1 for c in calls if c[1] == 4) == 5  # the 5 timed again over twice the sweeps
    assert r.model_error <= 0.25


def test_model_that_stays_wrong_falls_back_to_the_sweep(timings):
    state, calls = timings
    state["glups"] = {b: 10.0 + i for i, b in enumerate(BLOCKS)}
    wrong = [-v for v in _pred_from(state["glups"])]  # ranks the blocks backwards
    wrong = [w + (5.0 if i == 0 else 0.0) for i, w in enumerate(wrong)]
    r = A.Autotuner(FakeModel(wrong)).tune(FakeStencil(), None, None, None)
    assert r.fell_back and "prediction error" in r.reason and r.model_error > 0.25
    assert r.block == BLOCKS[-1] and r.timed == len(BLOCKS)
