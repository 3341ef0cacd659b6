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

    def fake_time(b, grid, cand, mask, bufs, sweeps=3, form=(0, 0)):
        timed.append((cand, form))
        # the lockstep ring form is faster, the other non-default forms slower
        return timings[cand] + {(0, 0): 0.0, (1, 1): 5.0}.get(tuple(form), -1.0)

    monkeypatch.setattr(P, "time_candidate", fake_time)
    model = _FakeModel(in_domain=scenario != "outside")
    r = P.PipeTuner(model, top_k=5).tune(base, (100, 100, 100))
    forms_of = lambda cs: sum(len(P.forms(base, c)) for c in cs)  # noqa: E731
    if scenario == "agrees":
        # the model's top 5 shapes in the default form, then their other forms
        assert not r.fell_back and r.candidate == cands[0]
        assert len(timed) == r.timed == forms_of(cands[:5])
        assert r.form == ((1, 1) if P.tmem_applies(base, cands[0]) else (0, 0))
    else:
        assert r.fell_back and len(timed) == 5 * (scenario == "disagrees") + forms_of(cands)
        best = max(timings, key=lambda c: timings[c] + (5.0 if P.tmem_applies(base, c) else 0.0))
        assert r.candidate == best
    assert r.candidates == forms_of(cands)


def test_write_tuned_records_a_launch_the_workload_reads(tmp_path, monkeypatch):
    """The tuner's record is the tuned-launch format: the workload turns it back into the same
    coarsening, block and chunk; other entries of the file survive."""
    from threadcoarsenedstencilgenerator_b200 import workloads as W

    path = tmp_path / "tuned.json"
    path.write_text('{"other": {"block": [8, 8, 1]}}\n')
    r = P.PipeTuneResult((2, 2, 64, 8, 3), 270.0, 140, 148, True, 1.0, "no model",
                         {(2, 2, 64, 8, 3): 270.0, (2, 4, 64, 4, 3): 269.6})
    e = P.write_tuned(path, "3d_star_var_r4_512", "f64", r)
    assert "269.6" in e["source"] and "exhaustive" in e["source"]
    P.write_tuned(path, "3d_star_var_r4_512", "f32",
                  P.PipeTuneResult((1, 4, 128, 4, 2), 400.0, 5, 148, False, 0.1, "model top-5", {}))
    monkeypatch.setattr(W, "TUNED_PATH", path)
    w = W.WORKLOADS["3d_star_var_r4_512"]
    L, s = w.tuned_launch(), w.tuned_spec()
    assert (L.variant, tuple(L.block), L.chunk) == ("pipe", (64, 8, 1), 3)
    assert (s.cx, s.cy, s.cz) == (2, 2, 1)
    L32, s32 = w.tuned_launch("f32"), w.tuned_spec("f32")
    assert (tuple(L32.block), L32.chunk, s32.cx, s32.cy) == ((128, 4, 1), 2, 1, 4)
    import json

    assert json.loads(path.read_text())["other"] == {"block": [8, 8, 1]}


def test_forms_follow_the_ring_form_rules():
    """The ring form is offered exactly where the library builds it: 3D Star Row, FP64/FP32,
    4..32 TMEM columns per ring entry within 512, blocks of whole warps."""
    star = StencilSpec(dimension=3, neighbourhood="Star", coefficients="Variable", range=4)
    assert P.tmem_applies(star, (2, 4, 64, 7, 2)) and P.tmem_applies(star, (2, 2, 64, 8, 3))
    assert not P.tmem_applies(star, (4, 4, 64, 8, 2))      # 4 column groups x 8 entries x 32 > 512
    assert not P.tmem_applies(star, (1, 1, 32, 1, 2))      # 2 columns per entry
    assert not P.tmem_applies(star.replace(neighbourhood="Box"), (2, 4, 64, 4, 2))
    assert not P.tmem_applies(star.replace(precision="f32c"), (2, 4, 64, 4, 2))
    assert P.forms(star.replace(neighbourhood="Box"), (2, 4, 64, 4, 2)) == [(0, 0), (0, 1)]
    L = P.launch_of((2, 4, 64, 7, 2), (1, 1))
    assert L.tmem and L.lockstep and L.to_c().flags == P._lib.LAUNCH_TMEM | P._lib.LAUNCH_LOCKSTEP


def test_tuned_entry_records_the_form(tmp_path, monkeypatch):
    from threadcoarsenedstencilgenerator_b200 import workloads as W

    path = tmp_path / "tuned.json"
    r = P.PipeTuneResult((2, 4, 64, 7, 2), 324.0, 600, 640, True, 1.0, "no model",
                         {(2, 4, 64, 7, 2, 1, 1): 324.0, (2, 4, 64, 7, 2, 1, 0): 289.0}, (1, 1))
    e = P.write_tuned(path, "3d_star_var_r4_512", "f64", r)
    assert e["tmem"] and e["lockstep"] and "289.0" in e["source"]
    monkeypatch.setattr(W, "TUNED_PATH", path)
    L = W.WORKLOADS["3d_star_var_r4_512"].tuned_launch()
    assert (tuple(L.block), L.chunk, L.tmem, L.lockstep) == ((64, 7, 1), 2, True, True)


def test_batch_candidates_and_record(tmp_path, monkeypatch):
    """The batched search covers blocks within the TMA box and the thread limits; its record is
    what the batch workload reads back (block and chunk on the batch's own coarsening)."""
    from threadcoarsenedstencilgenerator_b200 import workloads as W

    w = W.BATCH_WORKLOADS["batch_3d_star_jacobi_r2_64"]
    cands = P.batch_candidates(w.spec)
    assert cands and all(64 <= bx * by <= 1024 and bx * w.spec.cx + 2 * w.spec.range + 2 <= 256
                         for bx, by, ch in cands)
    assert {ch for _, _, ch in cands} == {1, 2, 3}
    path = tmp_path / "tuned.json"
    r = P.PipeTuneResult((64, 4, 3, 1776), 230.0, 39, 39, True, 1.0, "batched sweep: exhaustive",
                         {(64, 4, 3, 1776): 230.0, (32, 8, 2, 0): 228.0})
    e = P.write_tuned(path, w.name, "f32", r, batch=True)
    assert e["block"] == [64, 4, 1] and e["chunk"] == 3 and e["segments"] == 1776 and "228.0" in e["source"]
    monkeypatch.setattr(W, "TUNED_PATH", path)
    L = w.tuned_launch("f32")
    assert (tuple(L.block), L.chunk, L.variant, L.segments) == ((64, 4, 1), 3, "pipe", 1776)


def test_batch_tuner_searches_cta_counts_of_its_fastest_shapes(monkeypatch):
    """Stage 1 times every shape at one wave; stage 2 times the three fastest at BATCH_WAVES waves
    of CTAs, and the record keeps the fastest (shape, CTA count) (scripted timings, no GPU)."""
    from threadcoarsenedstencilgenerator_b200 import workloads as W

    w = W.BATCH_WORKLOADS["batch_3d_star_jacobi_r2_64"]
    timed = []

    def fake_time(w_, prec, cand, state, sweeps=10):
        timed.append(tuple(cand))
        bx, by, ch, ctas = cand
        return 100.0 + bx * by / 64.0 + ch + (ctas == 12 * 148 and (bx, by, ch) == (64, 8, 3)) * 50.0

    monkeypatch.setattr(P, "time_batch", fake_time)
    r = P.tune_batch(w, "f32", num_sms=148)
    shapes = P.batch_candidates(w.spec)
    assert len(timed) == len(shapes) + 3 * (len(P.BATCH_WAVES) - 1)
    assert all(t[3] == 0 for t in timed[:len(shapes)])
    assert {t[3] for t in timed[len(shapes):]} == {k * 148 for k in P.BATCH_WAVES[1:]}
    e = P.batch_entry(r)
    if (64, 8, 3) in {tuple(t[:3]) for t in timed[len(shapes):]}:
        assert r.candidate == (64, 8, 3, 12 * 148) and e["segments"] == 12 * 148
