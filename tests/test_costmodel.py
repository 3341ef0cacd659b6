"""Autotuner pieces that need no GPU: the cost-model oracle (its gradient against finite
differences, Adam), the candidate blocks, the features and the seeded corpus sampler."""

import math

import numpy as np
import pytest

from oracle import mlp_oracle as M


def _params(n_in, h, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(M.param_count(n_in, h)) * 0.3


def test_oracle_gradient_matches_finite_differences():
    n_in, h, n = 5, 7, 11
    rng = np.random.default_rng(0)
    p = _params(n_in, h, 1)
    x = rng.standard_normal((n, n_in))
    t = rng.standard_normal(n)
    loss, g = M.gradient(p, x, t, n_in, h)
    assert g.shape == p.shape
    assert math.isclose(loss, float(np.mean((M.forward(p, x, n_in, h) - t) ** 2)), rel_tol=1e-12)
    eps = 1e-6
    for i in rng.choice(p.size, size=40, replace=False):
        q = p.copy()
        q[i] += eps
        lp = np.mean((M.forward(q, x, n_in, h) - t) ** 2)
        q[i] -= 2 * eps
        lm = np.mean((M.forward(q, x, n_in, h) - t) ** 2)
        assert abs((lp - lm) / (2 * eps) - g[i]) <= 1e-6 * max(1.0, abs(g[i]))


def test_oracle_adam_first_step_moves_by_lr():
    p = np.zeros(4)
    g = np.array([1.0, -2.0, 0.5, 0.0])
    q, m, v = M.adam(p, g, np.zeros(4), np.zeros(4), 1, 0.01)
    # bias-corrected first step: -lr * sign(g) (up to eps) where g != 0
    assert np.allclose(q[:3], -0.01 * np.sign(g[:3]), atol=1e-6) and q[3] == 0.0


def test_candidate_blocks():
    from threadcoarsenedstencilgenerator_b200.autotune import candidate_blocks

    b2, b3 = candidate_blocks(2), candidate_blocks(3)
    assert len(b2) == 51 and len(b3) == 231
    for b in b2 + b3:
        n = b[0] * b[1] * b[2]
        assert 32 <= n <= 1024 and n & (n - 1) == 0 and b[2] <= 64
    assert all(b[2] == 1 for b in b2)
    assert len(set(b3)) == len(b3)


def test_features_and_sampler():
    from threadcoarsenedstencilgenerator_b200 import StencilSpec
    from threadcoarsenedstencilgenerator_b200.autotune import FEATURES, TERM_BUDGET, corpus_grid, features, \
        sample_configs

    specs = sample_configs(40, seed=7)
    assert specs == sample_configs(40, seed=7)
    assert len({repr(s) for s in specs}) == 40
    for s in specs:
        assert s.stencil_size * s.cx * s.cy * (s.cz if s.dimension == 3 else 1) <= TERM_BUDGET
        assert 1 <= s.range <= 8 and max(s.cx, s.cy, s.cz) <= 8
    spec = StencilSpec(dimension=3, neighbourhood="Star", coefficients="Variable", range=2, cx=2, cy=1, cz=4)
    geom = spec.geometry(*corpus_grid(spec))
    assert geom.n_points * 8 <= (512 << 20) * 1.05
    from types import SimpleNamespace

    plan = SimpleNamespace(grid_blocks=(8, 8, 4), ctas_per_sm=2, num_sms=148)
    f = features(spec, geom, (32, 4, 2), 256, plan)
    assert f.shape == (len(FEATURES),) and f.dtype == np.float32
    d = dict(zip(FEATURES, f))
    assert d["dim3"] == 1 and d["star"] == 1 and d["variable"] == 1 and d["f64"] == 1
    assert d["log_tile_x"] == 6 and d["log_tile_z"] == 3 and d["log_threads"] == 8
    assert d["log_S"] == pytest.approx(math.log2(13))
    assert d["log_warps_per_sm"] == pytest.approx(math.log2(2 * 256 / 32))
    assert d["tail_efficiency"] == pytest.approx(256 / 296)


def test_tuned_entries_per_precision(tmp_path, monkeypatch):
    """A workload's FP32 sweeps take the `<name>_f32` entry of tuned.json when there is one, else
    the FP64 entry; the workload's own precision is kept."""
    import json

    from threadcoarsenedstencilgenerator_b200 import workloads as W

    w = W.WORKLOADS["2d_box_var_r6_16384x8192"]
    p = tmp_path / "tuned.json"
    p.write_text(json.dumps({w.name: {"coarsening": [4, 1, 1], "block": [32, 1, 1], "variant": "pipe", "chunk": 1}}))
    monkeypatch.setattr(W, "TUNED_PATH", p)
    assert w.tuned_spec("f32").coarsening == w.tuned_spec().coarsening == (4, 1, 1)
    assert w.tuned_launch("f32").block == (32, 1, 1)
    d = json.loads(p.read_text())
    d[w.name + "_f32"] = {"coarsening": [8, 1, 1], "block": [64, 1, 1], "variant": "pipe", "chunk": 2}
    p.write_text(json.dumps(d))
    assert w.tuned_spec("f32").coarsening == (8, 1, 1)
    assert w.tuned_spec("f32").precision == w.spec.precision
    assert w.tuned_launch("f32").block == (64, 1, 1) and w.tuned_launch("f32").chunk == 2
    assert w.tuned_spec().coarsening == (4, 1, 1) and w.tuned_launch().block == (32, 1, 1)
