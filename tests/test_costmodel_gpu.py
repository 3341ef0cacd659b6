"""The cost model's GPU kernels against the float64 oracle, its training, and what the trained
model gains over choosing blocks without it.

Tolerances: FP32 kernels against the float64 oracle -- forward outputs within 1e-5 of the output
scale, gradients within 1e-4 of the largest gradient component, the Adam update (fed with the
kernels' own gradient) within 1e-6 absolute of the oracle's (the step is about lr = 1e-3).
"""

import numpy as np
import pytest

from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu


def _data(n, n_in, seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, n_in)).astype(np.float32)
    t = (np.sin(x[:, 0]) + 0.5 * x[:, 1] * x[:, 2 % n_in]).astype(np.float32)
    return x, t


@pytest.fixture(scope="module")
def model():
    from threadcoarsenedstencilgenerator_b200.autotune import CostModel, init_params

    m = CostModel(n_in=9, hidden=128, max_batch=512, params=init_params(9, 128, 5))
    yield m
    m.close()


def test_forward_and_gradient_match_oracle(model):
    import torch

    from threadcoarsenedstencilgenerator_b200.autotune import init_params

    p = init_params(9, 128, 5)
    model.set_params(p)
    x, t = _data(300, 9, 1)
    xd, td = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    y = torch.empty(300, device="cuda")
    model.forward_raw(xd, y)
    want = M.forward(p, x, 9, 128)
    assert np.max(np.abs(y.cpu().numpy() - want)) <= 1e-5 * max(1.0, np.max(np.abs(want)))
    g = torch.empty(model.n_params, device="cuda")
    loss = model.gradient_raw(xd, td, g)
    wl, wg = M.gradient(p, x, t, 9, 128)
    assert abs(loss - wl) <= 1e-5 * max(1.0, wl)
    gg = g.cpu().numpy()
    assert np.max(np.abs(gg - wg)) <= 1e-4 * np.max(np.abs(wg))
    # forward beyond one batch of buffers
    x2, _ = _data(1300, 9, 2)
    y2 = torch.empty(1300, device="cuda")
    model.forward_raw(torch.from_numpy(x2).cuda(), y2)
    assert np.max(np.abs(y2.cpu().numpy() - M.forward(p, x2, 9, 128))) <= 1e-5 * max(1.0, np.max(np.abs(want)))


def test_adam_step_matches_oracle(model):
    import torch

    from threadcoarsenedstencilgenerator_b200.autotune import init_params

    p = init_params(9, 128, 6)
    model.set_params(p)
    x, t = _data(256, 9, 3)
    xd, td = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    pp, m, v = p.astype(np.float64), np.zeros(p.size), np.zeros(p.size)
    g = torch.empty(model.n_params, device="cuda")
    for step in (1, 2):
        # the update itself, fed with the kernels' own gradient (checked against the oracle above)
        model.gradient_raw(xd, td, g)
        model.adam_step_raw(xd, td, 1e-3)
        pp, m, v = M.adam(pp, g.cpu().numpy().astype(np.float64), m, v, step, 1e-3)
        assert np.max(np.abs(model.params() - pp)) <= 1e-6


def test_training_lowers_the_loss(model):
    from threadcoarsenedstencilgenerator_b200.autotune import init_params

    model.set_params(init_params(9, 128, 7))
    x, t = _data(4096, 9, 4)
    hist = model.fit(x, t, epochs=30, batch=512, lr=3e-3)
    assert hist[-1] < 0.1 * hist[0]
    pred = model.predict(x)
    assert np.mean((pred - t) ** 2) < 0.1 * np.var(t)


def test_trained_model_gains_over_choosing_without_it():
    """On the held-out configurations of the committed corpus, the best of the model's top 3
    blocks comes closer to the exhaustive best than 3 random blocks or the first 3 of the sweep
    order (the same timing budget without the model)."""
    from threadcoarsenedstencilgenerator_b200.autotune import CORPUS_PATH, MODEL_PATH, CostModel, evaluate, \
        load_corpus, split

    if not (CORPUS_PATH.exists() and MODEL_PATH.exists()):
        pytest.skip("no corpus / trained model committed yet")
    cfg, X, y = load_corpus()
    hold, _ = split(cfg)
    m = CostModel.load()
    r = evaluate(m, cfg, X, y, hold)
    assert r["configs"] >= 10
    assert r["mean_ratio_to_best"] > r["random_k_mean_ratio"] + 0.05
    assert r["mean_ratio_to_best"] > r["first_k_mean_ratio"]
    assert r["mean_ratio_to_best"] >= 0.9
    assert r["timed_fraction"] < 0.1
    m.close()


def test_tuner_on_a_held_out_set():
    """The learned tuner on a held-out 2D parameter set of the corpus, at the corpus grid size:
    it times the model's top 5 (or falls back to the sweep with the reason recorded), and its
    block comes within reach of the exhaustive sweep's, which times every runnable candidate."""
    import torch

    from threadcoarsenedstencilgenerator_b200 import Stencil
    from threadcoarsenedstencilgenerator_b200.autotune import (CORPUS_PATH, MODEL_PATH, Autotuner, CostModel,
                                                               _alloc, corpus_grid, load_corpus, sample_configs,
                                                               split, time_block)

    if not (CORPUS_PATH.exists() and MODEL_PATH.exists()):
        pytest.skip("no corpus / trained model committed yet")
    cfg, _, _ = load_corpus()
    hold, _ = split(cfg)
    specs = sample_configs(400, 7)
    cid = next(c for c in hold if specs[c].dimension == 2)
    spec = specs[cid]
    geom = spec.geometry(*corpus_grid(spec))
    st = Stencil(spec)
    if spec.coefficients == "Variable":
        st.copy_mask(np.random.default_rng(cid).standard_normal(spec.stencil_size) / spec.stencil_size)
    x, y = _alloc(spec, geom, cid)
    m = CostModel.load()
    learned = Autotuner(m).tune(st, geom, x, y)
    full = Autotuner(None).tune(st, geom, x, y)
    assert full.fell_back and full.reason == "no model" and full.timed == len(full.measured) >= 5
    if learned.fell_back:  # outside the corpus's feature ranges, or the model disagreed with timings
        assert "outside" in learned.reason or learned.model_error > 0.25
    else:
        assert learned.timed == 5 and learned.model_error <= 0.25
        assert learned.block in learned.measured
    g_l = time_block(st, geom, x, y, learned.block, 6)
    g_f = time_block(st, geom, x, y, full.block, 6)
    assert g_l >= 0.7 * g_f
    assert st.device_status() == 0
    m.close()
    st.close()
    del x, y
    torch.cuda.empty_cache()
