"""The learned pipelined-launch tuner on the GPU, on a problem its model never trained on.

The committed model (data/pipe_costmodel.npz) ranks the launch shapes of a held-out 3D Star Jacobi
r3 FP64 problem; the tuner times its top 5 shapes in each of their forms (register pipeline or
ring form in tensor memory, even split or lockstep), and the exhaustive search times every shape in
every form.  The learned choice must not fall back to the exhaustive search and must reach 90% of
the exhaustive choice's rate (both re-timed with 10 sweeps), having timed at most 5 shapes.
"""

import pytest

pytestmark = pytest.mark.gpu


def test_learned_choice_on_a_held_out_problem():
    import torch

    from threadcoarsenedstencilgenerator_b200 import pipetune as P
    from threadcoarsenedstencilgenerator_b200.autotune import CostModel

    assert torch.cuda.is_available()
    m = CostModel.load(P.PIPE_MODEL_PATH, P.PIPE_FEATURES)
    pid = P.live_check_problem(40)
    assert pid in P.holdout_ids(40)
    out = P.live(m, [pid], 40, log=lambda *_: None)
    row = out["rows"][0]
    m.close()
    assert not row["fell_back"], row["reason"]
    assert row["timed"] <= 5 * len(P.FORMS)
    assert row["ratio"] >= 0.9, row
