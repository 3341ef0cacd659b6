"""Failure detection on the GPU without a fault: a bounded device wait that nothing satisfies
gives up after its budget, the host reads the timeout from the device status word, and the
context stays usable (the next sweep still equals the oracle)."""

import numpy as np
import pytest

import gpu_util as G
import oracle as O

pytestmark = pytest.mark.gpu


def test_expired_wait_is_reported_and_the_context_stays_usable():
    import torch

    import threadcoarsenedstencilgenerator_b200 as tcs

    cfg = (2, "Box", "Row", "Variable", 2, 2, 2, 1, "None", 0)
    st = tcs.Stencil(G.spec_of(cfg))
    assert st.device_status() == 0
    assert st.self_test_wait(2_000_000) is True      # about a millisecond, then the timeout bit
    assert st.device_status() == 0                   # read and cleared by the self-test
    with pytest.raises(tcs.CudaErrorInvalidValue):
        st.self_test_wait(10)                        # budget below the accepted range
    geom = st.spec.geometry(130, 70)
    rng = np.random.default_rng(2)
    a = rng.random(geom.shape)
    mask = rng.standard_normal(st.spec.stencil_size)
    st.copy_mask(mask)
    x = torch.from_numpy(a).cuda()
    y = x.clone()
    res = st.sweeps(geom, x, y, 2, tcs.Launch(block=(32, 1, 1), variant="pipe"))
    torch.cuda.synchronize()
    assert st.device_status() == 0
    assert np.array_equal(res.cpu().numpy(), O.sweeps(O.make_spec(*cfg), a, 2, geom.right_offset, mask))
