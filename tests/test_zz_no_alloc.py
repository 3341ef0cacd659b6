"""tcs_residual_static: the allocation-free residual, checked against tcs_residual.

Some callers of the residual norm cannot allocate device memory where they need it: code whose
device memory belongs to another allocator (a framework's caching allocator), solver loops that
cannot afford the implicit device synchronisation of cudaMalloc/cudaFree, processes held to a fixed
memory budget.  tcs_residual_static serves them: its per-block partial sums live in a static device
array of libtcs.so instead of library-allocated scratch.

Both entry points are called through the C ABI on the same inputs, twice in a row with different
data (the static array keeps the previous call's contents).  The defect fields must be identical
and the norms equal within the 1e-12 relative tolerance of the other norm tests (the reductions
run in the same order, so they agree exactly).  The file is collected last so that a run stopping
at its first failure has run everything else; it also passes alone in a fresh process.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _call_residual(lib, fn, h, geom, x, sx, r, extra=()):
    from threadcoarsenedstencilgenerator_b200 import _lib

    norms = (ctypes.c_double * 2)()
    args = [h, _lib.U3(*geom.grid), geom.right_offset, x.data_ptr(), sx.data_ptr(), r.data_ptr(), norms]
    rc = getattr(lib, fn)(*args, *extra, None)
    return rc, (norms[0], norms[1])


def test_static_scratch_residual_matches_allocating_entry_point():
    import torch

    import threadcoarsenedstencilgenerator_b200 as tcs
    from threadcoarsenedstencilgenerator_b200 import _lib

    lib = _lib.load()
    spec = tcs.StencilSpec(dimension=3, neighbourhood="Star", orientation="Row", coefficients="Variable", range=4,
                           cx=2, cy=2, alignment="Read", cl_size=16)
    st = tcs.Stencil(spec)
    geom = spec.geometry(96, 80, 72)
    rng = np.random.default_rng(77)
    for trial in range(2):
        x = torch.from_numpy(rng.random(geom.shape)).cuda()
        sx = x + torch.from_numpy(1e-3 * rng.standard_normal(geom.shape) * (trial + 1)).cuda()
        r_alloc = torch.zeros(geom.shape, dtype=torch.float32, device="cuda")
        r_static = torch.full(geom.shape, 0.0, dtype=torch.float32, device="cuda")
        rc, n_alloc = _call_residual(lib, "tcs_residual", st._h, geom, x, sx, r_alloc)
        assert rc == 0, _lib.last_error()
        rc, n_static = _call_residual(lib, "tcs_residual_static", st._h, geom, x, sx, r_static, (0,))
        assert rc == 0, _lib.last_error()
        assert torch.equal(r_alloc, r_static)
        assert n_static[0] == n_alloc[0]
        assert abs(n_static[1] - n_alloc[1]) <= 1e-12 * n_alloc[1]
        sl = geom.interior_slices(spec.range)
        d = (sx - x).cpu().numpy()[sl]
        assert n_static[0] == np.abs(d).max()


def _scratch_bytes(lib, h) -> int:
    v = ctypes.c_ulonglong(123)
    assert lib.tcs_scratch_bytes(h, ctypes.byref(v)) == 0
    return v.value


def test_static_scratch_residual_allocates_nothing_and_enforces_its_limit():
    """Free device memory is unchanged across the calls, and the handle's library scratch (which
    tcs_residual allocates on first use) stays unallocated: a cudaMalloc undone by a cudaFree, or an
    allocation below the driver's 2 MiB granularity, would escape the first check, not the second."""
    import torch

    import threadcoarsenedstencilgenerator_b200 as tcs
    from threadcoarsenedstencilgenerator_b200 import _lib

    lib = _lib.load()
    spec = tcs.StencilSpec(dimension=2, neighbourhood="Box", coefficients="Variable", range=6, cx=4)
    st = tcs.Stencil(spec)
    assert _scratch_bytes(lib, st._h) == 0
    geom = spec.geometry(1024, 512)
    x = torch.rand(geom.shape, dtype=torch.float64, device="cuda")
    sx = x * 0.5
    r = torch.zeros(geom.shape, dtype=torch.float32, device="cuda")
    rc, first = _call_residual(lib, "tcs_residual_static", st._h, geom, x, sx, r, (64,))
    assert rc == 0, _lib.last_error()
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for nblocks in (0, 1, 2047):
        rc, norms = _call_residual(lib, "tcs_residual_static", st._h, geom, x, sx, r, (nblocks,))
        assert rc == 0, _lib.last_error()
        assert norms[0] == first[0] and abs(norms[1] - first[1]) <= 1e-12 * first[1]
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
    assert _scratch_bytes(lib, st._h) == 0
    rc, _ = _call_residual(lib, "tcs_residual_static", st._h, geom, x, sx, r, (2048,))
    assert rc == _lib.TCS_ERR_INVALID_VALUE
    assert "4096" in _lib.last_error()
    # the allocating entry point does allocate, through the same handle
    rc, _ = _call_residual(lib, "tcs_residual", st._h, geom, x, sx, r)
    assert rc == 0, _lib.last_error()
    assert _scratch_bytes(lib, st._h) > 0
