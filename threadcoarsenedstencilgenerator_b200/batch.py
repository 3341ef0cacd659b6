"""`BatchedSweeps`: many grids of one parameter set swept by one persistent launch.

The reference sweeps one grid per launch (cuda/generateLaunchUpdateGrid.py:103-147); a solver
with many small independent grids then pays a launch, a ramp-up and a tail per grid.  Here the
pipelined kernel's persistent CTAs take equal shares of the concatenated (grid, tile, plane) work
of all grids, so one launch per sweep keeps every SM busy whatever the grid sizes, and a CUDA
graph of n sweeps replays them without host work.  Every grid's result is bit-identical to a
single-grid sweep of that grid (the per-point arithmetic is the same code).
"""

from __future__ import annotations

import ctypes

from . import _lib
from .spec import Geometry
from .stencil import Launch, Plan, Stencil, _ptr, _stream


class BatchedSweeps:
    """A batch of grids (each with buffers a and b) of ``stencil``'s parameter set.

    ``launch`` is the pipe launch shape shared by all grids: block (bx, by, 1), chunk and depth
    (0 = the planner's defaults) and ``segments`` = CTA count (0 = every SM at full occupancy).
    The buffers must stay alive while the batch exists; ``close`` releases the device tables.
    """

    def __init__(self, stencil: Stencil, geoms: list[Geometry], a: list, b: list,
                 launch: Launch | None = None):
        if not (len(geoms) == len(a) == len(b)) or not geoms:
            raise ValueError("need one (geometry, a, b) triple per grid")
        self.stencil = stencil
        self.geoms = list(geoms)
        self.a = list(a)
        self.b = list(b)
        self.launch = launch or Launch(block=(32, 4, 1), variant="pipe")
        self._lib = _lib.load()
        self._graph_n = 0
        n = len(geoms)
        dims = (ctypes.c_uint * (3 * n))(*[int(v) for g in geoms for v in tuple(g.grid) + (1,) * (3 - len(g.grid))])
        ro = (ctypes.c_uint * n)(*[int(g.right_offset) for g in geoms])
        pa = (ctypes.c_void_p * n)(*[_ptr(x) for x in a])
        pb = (ctypes.c_void_p * n)(*[_ptr(x) for x in b])
        h = ctypes.c_void_p()
        _lib.check(self._lib.tcs_batch_create(stencil._h, n, dims, ro, ctypes.byref(self.launch.to_c()), pa, pb,
                                              ctypes.byref(h)))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.tcs_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def plan(self) -> Plan:
        p = _lib.CPlan()
        _lib.check(self._lib.tcs_batch_plan(self._h, ctypes.byref(p)))
        return Plan("pipe", tuple(p.grid_blocks), tuple(p.block), p.dyn_smem, p.seg_len, p.nslot, p.width,
                    p.chunk, p.depth, "tma" if p.loader == 0 else "mixed", p.ctas_per_sm, p.num_sms)

    def sweep(self, from_b: bool = False, stream=None) -> None:
        """One sweep of every grid (a -> b, or b -> a with from_b): one launch."""
        _lib.check(self._lib.tcs_batch_sweep(self._h, int(bool(from_b)), _stream(stream)))

    def sweep_separate(self, from_b: bool = False, stream=None) -> None:
        """The same sweep as one single-grid launch per grid."""
        _lib.check(self._lib.tcs_batch_sweep_separate(self._h, int(bool(from_b)), _stream(stream)))

    def sweeps(self, n: int, stream=None, separate: bool = False) -> list:
        """n ping-pong sweeps starting from the a buffers; returns the list holding the result."""
        for i in range(int(n)):
            (self.sweep_separate if separate else self.sweep)(from_b=bool(i & 1), stream=stream)
        return self.b if n % 2 == 1 else self.a

    def capture(self, n: int, separate: bool = False) -> None:
        """Capture n ping-pong sweeps starting from a into a CUDA graph held by the batch."""
        _lib.check(self._lib.tcs_batch_graph(self._h, int(n), int(bool(separate))))
        self._graph_n = int(n)

    def replay(self, stream=None) -> list:
        """Launch the captured graph; returns the list holding the result."""
        _lib.check(self._lib.tcs_batch_graph_launch(self._h, _stream(stream)))
        return self.b if self._graph_n % 2 == 1 else self.a


def precompile_batch(spec, block, chunk: int) -> str:
    """Instantiate the batched sweep of ``spec`` for one launch shape into the cubin cache."""
    buf = ctypes.create_string_buffer(1024)
    b = tuple(block) + (1,) * (3 - len(block))
    _lib.check(_lib.load().tcs_precompile_batch(ctypes.byref(spec.to_c()), b[0], b[1], int(chunk), buf, 1024))
    return buf.value.decode()
