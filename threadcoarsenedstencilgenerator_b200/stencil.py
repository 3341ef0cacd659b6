"""`Stencil`: one instantiated parameter set on the current CUDA device.

The object is the engine-side counterpart of one generated ``kernels.cu`` +
``launchUpdateGrid.cu`` pair of the reference (cuda/RunBenchmark.sh:118-129): creating it
instantiates the sm_100a kernels for the spec (NVRTC, cubin cache) and loads them.  Device
buffers are any objects exposing ``data_ptr()`` (torch tensors) or raw integer addresses; torch is
used only to own device memory and streams.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

from . import _lib
from .spec import Geometry, StencilSpec


def _ptr(buf) -> int:
    if isinstance(buf, int):
        return buf
    if hasattr(buf, "data_ptr"):
        return int(buf.data_ptr())
    raise TypeError("expected a device tensor or an integer device address, got %r" % type(buf))


def _stream(stream) -> int | None:
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return int(stream.cuda_stream)


@dataclass
class Launch:
    """Launch parameters of a sweep (see tcs_launch in include/tcs.h)."""

    block: tuple = (128, 1, 1)
    variant: str = "auto"          # auto | direct | march | pipe
    grid_blocks: tuple = (0, 0, 0)  # direct only; zeros: cover the interior
    segments: int = 0               # march: CTAs along the march axis per tile column (0 = auto)
    depth: int = 0                  # march/pipe: chunks in flight (0 = auto)
    chunk: int = 0                  # pipe: planes per ring chunk (0 = auto)
    shuffle: bool | None = None     # pipe, Star: middle rows through warp shuffles (None: planner's choice)
    tmem: bool = False              # pipe, 3D Star Row: the ring form in tensor memory
    lockstep: bool = False          # pipe: one tile column (or an equal part) per persistent CTA

    _VARIANTS = {"auto": _lib.VARIANT_AUTO, "direct": _lib.VARIANT_DIRECT, "march": _lib.VARIANT_MARCH,
                 "pipe": _lib.VARIANT_PIPE}

    def to_c(self) -> _lib.CLaunch:
        b = tuple(self.block) + (1,) * (3 - len(self.block))
        g = tuple(self.grid_blocks) + (0,) * (3 - len(self.grid_blocks))
        flags = 0 if self.shuffle is None else (_lib.LAUNCH_SHUFFLE if self.shuffle else _lib.LAUNCH_NO_SHUFFLE)
        if self.tmem:
            flags |= _lib.LAUNCH_TMEM
        if self.lockstep:
            flags |= _lib.LAUNCH_LOCKSTEP
        return _lib.CLaunch(_lib.U3(*b), _lib.U3(*g), self._VARIANTS[self.variant], int(self.segments),
                            int(self.depth), int(self.chunk), flags)


@dataclass
class Plan:
    variant: str
    grid_blocks: tuple
    block: tuple
    dyn_smem: int
    seg_len: int
    nslot: int
    width: int
    chunk: int
    depth: int
    loader: str
    ctas_per_sm: int
    num_sms: int


class Stencil:
    """Kernels of one StencilSpec, loaded on the current device."""

    def __init__(self, spec: StencilSpec):
        self.spec = spec
        self._lib = _lib.load()
        h = ctypes.c_void_p()
        _lib.check(self._lib.tcs_create(ctypes.byref(spec.to_c()), ctypes.byref(h)))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.tcs_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- reference helper functions (cuda/launchUpdateGrid.h:16-18) -----------------------------
    def copy_mask(self, mask) -> None:
        vals = [float(v) for v in mask]
        arr = (ctypes.c_double * len(vals))(*vals)
        _lib.check(self._lib.tcs_copy_mask(self._h, arr, len(vals)))

    def max_potential_block_size(self) -> int:
        v = ctypes.c_int()
        _lib.check(self._lib.tcs_max_potential_block_size(self._h, ctypes.byref(v)))
        return v.value

    # -- sweeps ---------------------------------------------------------------------------------
    def geometry(self, nx: int, ny: int, nz: int = 1) -> Geometry:
        return self.spec.geometry(nx, ny, nz)

    def plan(self, geom: Geometry, launch: Launch) -> Plan:
        p = _lib.CPlan()
        _lib.check(self._lib.tcs_plan_launch(self._h, _lib.U3(*geom.grid), geom.right_offset,
                                             ctypes.byref(launch.to_c()), ctypes.byref(p)))
        names = {v: k for k, v in Launch._VARIANTS.items()}
        return Plan(names[p.variant], tuple(p.grid_blocks), tuple(p.block), p.dyn_smem, p.seg_len, p.nslot,
                    p.width, p.chunk, p.depth, {0: "tma", 2: "cp.async pairs"}.get(p.loader, "cp.async"), p.ctas_per_sm, p.num_sms)

    def update_grid(self, geom: Geometry, src, dst, launch: Launch | None = None, stream=None) -> None:
        """One sweep dst = stencil(src) over the interior (asynchronous)."""
        launch = launch or Launch()
        _lib.check(self._lib.tcs_update_grid(self._h, _lib.U3(*geom.grid), geom.right_offset,
                                             ctypes.byref(launch.to_c()), _ptr(src), _ptr(dst), _stream(stream)))

    def sweeps(self, geom: Geometry, a, b, n: int, launch: Launch | None = None, stream=None):
        """n ping-pong sweeps starting from a; returns the buffer holding the result."""
        launch = launch or Launch()
        in_b = ctypes.c_int()
        _lib.check(self._lib.tcs_sweeps(self._h, _lib.U3(*geom.grid), geom.right_offset,
                                        ctypes.byref(launch.to_c()), _ptr(a), _ptr(b), int(n), _stream(stream),
                                        ctypes.byref(in_b)))
        return b if in_b.value else a

    def time_sweeps(self, geom: Geometry, a, b, n: int, launch: Launch | None = None, stream=None) -> float:
        """n ping-pong sweeps timed with CUDA events; returns milliseconds."""
        launch = launch or Launch()
        ms = ctypes.c_float()
        _lib.check(self._lib.tcs_time_sweeps(self._h, _lib.U3(*geom.grid), geom.right_offset,
                                             ctypes.byref(launch.to_c()), _ptr(a), _ptr(b), int(n),
                                             _stream(stream), ctypes.byref(ms)))
        return ms.value

    def sweep_host_jobs(self, geom: Geometry, host_in: list, host_out: list, n: int, launch: Launch | None = None,
                        slots: int = 3, dev: list | None = None) -> float:
        """Sweep host-resident grids: job j uploads host_in[j], runs n ping-pong sweeps and
        downloads the result into host_out[j].  Jobs rotate over ``slots`` pairs of device
        buffers, one stream each, so the upload, the sweeps and the download of different jobs
        overlap (pin the host tensors for that).  ``dev`` optionally gives the slots as (a, b)
        device tensor pairs; they are allocated here otherwise.  Returns once every result is
        on the host; each equals the same sweeps run alone, bit for bit.  Returns the device time
        in milliseconds from the first upload's start to the last download's end."""
        import torch

        launch = launch or Launch()
        if len(host_in) != len(host_out):
            raise ValueError("need one host output per host input")
        shape = tuple(geom.shape)
        dtype = torch.float64 if self.spec.precision == "f64" else torch.float32
        for t in list(host_in) + list(host_out):
            if t.device.type != "cpu" or tuple(t.shape) != shape or t.dtype != dtype or not t.is_contiguous():
                raise ValueError("host grids must be contiguous CPU tensors of shape %s and %s" % (shape, dtype))
        nj = len(host_in)
        ns = len(dev) if dev is not None else max(1, min(int(slots), nj))
        ms = ctypes.c_float()
        outs = [int(t.data_ptr()) for t in host_out]
        first = {}
        for j, o in enumerate(outs):  # a host output may repeat only within one slot's jobs
            if first.setdefault(o, j) % ns != j % ns:
                raise ValueError("host outputs of jobs on different slots must be distinct")
        if set(outs) & {int(t.data_ptr()) for t in host_in}:
            raise ValueError("host outputs must be distinct from the inputs")
        if dev is None:
            dev = [(torch.empty(shape, dtype=dtype, device="cuda"), torch.empty(shape, dtype=dtype, device="cuda"))
                   for _ in range(ns)]
        arr = ctypes.c_void_p * max(1, nj)
        sarr = ctypes.c_void_p * max(1, ns)
        _lib.check(self._lib.tcs_sweep_host_jobs(
            self._h, _lib.U3(*geom.grid), geom.right_offset, ctypes.byref(launch.to_c()),
            arr(*[int(t.data_ptr()) for t in host_in]), arr(*outs), nj, int(n),
            sarr(*[_ptr(a) for a, _ in dev]), sarr(*[_ptr(b) for _, b in dev]), ns, ctypes.byref(ms)))
        return ms.value

    def update_grid_source(self, geom: Geometry, src, source, dst, launch: Launch | None = None,
                           stream=None) -> None:
        """One sweep dst = stencil(src) + source (asynchronous)."""
        launch = launch or Launch()
        _lib.check(self._lib.tcs_update_grid_source(self._h, _lib.U3(*geom.grid), geom.right_offset,
                                                    ctypes.byref(launch.to_c()), _ptr(src), _ptr(source),
                                                    _ptr(dst), _stream(stream)))

    def defect_sweep(self, geom: Geometry, x, r, launch: Launch | None = None, stream=None, norms: bool = True):
        """One FP64 sweep of x whose epilogue writes r = fl32(S(x) - x) (S(x) is not stored);
        returns (max |S(x) - x|, ||S(x) - x||_2) when norms.  Pipelined kernel only."""
        launch = launch or Launch()
        out = (ctypes.c_double * 2)()
        _lib.check(self._lib.tcs_defect_sweep(self._h, _lib.U3(*geom.grid), geom.right_offset,
                                              ctypes.byref(launch.to_c()), _ptr(x), _ptr(r), out if norms else None,
                                              _stream(stream)))
        return (out[0], out[1]) if norms else None

    def update_grid_accumulate(self, geom: Geometry, src, source, x, launch: Launch | None = None,
                               stream=None) -> None:
        """One FP32 sweep added to the FP64 state: x += S(src) + source (source may be None)."""
        launch = launch or Launch()
        _lib.check(self._lib.tcs_update_grid_accumulate(self._h, _lib.U3(*geom.grid), geom.right_offset,
                                                        ctypes.byref(launch.to_c()), _ptr(src),
                                                        None if source is None else _ptr(source), _ptr(x),
                                                        _stream(stream)))

    def sweeps_tb2(self, geom: Geometry, a, b, n: int, stream=None):
        """n ping-pong sweeps starting from a with temporal blocking (2D: two sweeps per pass over
        HBM, bit-identical to n ordinary sweeps); returns the buffer holding the result."""
        in_b = ctypes.c_int()
        _lib.check(self._lib.tcs_sweeps_tb2(self._h, _lib.U3(*geom.grid), geom.right_offset, _ptr(a), _ptr(b),
                                            int(n), _stream(stream), ctypes.byref(in_b)))
        return b if in_b.value else a

    def sweeps_tb3(self, geom: Geometry, a, b, n: int, launch: Launch | None = None, stream=None):
        """n ping-pong sweeps starting from a, two per pass over HBM (3D temporal blocking,
        bit-identical to n ordinary sweeps); returns the buffer holding the result.  ``launch``
        optionally sets the kernel's block, ring chunk and depth."""
        in_b = ctypes.c_int()
        _lib.check(self._lib.tcs_sweeps_tb3(self._h, _lib.U3(*geom.grid), geom.right_offset,
                                            None if launch is None else ctypes.byref(launch.to_c()), _ptr(a),
                                            _ptr(b), int(n), _stream(stream), ctypes.byref(in_b)))
        return b if in_b.value else a

    def plan_tb3(self, geom: Geometry, launch: Launch | None = None) -> Plan:
        """The launch of the two-sweep kernel for this grid."""
        p = _lib.CPlan()
        _lib.check(self._lib.tcs_plan_tb3(self._h, _lib.U3(*geom.grid), geom.right_offset,
                                          None if launch is None else ctypes.byref(launch.to_c()), ctypes.byref(p)))
        return Plan("tb3", tuple(p.grid_blocks), tuple(p.block), p.dyn_smem, p.seg_len, p.nslot, p.width, p.chunk,
                    p.depth, {0: "tma"}.get(p.loader, "cp.async"), p.ctas_per_sm, p.num_sms)

    def tc_update_grid(self, geom: Geometry, src, dst, source=None, stream=None) -> None:
        """One FP32 sweep dst = stencil(src) (+ source) on the tensor cores (2D Box only; BF16
        hi/lo split, FP32 accumulation: a precision option, not the reference's bits)."""
        _lib.check(self._lib.tcs_tc_update_grid(self._h, _lib.U3(*geom.grid), geom.right_offset, _ptr(src),
                                                None if source is None else _ptr(source), _ptr(dst),
                                                _stream(stream)))

    def residual(self, geom: Geometry, x, sx, r, stream=None, norms: bool = True):
        """r = fl32(sx - x) on the interior; returns (max |sx - x|, ||sx - x||_2) when norms."""
        out = (ctypes.c_double * 2)()
        _lib.check(self._lib.tcs_residual(self._h, _lib.U3(*geom.grid), geom.right_offset, _ptr(x), _ptr(sx),
                                          _ptr(r), out if norms else None, _stream(stream)))
        return (out[0], out[1]) if norms else None

    def accumulate(self, geom: Geometry, x, e, stream=None) -> None:
        """x += e on the interior (x FP64, e FP32)."""
        _lib.check(self._lib.tcs_accumulate(self._h, _lib.U3(*geom.grid), geom.right_offset, _ptr(x), _ptr(e),
                                            _stream(stream)))

    def compare(self, geom: Geometry, a, b, a_precision: str = "f64", stream=None) -> dict:
        """Error statistics of a against the FP64 field b over the interior."""
        out = (ctypes.c_double * 4)()
        _lib.check(self._lib.tcs_compare(self._h, _lib.U3(*geom.grid), geom.right_offset, _ptr(a),
                                         0 if a_precision == "f64" else 1, _ptr(b), out, _stream(stream)))
        max_abs, l2, max_ref, l2_ref = out[0], out[1], out[2], out[3]
        return {"max_abs": max_abs, "l2": l2, "max_ref": max_ref, "l2_ref": l2_ref,
                "max_rel": max_abs / max_ref if max_ref else 0.0, "rms_rel": l2 / l2_ref if l2_ref else 0.0}

    def device_status(self, clear: bool = True) -> int:
        v = ctypes.c_uint()
        _lib.check(self._lib.tcs_device_status(self._h, ctypes.byref(v), 1 if clear else 0))
        return v.value

    def self_test_wait(self, cycles: int = 2_000_000) -> bool:
        """Failure-detection self-test: a bounded device wait on a barrier nothing arrives at.
        True when the kernel gave up after ``cycles`` and the host read the timeout from the
        device status word (the expected outcome; the word is cleared and the context usable)."""
        rc = self._lib.tcs_self_test_wait(self._h, int(cycles))
        if rc == _lib.TCS_ERR_DEVICE_TIMEOUT:
            return True
        _lib.check(rc)
        return False

    def set_dropin_launch(self, variant: str = "auto", segments: int = 0, depth: int = 0) -> None:
        _lib.check(self._lib.tcs_set_dropin_launch(self._h, Launch._VARIANTS[variant], segments, depth))

    # -- reference host interface (cuda/launchUpdateGrid.h:13-14) -------------------------------
    def benchmark_update_grid(self, coeff_type: str, neighbourhood: str, stencil_range: int, dimension: int,
                              alignment: str, max_time: float, grid_size, block_size, grid_blocks, d_array0,
                              d_array1, right_offset: int) -> list:
        """Every per-launch duration [s] of the doubling loop (2^k - 1 of them)."""
        n = ctypes.c_uint()
        _lib.check(self._lib.tcs_benchmark_update_grid(
            self._h, coeff_type.encode(), neighbourhood.encode(), int(stencil_range), int(dimension),
            alignment.encode(), float(max_time), _lib.U3(*_dim3(grid_size)), _lib.U3(*_dim3(block_size)),
            _lib.U3(*_dim3(grid_blocks)), _ptr(d_array0), _ptr(d_array1), int(right_offset), None, 0,
            ctypes.byref(n)))
        dur = (ctypes.c_double * max(1, n.value))()
        got = ctypes.c_uint()
        _lib.check(self._lib.tcs_benchmark_durations(self._h, dur, n.value, ctypes.byref(got)))
        return list(dur[: got.value])

    def launch_init(self, grid_size, block_size, grid_blocks, d_array, right_offset: int) -> None:
        _lib.check(self._lib.tcs_launch_init(self._h, _lib.U3(*_dim3(grid_size)), _lib.U3(*_dim3(block_size)),
                                             _lib.U3(*_dim3(grid_blocks)), _ptr(d_array), int(right_offset)))


def _dim3(v) -> tuple:
    v = tuple(int(x) for x in v)
    return v + (1,) * (3 - len(v))


def precompile(spec: StencilSpec) -> str:
    """Instantiate the kernels of ``spec`` into the cubin cache (NVRTC only, no GPU needed)."""
    buf = ctypes.create_string_buffer(1024)
    _lib.check(_lib.load().tcs_precompile(ctypes.byref(spec.to_c()), buf, 1024))
    return buf.value.decode()


def precompile_pipe(spec: StencilSpec, block, chunk: int, shuffle: bool = False, tmem: bool = False) -> str:
    """Instantiate the pipelined sweep of ``spec`` for one launch shape into the cubin cache."""
    buf = ctypes.create_string_buffer(1024)
    b = tuple(block) + (1,) * (3 - len(block))
    if shuffle or tmem:
        flags = (_lib.LAUNCH_SHUFFLE if shuffle else 0) | (_lib.LAUNCH_TMEM if tmem else 0)
        _lib.check(_lib.load().tcs_precompile_pipe_flags(ctypes.byref(spec.to_c()), b[0], b[1], int(chunk),
                                                         flags, buf, 1024))
    else:
        _lib.check(_lib.load().tcs_precompile_pipe(ctypes.byref(spec.to_c()), b[0], b[1], int(chunk), buf, 1024))
    return buf.value.decode()


def precompile_pipe_epilogue(spec: StencilSpec, block, chunk: int, epi: int) -> str:
    """Instantiate the pipelined sweep with epilogue 1 (FP64 defect) or 2 (FP32 accumulate)."""
    buf = ctypes.create_string_buffer(1024)
    b = tuple(block) + (1,) * (3 - len(block))
    _lib.check(_lib.load().tcs_precompile_pipe_epilogue(ctypes.byref(spec.to_c()), b[0], b[1], int(chunk), int(epi),
                                                        buf, 1024))
    return buf.value.decode()


def precompile_tb3(spec: StencilSpec, block=(0, 0), chunk: int = 0) -> str:
    """Instantiate the 3D two-sweep kernel of ``spec`` into the cubin cache."""
    buf = ctypes.create_string_buffer(1024)
    _lib.check(_lib.load().tcs_precompile_tb3(ctypes.byref(spec.to_c()), int(block[0]), int(block[1]), int(chunk),
                                              buf, 1024))
    return buf.value.decode()


def precompile_fringe(spec: StencilSpec) -> str:
    """Instantiate the coarsening-1 instance of ``spec`` (ragged fringe) and, in 2D, the 1 x 8
    temporal-blocking instance."""
    buf = ctypes.create_string_buffer(1024)
    _lib.check(_lib.load().tcs_precompile_fringe(ctypes.byref(spec.to_c()), buf, 1024))
    return buf.value.decode()


def device_sm_count() -> int:
    v = ctypes.c_int()
    _lib.check(_lib.load().tcs_device_sm_count(ctypes.byref(v)))
    return v.value
