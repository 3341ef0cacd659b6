"""Learned tuner of the pipelined sweep's launch: thread coarsening, block and planes per ring chunk.

The reference tunes one thing, the thread-block shape of one generated kernel, by timing every
shape (cuda/benchmark.cpp:223-251, 287-318); the coarsening is fixed when the generator runs, so
choosing it means generating, compiling and sweeping one kernel per coarsening.  The engine's
pipelined kernel (tcs_pipe) has the same two choices and a third, the planes per ring chunk, and
every (coarsening, block, chunk) is a separate NVRTC instantiation: an exhaustive search pays a
compilation and a timing per candidate.

``PipeTuner`` ranks every candidate of the space with a cost model -- the 3-layer perceptron of
autotune.py, trained by the library's own kernels on timings of this space -- from features that
need no compilation (stencil, precision, coarsening, block, tile and halo sizes, register and
shared-memory estimates, loads per update), then compiles and times only the top k.  It falls back
to the exhaustive search when the model is missing, the problem lies outside the corpus's feature
ranges, or the timed candidates disagree with the predicted ordering by more than a tolerance.

    python -m threadcoarsenedstencilgenerator_b200.pipetune precompile|corpus|train|evaluate|tune

``tune --workload NAME [--precision f32] --exhaustive --write`` records the chosen launch in the
package's tuned.json, the file the benchmark workloads read their launches from.  For the batched
workload (many grids, one launch per sweep) ``tune`` searches the batched kernel's block and planes
per chunk exhaustively.
"""

from __future__ import annotations

import argparse
import json
import math
import sys
import time
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import _lib
from .autotune import CostModel
from .spec import Geometry, StencilSpec
from .stencil import Launch, Stencil

DATA = Path(__file__).resolve().parent / "data"
PIPE_CORPUS_PATH = DATA / "pipe_corpus.npz"
PIPE_MODEL_PATH = DATA / "pipe_costmodel.npz"
TUNED_PATH = Path(__file__).resolve().parent / "tuned.json"
GRID_BYTES = 256 << 20  # one buffer of a corpus grid (two buffers: ~0.5 GB)

PIPE_FEATURES = [
    "dim2", "dim3", "box", "star", "jacobi", "variable", "f64", "f32",
    "range", "log_S", "log_cx", "log_cy", "log_nep", "log_terms",
    "log_bx", "log_by", "log_threads", "log_tile_x", "log_tile_y", "chunk",
    "log_regs_est", "log_warps_est", "log_smem_est", "halo_ratio", "loads_per_lup", "tile_efficiency",
    "log_nx", "log_ny", "log_nz",
]


def _l2(v) -> float:
    return math.log2(max(1.0, float(v)))


def candidates(base: StencilSpec) -> list:
    """(cx, cy, bx, by, chunk) of the pipelined kernel for a problem: coarsening 1/2/4 per tiled axis
    (1..8 in x for 2D), blocks of 32..128 x 1..16 threads (heights 1, 2, 4, 6, 7, 8, 16) with
    64..1024 in all (2D: 16..128 x 1),
    tile rows that fit a 256-element TMA box and a 16-byte granule, 2 or 3 planes per chunk (1 or 2
    in 2D), and at most ~200 registers of accumulators per thread."""
    R, es = base.range, base.itemsize
    vec = 16 // es
    out = []
    if base.dimension == 2:
        if base.orientation == "Column":
            return []
        for cx in (1, 2, 4, 8):
            for bx in (16, 32, 64, 128):
                tx = bx * cx
                if tx % vec or tx + 2 * R + vec > 256:
                    continue
                if (2 * R + 1) * cx * es // 4 > 200:
                    continue
                for ch in (1, 2):
                    out.append((cx, 1, bx, 1, ch))
        return out
    for cx in (1, 2, 4):
        for cy in (1, 2, 4):
            nep = cx * cy
            if (2 * R + 1) * nep * es // 4 > 200:
                continue
            for bx in (32, 64, 128):
                tx = bx * cx
                if tx % vec or tx + 2 * R + vec > 256:
                    continue
                for by in (1, 2, 4, 6, 7, 8, 16):
                    if not 64 <= bx * by <= 1024 or by * cy + 2 * R > 256:
                        continue
                    for ch in (2, 3):
                        out.append((cx, cy, bx, by, ch))
    return out


def problem_spec(base: StencilSpec, cand) -> StencilSpec:
    cx, cy = cand[0], cand[1]
    return base.replace(cx=cx, cy=cy, cz=1) if base.dimension == 3 else base.replace(cx=cx, cy=1)


def features(base: StencilSpec, grid, cand) -> np.ndarray:
    """Analytic features of a candidate (order: PIPE_FEATURES): nothing is compiled."""
    cx, cy, bx, by, ch = cand
    d3 = base.dimension == 3
    R, es = base.range, base.itemsize
    S = base.stencil_size
    nep = cx * (cy if d3 else 1)
    threads = bx * (by if d3 else 1)
    tx, ty = bx * cx, (by * cy if d3 else 1)
    rows = ty + 2 * R if d3 else 1
    w = tx + 2 * R + 16 // es
    regs = (2 * R + 1) * nep * es / 4 + 40
    smem = 2 * ch * rows * w * es
    occ = max(1, min(2048 // threads, 65536 // max(1, int(threads * min(255, regs))), (228 << 10) // max(1, smem)))
    halo = ((tx + 2 * R) * (ty + 2 * R)) / float(tx * ty) if d3 else (tx + 2 * R) / float(tx)
    if base.neighbourhood == "Box":
        loads = ((2 * R + cx) * ((2 * R + cy) if d3 else 1)) / float(nep)
    else:
        loads = (nep + 2 * R * (cx + (cy if d3 else 0))) / float(nep) if d3 else (cx + 2 * R) / float(cx)
    nx, ny, nz = grid[0], grid[1], grid[2] if d3 else 1
    ex, ey = nx - 2 * R, ny - 2 * R
    eff = (ex / (math.ceil(ex / tx) * tx)) * ((ey / (math.ceil(ey / ty) * ty)) if d3 else 1.0)
    return np.array([
        not d3, d3, base.neighbourhood == "Box", base.neighbourhood == "Star",
        base.coefficients == "Jacobi", base.coefficients == "Variable",
        base.precision == "f64", base.precision == "f32",
        R, _l2(S), _l2(cx), _l2(cy if d3 else 1), _l2(nep), _l2(S * nep),
        _l2(bx), _l2(by if d3 else 1), _l2(threads), _l2(tx), _l2(ty), ch,
        _l2(regs), _l2(occ * threads / 32.0), _l2(smem), halo, loads, eff,
        _l2(nx), _l2(ny), _l2(nz),
    ], dtype=np.float32)


def corpus_grid(base: StencilSpec) -> tuple:
    pts = GRID_BYTES // base.itemsize
    if base.dimension == 2:
        s = int(math.sqrt(pts))
        return (s, s, 1)
    s = int(round(pts ** (1.0 / 3.0)))
    return (s, s, s)


def sample_problems(n: int, seed: int = 13) -> list:
    """Seeded problems of the pipelined kernel: dim 2/3, Box/Star, range 1-6, Jacobi/Variable,
    FP64/FP32, Row order, no alignment (coarsening 1: the tuner chooses it)."""
    rng = np.random.default_rng(seed)
    out, seen = [], set()
    while len(out) < n:
        d = int(rng.choice([2, 3], p=[0.35, 0.65]))
        sh = str(rng.choice(["Box", "Star"]))
        r = int(rng.integers(1, 7 if sh == "Star" or d == 2 else 4))
        spec = StencilSpec(dimension=d, neighbourhood=sh, orientation="Row",
                           coefficients=str(rng.choice(["Jacobi", "Variable"])), range=r,
                           precision=str(rng.choice(["f64", "f32"])))
        if repr(spec) in seen:
            continue
        seen.add(repr(spec))
        out.append(spec)
    return out


def subset(cands: list, k: int, rng) -> list:
    if len(cands) <= k:
        return list(cands)
    idx = rng.choice(len(cands), size=k, replace=False)
    return [cands[i] for i in sorted(idx)]


# ---- launch forms ---------------------------------------------------------------------------------
# Each shape runs in up to four forms (tmem, lockstep): the register pipeline or the ring form in
# tensor memory (3D Star stencils in Row order), and the persistent CTAs splitting the work list
# evenly or taking whole tile columns in step (TCS_LAUNCH_LOCKSTEP).  The form changes no feature
# of the model, which ranks shapes; the tuner times every form of the shapes it times.
FORMS = ((0, 0), (0, 1), (1, 0), (1, 1))


def tmem_applies(base: StencilSpec, cand) -> bool:
    """The ring form's conditions (tcs_capi.cpp tmem_cols): 3D Star Row, FP64 or FP32, 4..32
    columns per ring entry, whole warps, the ring within 512 columns."""
    cx, cy, bx, by, ch = cand[:5]
    if base.dimension != 3 or base.neighbourhood != "Star" or base.orientation != "Row":
        return False
    if base.precision not in ("f64", "f32") or (bx * by) % 32:
        return False
    w = cx * cy * (2 if base.precision == "f64" else 1)
    need = ((bx * by + 127) // 128) * 2 * base.range * w
    return w in (4, 8, 16, 32) and need <= 512


def forms(base: StencilSpec, cand) -> list:
    return [f for f in FORMS if not f[0] or tmem_applies(base, cand)]


# ---- timing -----------------------------------------------------------------------------------
def launch_of(cand, form=(0, 0)) -> Launch:
    cx, cy, bx, by, ch = cand[:5]
    return Launch(block=(bx, by, 1), variant="pipe", chunk=ch, tmem=bool(form[0]), lockstep=bool(form[1]))


def time_candidate(base: StencilSpec, grid, cand, mask, bufs: dict, sweeps: int = 3, form=(0, 0)) -> float | None:
    """GLup/s of the pipelined kernel at this candidate on the problem's grid (geometry of the
    candidate's coarsening), or None when it cannot run."""
    import torch

    spec = problem_spec(base, cand)
    try:
        geom = spec.geometry(*grid)
        st = Stencil(spec)
    except _lib.TcsError:
        return None
    try:
        if mask is not None:
            st.copy_mask(mask)
        shape = tuple(geom.shape)
        if bufs.get("shape") != shape:
            bufs.clear()
            torch.cuda.empty_cache()
            dt = torch.float64 if spec.precision == "f64" else torch.float32
            g = torch.Generator(device="cuda")
            g.manual_seed(5)
            bufs["x"] = torch.rand(shape, dtype=dt, device="cuda", generator=g)
            bufs["y"] = bufs["x"].clone()
            bufs["shape"] = shape
        launch = launch_of(cand, form)
        st.update_grid(geom, bufs["x"], bufs["y"], launch)
        ms = st.time_sweeps(geom, bufs["x"], bufs["y"], sweeps, launch)
        if st.device_status() != 0:
            raise RuntimeError("device status word set while timing %s" % (cand,))
    except _lib.TcsError:
        return None
    finally:
        st.close()
    return geom.interior_points * sweeps / (ms / 1e3) / 1e9 if ms > 0 else None


def precompile(base: StencilSpec, cand, tmem: bool = False) -> bool:
    from .stencil import precompile_pipe

    try:
        precompile_pipe(problem_spec(base, cand), (cand[2], cand[3], 1), cand[4], tmem=tmem)
        return True
    except _lib.TcsError:
        return False


# ---- the tuner ----------------------------------------------------------------------------------
@dataclass
class PipeTuneResult:
    candidate: tuple                 # (cx, cy, bx, by, chunk)
    glups: float
    timed: int                       # launches (shape x form) compiled and timed
    candidates: int                  # launches in the space
    fell_back: bool
    seconds: float
    reason: str = ""
    measured: dict = field(default_factory=dict)  # (cx, cy, bx, by, chunk, tmem, lockstep) -> GLup/s
    form: tuple = (0, 0)             # (tmem, lockstep) of the chosen launch


class PipeTuner:
    def __init__(self, model: CostModel | None = None, top_k: int = 5, tolerance: float = 0.3, sweeps: int = 3):
        self.model, self.top_k, self.tolerance, self.sweeps = model, top_k, tolerance, sweeps

    def rank(self, base: StencilSpec, grid, cands: list) -> np.ndarray:
        X = np.stack([features(base, grid, c) for c in cands])
        return X, self.model.predict(X)

    def _space(self, base, cands) -> int:
        return sum(len(forms(base, c)) for c in cands)

    def _result(self, res, n_space, fell_back, t0, reason) -> PipeTuneResult:
        best = max(res, key=res.get)
        return PipeTuneResult(tuple(best[:5]), res[best], len(res), n_space, fell_back, time.perf_counter() - t0,
                              reason, res, tuple(best[5:]))

    def tune(self, base: StencilSpec, grid, mask=None) -> PipeTuneResult:
        """The model ranks the shapes (register form, even split); the top k are timed in that form
        (the model is checked against those timings) and then in their other forms."""
        t0 = time.perf_counter()
        cands = candidates(base)
        bufs = {}
        if self.model is None:
            return self._exhaustive(base, grid, cands, mask, bufs, t0, "no model")
        X, pred = self.rank(base, grid, cands)
        if not self.model.in_domain(X):
            return self._exhaustive(base, grid, cands, mask, bufs, t0, "problem outside the training corpus")
        measured, predicted = {}, {}
        for i in np.argsort(-pred):
            if len(measured) >= self.top_k:
                break
            g = time_candidate(base, grid, cands[i], mask, bufs, self.sweeps)
            if g is not None:
                measured[cands[i]] = g
                predicted[cands[i]] = float(pred[i])
        if not measured:
            return self._exhaustive(base, grid, cands, mask, bufs, t0, "no predicted candidate runs")
        best = max(measured, key=measured.get)
        err = max(abs((predicted[c] - predicted[best]) - math.log(measured[c] / measured[best])) for c in measured)
        if err > self.tolerance:
            return self._exhaustive(base, grid, cands, mask, bufs, t0,
                                    "prediction error %.2f (log) above %.2f" % (err, self.tolerance))
        res = {tuple(c) + (0, 0): g for c, g in measured.items()}
        for c in measured:
            for f in forms(base, c):
                if f != (0, 0):
                    g = time_candidate(base, grid, c, mask, bufs, self.sweeps, f)
                    if g is not None:
                        res[tuple(c) + f] = g
        return self._result(res, self._space(base, cands), False, t0, "model top-%d" % self.top_k)

    def _exhaustive(self, base, grid, cands, mask, bufs, t0, reason) -> PipeTuneResult:
        res = {}
        for c in cands:
            for f in forms(base, c):
                g = time_candidate(base, grid, c, mask, bufs, self.sweeps, f)
                if g is not None:
                    res[tuple(c) + f] = g
        if not res:
            raise _lib.UnsupportedLaunch(_lib.TCS_ERR_UNSUPPORTED, "no pipelined launch runs this problem")
        return self._result(res, self._space(base, cands), True, t0, reason)


# ---- corpus, training, evaluation ---------------------------------------------------------------
def _problem_mask(base: StencilSpec, seed: int):
    if base.coefficients != "Variable":
        return None
    return np.random.default_rng(seed).standard_normal(base.stencil_size) / base.stencil_size


def corpus_plan(n_problems: int, per_problem: int, seed: int = 13) -> list:
    """[(problem id, base spec, grid, candidate)] of the corpus: a seeded subset of each problem's
    candidates."""
    rng = np.random.default_rng(seed + 1)
    plan = []
    for pid, base in enumerate(sample_problems(n_problems, seed)):
        grid = corpus_grid(base)
        for c in subset(candidates(base), per_problem, rng):
            plan.append((pid, base, grid, c))
    return plan


def _precompile_job(job):
    pid, base, grid, c = job[:4]
    return precompile(base, c, bool(job[4]) if len(job) > 4 else False)


def build_corpus(n_problems: int, per_problem: int, out: Path, seed: int = 13, log=print) -> dict:
    """Time the planned candidates on the GPU; rows (problem id, features..., log GLup/s)."""
    import torch

    rows = []
    plan = corpus_plan(n_problems, per_problem, seed)
    t0 = time.perf_counter()
    by_problem = {}
    for pid, base, grid, c in plan:
        by_problem.setdefault(pid, (base, grid, []))[2].append(c)
    for pid, (base, grid, cands) in by_problem.items():
        bufs = {}
        mask = _problem_mask(base, pid)
        best = 0.0
        for c in cands:
            g = time_candidate(base, grid, c, mask, bufs)
            if g is not None:
                rows.append((pid, *features(base, grid, c), math.log(g)))
                best = max(best, g)
        log("problem %d %s: %d candidates, best %.1f GLup/s" % (pid, _name(base), len(cands), best))
        bufs.clear()
        torch.cuda.empty_cache()
    a = np.array(rows, dtype=np.float32).reshape(-1, len(PIPE_FEATURES) + 2)
    out.parent.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(out, samples=a, features=np.array(PIPE_FEATURES), n_problems=n_problems, seed=seed)
    return {"samples": len(rows), "seconds": time.perf_counter() - t0}


# ---- batched sweeps -------------------------------------------------------------------------------
def batch_candidates(spec: StencilSpec) -> list:
    """(bx, by, chunk) of the batched pipelined sweep for a batch's parameter set (its coarsening
    is the batch's own): blocks of 32..128 x 1..16 threads with 64..1024 in all, tiles within the
    256-element TMA box, 1 to 3 planes per chunk."""
    R, es = spec.range, spec.itemsize
    vec = 16 // es
    out = []
    for bx in (32, 64, 128):
        tx = bx * spec.cx
        if tx % vec or tx + 2 * R + vec > 256:
            continue
        for by in (1, 2, 4, 6, 7, 8, 16):
            if not 64 <= bx * by <= 1024 or by * spec.cy + 2 * R > 256:
                continue
            for ch in (1, 2, 3):
                out.append((bx, by, ch))
    return out


def time_batch(w, precision: str, cand, state: dict, sweeps: int = 10) -> float | None:
    """GLup/s of one batched launch (one launch per sweep over every grid of the batch), CUDA
    events around `sweeps` sweeps after two warm-up sweeps; None when the shape does not run."""
    import torch

    from .batch import BatchedSweeps

    if "st" not in state:
        spec = w.spec.replace(precision=precision)
        state["st"] = Stencil(spec)
        geoms = w.geometries(spec)
        dt = np.float64 if precision == "f64" else np.float32
        state["geoms"] = geoms
        state["xs"] = [torch.from_numpy(np.ascontiguousarray(v)).cuda() for v in w.make_inputs(geoms, dt)]
        state["ys"] = [x.clone() for x in state["xs"]]
        state["points"] = sum(g.interior_points for g in geoms)
    bx, by, ch = cand[:3]
    ctas = cand[3] if len(cand) > 3 else 0
    try:
        bt = BatchedSweeps(state["st"], state["geoms"], state["xs"], state["ys"],
                           Launch(block=(bx, by, 1), variant="pipe", chunk=ch, segments=ctas))
    except _lib.TcsError:
        return None
    try:
        stream = torch.cuda.current_stream()
        bt.sweeps(2, stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        bt.sweeps(sweeps, stream)
        e1.record(stream)
        torch.cuda.synchronize()
        if state["st"].device_status() != 0:
            raise RuntimeError("device status word set while timing %s" % (cand,))
        ms = e0.elapsed_time(e1)
    finally:
        bt.close()
    return state["points"] * sweeps / (ms / 1e3) / 1e9 if ms > 0 else None


# CTA counts of the batched launch's second stage, in waves of one CTA per SM (0: one wave of
# every resident CTA).  Several waves of short contiguous work runs let the CTAs that finish early
# (runs of TMA-loaded grids) take more of the work list than those on cp.async-loaded grids.
BATCH_WAVES = (0, 2, 4, 6, 8, 12, 16)


def tune_batch(w, precision: str = "f64", num_sms: int | None = None) -> PipeTuneResult:
    """Exhaustive search of the batched sweep's launch (the cost model covers single grids):
    every (bx, by, chunk) at one wave of CTAs, then the CTA count (BATCH_WAVES) for the three
    fastest shapes.  Candidates are (bx, by, chunk, ctas)."""
    from .stencil import device_sm_count

    t0 = time.perf_counter()
    cands = batch_candidates(w.spec)
    state, res = {}, {}
    for c in cands:
        g = time_batch(w, precision, tuple(c) + (0,), state)
        if g is not None:
            res[tuple(c) + (0,)] = g
    n_sms = num_sms or device_sm_count()
    top = sorted(res, key=res.get, reverse=True)[:3]
    n_cands = len(cands)
    for c in top:
        for waves in BATCH_WAVES[1:]:
            cc = tuple(c[:3]) + (waves * n_sms,)
            n_cands += 1
            g = time_batch(w, precision, cc, state)
            if g is not None:
                res[cc] = g
    if "st" in state:
        state["st"].close()
    if not res:
        raise _lib.UnsupportedLaunch(_lib.TCS_ERR_UNSUPPORTED, "no batched launch runs this batch")
    best = max(res, key=res.get)
    return PipeTuneResult(best, res[best], len(res), n_cands, True, time.perf_counter() - t0,
                          "batched sweep: exhaustive", res)


def batch_entry(r: PipeTuneResult) -> dict:
    """A tuned-launch record of a batched tuning result (block, chunk and CTA count; the batch's
    coarsening)."""
    bx, by, ch = r.candidate[:3]
    ctas = r.candidate[3] if len(r.candidate) > 3 else 0
    runner_up = sorted(((v, k) for k, v in r.measured.items() if tuple(k) != tuple(r.candidate)), reverse=True)[:1]
    src = "pipetune exhaustive over %d of %d batched launches: %.1f GLup/s" % (r.timed, r.candidates, r.glups)
    if runner_up:
        src += "; next %s: %.1f" % ("x".join(map(str, runner_up[0][1])), runner_up[0][0])
    e = {"block": [bx, by, 1], "variant": "pipe", "chunk": ch, "source": src}
    if ctas:
        e["segments"] = ctas
    return e


def _precompile_batch_job(job):
    from .batch import precompile_batch

    spec, cand = job
    try:
        precompile_batch(spec, (cand[0], cand[1], 1), cand[2])
        return True
    except _lib.TcsError:
        return False


def workload_base(w, precision: str = "f64") -> StencilSpec:
    """The problem of a benchmark workload: its stencil at coarsening 1 (the tuner chooses it)."""
    return w.spec.replace(precision=precision, cx=1, cy=1, cz=1)


def tuned_entry(r: PipeTuneResult) -> dict:
    """A tuned-launch record (the format workloads.py reads) of a tuning result."""
    cx, cy, bx, by, ch = r.candidate
    chosen = tuple(r.candidate) + tuple(r.form)
    full = lambda k: tuple(k) if len(k) == 7 else tuple(k) + (0, 0)  # noqa: E731  (shape keys: default form)
    runner_up = sorted(((v, k) for k, v in r.measured.items() if full(k) != chosen), reverse=True)[:1]
    how = "exhaustive" if r.fell_back else "learned (%s)" % r.reason
    src = "pipetune %s over %d of %d pipelined launches: %.1f GLup/s" % (how, r.timed, r.candidates, r.glups)
    if runner_up:
        src += "; next %s: %.1f" % ("x".join(map(str, runner_up[0][1])), runner_up[0][0])
    e = {"coarsening": [cx, cy, 1], "block": [bx, by, 1], "variant": "pipe", "chunk": ch}
    if r.form[0]:
        e["tmem"] = True
    if r.form[1]:
        e["lockstep"] = True
    e["source"] = src
    return e


def write_tuned(path: Path, name: str, precision: str, r: PipeTuneResult, batch: bool = False) -> dict:
    """Record a workload's tuned pipelined launch under ``name`` (FP64) or ``name_precision``,
    keeping the file's other entries."""
    d = json.loads(path.read_text()) if path.exists() else {}
    k = name if precision == "f64" else name + "_" + precision
    d[k] = batch_entry(r) if batch else tuned_entry(r)
    path.parent.mkdir(parents=True, exist_ok=True)
    path.write_text(json.dumps(d, indent=1) + "\n")
    return d[k]


def _name(s: StencilSpec) -> str:
    return "%dD %s %s r%d %s" % (s.dimension, s.neighbourhood, s.coefficients, s.range, s.precision)


def load_corpus(path: Path = PIPE_CORPUS_PATH):
    d = np.load(path)
    a = d["samples"]
    return a[:, 0].astype(np.int64), a[:, 1:-1], a[:, -1]


def holdout_ids(n_problems: int, n_holdout: int = 8, seed: int = 3) -> list:
    """Seeded held-out problem ids (never trained on)."""
    rng = np.random.default_rng(seed)
    return sorted(rng.choice(n_problems, size=min(n_holdout, n_problems // 4), replace=False).tolist())


def live_check_problem(n_problems: int = 40) -> int:
    """The held-out problem a quick live check tunes: the first 3D FP64 Jacobi one (its 148
    instantiations compile fastest of the 3D spaces)."""
    problems = sample_problems(n_problems)
    for pid in holdout_ids(n_problems):
        b = problems[pid]
        if b.dimension == 3 and b.precision == "f64" and b.coefficients == "Jacobi":
            return pid
    return holdout_ids(n_problems)[0]


def split(pids: np.ndarray, n_problems: int):
    hold = holdout_ids(n_problems)
    return hold, np.array([p not in hold for p in pids])


def evaluate_corpus(model: CostModel, pids, X, y, ids, top_k: int = 5, seed: int = 3) -> dict:
    """Held-out quality on the corpus timings: best of the model's top-k against the best timed
    candidate, and against k random candidates (the method without a model, same budget)."""
    rng = np.random.default_rng(seed)
    ratios, rnd = [], []
    for p in ids:
        sel = pids == p
        g = np.exp(y[sel])
        pred = model.predict(X[sel])
        ratios.append(g[np.argsort(-pred)[:top_k]].max() / g.max())
        rnd.append(np.mean([g[rng.choice(len(g), size=min(top_k, len(g)), replace=False)].max() / g.max()
                            for _ in range(20)]))
    r = np.array(ratios)
    return {"problems": len(ids), "top_k": top_k, "mean_ratio_to_best": float(r.mean()),
            "within_5pct": float(np.mean(r >= 0.95)), "min_ratio": float(r.min()),
            "random_k_mean_ratio": float(np.mean(rnd))}


def live(model: CostModel, ids, n_problems: int, seed: int = 13, log=print) -> dict:
    """Tune held-out problems on the GPU with the learned tuner and exhaustively over the whole
    candidate space; both choices re-timed with 10 sweeps."""
    rows = []
    problems = sample_problems(n_problems, seed)
    for pid in ids:
        base = problems[int(pid)]
        grid = corpus_grid(base)
        mask = _problem_mask(base, int(pid))
        learned = PipeTuner(model).tune(base, grid, mask)
        full = PipeTuner(None).tune(base, grid, mask)
        bufs = {}
        g_l = time_candidate(base, grid, learned.candidate, mask, bufs, 10, learned.form)
        g_f = time_candidate(base, grid, full.candidate, mask, bufs, 10, full.form)
        rows.append({"problem": int(pid), "spec": _name(base), "learned": list(learned.candidate) + list(learned.form),
                     "exhaustive": list(full.candidate) + list(full.form), "ratio": g_l / g_f,
                     "learned_s": learned.seconds,
                     "exhaustive_s": full.seconds, "timed": learned.timed, "candidates": full.candidates,
                     "fell_back": learned.fell_back, "reason": learned.reason})
        log(json.dumps(rows[-1]))
    r = np.array([q["ratio"] for q in rows])
    return {"problems": len(rows), "mean_ratio": float(r.mean()), "min_ratio": float(r.min()),
            "within_5pct": float(np.mean(r >= 0.95)),
            "time_fraction": float(sum(q["learned_s"] for q in rows) / sum(q["exhaustive_s"] for q in rows)),
            "compiled_fraction": float(sum(q["timed"] for q in rows) / sum(q["candidates"] for q in rows)),
            "fallbacks": int(sum(q["fell_back"] for q in rows)), "rows": rows}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m threadcoarsenedstencilgenerator_b200.pipetune")
    sub = ap.add_subparsers(dest="cmd", required=True)
    for name in ("precompile", "corpus"):
        c = sub.add_parser(name)
        c.add_argument("--problems", type=int, default=40)
        c.add_argument("--per-problem", type=int, default=36)
        c.add_argument("--holdout-full", type=int, default=4, help="precompile: also the whole space of this "
                       "many held-out problems (for the live evaluation)")
        c.add_argument("--workload", action="append", default=[],
                       help="precompile: also the whole space of a benchmark workload (name:precision)")
    sub.add_parser("train")
    e = sub.add_parser("evaluate")
    e.add_argument("--live", type=int, default=0)
    e.add_argument("--problems", type=int, default=40)
    t = sub.add_parser("tune", help="tune a benchmark workload's pipelined launch (exhaustive or learned)")
    t.add_argument("--workload", required=True)
    t.add_argument("--precision", default="f64")
    t.add_argument("--exhaustive", action="store_true")
    t.add_argument("--write", type=Path, nargs="?", const=TUNED_PATH, default=None,
                   help="record the chosen launch in a tuned-launch file (default: the package's tuned.json)")
    a = ap.parse_args(argv)
    if a.cmd == "precompile":
        import multiprocessing as mp
        import os

        jobs = corpus_plan(a.problems, a.per_problem)
        problems = sample_problems(a.problems)
        for pid in holdout_ids(a.problems)[:a.holdout_full]:
            base = problems[pid]
            jobs += [(pid, base, corpus_grid(base), c, tm) for c in candidates(base)
                     for tm in sorted({f[0] for f in forms(base, c)})]
        batch_jobs = []
        if a.workload:
            from .workloads import BATCH_WORKLOADS, WORKLOADS

            for item in a.workload:
                name, _, prec = item.partition(":")
                if name in BATCH_WORKLOADS:
                    spec = BATCH_WORKLOADS[name].spec.replace(precision=prec or "f64")
                    batch_jobs += [(spec, c) for c in batch_candidates(spec)]
                    continue
                base = workload_base(WORKLOADS[name], prec or "f64")
                jobs += [(-1, base, WORKLOADS[name].grid, c, tm) for c in candidates(base)
                         for tm in sorted({f[0] for f in forms(base, c)})]
        with mp.get_context("spawn").Pool(os.cpu_count() or 4) as pool:
            ok = pool.map(_precompile_job, jobs, chunksize=1)
            ok += pool.map(_precompile_batch_job, batch_jobs, chunksize=1)
        print(json.dumps({"instantiations": len(jobs) + len(batch_jobs), "compiled": int(sum(ok))}))
        return 0
    if a.cmd == "corpus":
        print(json.dumps(build_corpus(a.problems, a.per_problem, PIPE_CORPUS_PATH)))
        return 0
    if a.cmd == "tune":
        from .workloads import BATCH_WORKLOADS, WORKLOADS

        if a.workload in BATCH_WORKLOADS:
            w = BATCH_WORKLOADS[a.workload]
            r = tune_batch(w, a.precision)
            print(json.dumps({"workload": w.name, "precision": a.precision, "candidate": list(r.candidate),
                              "glups": r.glups, "timed": r.timed, "candidates": r.candidates, "seconds": r.seconds,
                              "top": sorted(([list(k), v] for k, v in r.measured.items()), key=lambda q: -q[1])[:10]}))
            if a.write is not None:
                write_tuned(a.write, w.name, a.precision, r, batch=True)
            return 0
        w = WORKLOADS[a.workload]
        base = workload_base(w, a.precision)
        model = None if a.exhaustive else CostModel.load(PIPE_MODEL_PATH, PIPE_FEATURES)
        r = PipeTuner(model).tune(base, w.grid, w.make_mask())
        print(json.dumps({"workload": w.name, "candidate": list(r.candidate), "form": list(r.form), "glups": r.glups,
                          "timed": r.timed,
                          "candidates": r.candidates, "fell_back": r.fell_back, "seconds": r.seconds,
                          "reason": r.reason, "top": sorted(([list(k), v] for k, v in r.measured.items()),
                                                            key=lambda q: -q[1])[:10]}))
        if a.write is not None:
            write_tuned(a.write, w.name, a.precision, r)
        return 0
    pids, X, y = load_corpus()
    hold, train_mask = split(pids, int(np.load(PIPE_CORPUS_PATH)["n_problems"]))
    if a.cmd == "train":
        m = CostModel(features=PIPE_FEATURES)
        t0 = time.perf_counter()
        hist = m.fit(X[train_mask], y[train_mask], groups=pids[train_mask], epochs=300)
        dt = time.perf_counter() - t0
        m.save(PIPE_MODEL_PATH, epochs=300, train_seconds=dt, final_loss=hist[-1], holdout=[int(h) for h in hold])
        print(json.dumps({"train_seconds": dt, "final_loss": hist[-1], **evaluate_corpus(m, pids, X, y, hold)}))
        return 0
    m = CostModel.load(PIPE_MODEL_PATH, PIPE_FEATURES)
    out = {"corpus": evaluate_corpus(m, pids, X, y, hold)}
    if a.live:
        out["live"] = live(m, hold[:a.live], a.problems)
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
