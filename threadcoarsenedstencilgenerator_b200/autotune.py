"""Block-shape autotuner: exhaustive timed sweep, and a learned cost model that prunes it.

The reference picks a thread-block shape by timing every shape for about a second each
(cuda/benchmark.cpp:223-251, 287-318, with the doubling loop of
cuda/generateLaunchUpdateGrid.py:103-147).  Here

* ``exhaustive`` times every candidate block of the drop-in (direct) kernel with CUDA events over a
  few sweeps of the real grid (milliseconds per candidate instead of a second);
* ``CostModel`` is a 3-layer perceptron (128 hidden units, FP32) that predicts log GLup/s of a
  (parameter set, grid, block) triple from one-hot and numeric features, relative to the mean over
  that parameter set's candidates (the targets are centred per parameter set: ranking the blocks
  of one set needs only the differences).  It is trained and evaluated on the GPU by libtcs.so's
  own kernels (``tcs_mlp_*``);
* ``Autotuner.tune`` ranks all candidates with the model, times only the top k (5), and falls back
  to the exhaustive sweep when the model is missing, the parameter set lies outside the corpus the
  model was trained on, or the measured differences between the timed candidates disagree with the
  predicted ones by more than a tolerance even after the candidates are timed again over more
  sweeps (the sweep then also records the model's error).

``python -m threadcoarsenedstencilgenerator_b200.autotune corpus|train|evaluate`` builds the
timing corpus on a GPU, trains the model on it and reports its held-out quality.
"""

from __future__ import annotations

import argparse
import ctypes
import json
import math
import sys
import time
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import _lib
from .spec import Geometry, StencilSpec
from .stencil import Launch, Stencil, _ptr, _stream

DATA = Path(__file__).resolve().parent / "data"
CORPUS_PATH = DATA / "tuner_corpus.npz"
MODEL_PATH = DATA / "costmodel.npz"

HIDDEN = 128
TERM_BUDGET = 2048      # stencil points x outputs per thread: larger sets are not sampled
GRID_BYTES = 512 << 20  # one buffer of a corpus grid (two buffers: ~1 GB)

FEATURES = [
    "dim2", "dim3", "box", "star", "jacobi", "variable", "f64", "f32",
    "range", "log_cx", "log_cy", "log_cz", "log_S", "log_NE", "log_terms",
    "log_bx", "log_by", "log_bz", "log_threads", "log_tile_x", "log_tile_y", "log_tile_z",
    "log_potential_block", "log_nx", "log_ny", "log_nz",
    "log_warps_per_sm", "log_waves", "tail_efficiency", "tile_efficiency",
]


# ---- candidates and features ------------------------------------------------------------------
def candidate_blocks(dimension: int, max_threads: int = 1024) -> list:
    """Blocks with a power-of-two thread count from one warp to ``max_threads`` and power-of-two
    extents (z <= 64), x fastest: the shapes of the reference's sweep (cuda/primes.cpp) whose
    warp count is a power of two."""
    out = []
    n = 32
    while n <= max_threads:
        k = int(math.log2(n))
        if dimension == 2:
            for a in range(k, -1, -1):
                out.append((1 << a, 1 << (k - a), 1))
        else:
            for a in range(k, -1, -1):
                for b in range(k - a, -1, -1):
                    c = k - a - b
                    if (1 << c) <= 64:
                        out.append((1 << a, 1 << b, 1 << c))
        n *= 2
    return out


def reference_blocks(dimension: int, max_threads: int = 1024) -> list:
    """Every block shape of the reference's sweep (cuda/primes.cpp as restated by primes.py):
    464 in 2D, 2,723 in 3D at 1024 threads -- the space the reference times shape by shape."""
    from .primes import block_shapes

    return [tuple(b) + (1,) * (3 - len(b)) for b in block_shapes(dimension, max_threads)]


def blocks_of(space: str, dimension: int) -> list:
    """Candidate blocks of a search space: "pow2" (power-of-two shapes, the corpus's) or
    "reference" (the reference's whole enumeration)."""
    if space == "reference":
        return reference_blocks(dimension)
    return candidate_blocks(dimension)


def features(spec: StencilSpec, geom: Geometry, block, potential_block: int, plan) -> np.ndarray:
    """Feature vector of one candidate (order: FEATURES); ``plan`` is the direct launch resolved for
    it (CTA grid and resident CTAs per SM, from the driver's occupancy calculator)."""
    d3 = spec.dimension == 3
    cz = spec.cz if d3 else 1
    bz = block[2] if d3 else 1
    S = spec.stencil_size
    ne = spec.cx * spec.cy * cz
    l2 = lambda v: math.log2(max(1, v))  # noqa: E731
    return np.array([
        not d3, d3, spec.neighbourhood == "Box", spec.neighbourhood == "Star",
        spec.coefficients == "Jacobi", spec.coefficients == "Variable",
        spec.precision == "f64", spec.precision == "f32",
        spec.range, l2(spec.cx), l2(spec.cy), l2(cz), l2(S), l2(ne), l2(S * ne),
        l2(block[0]), l2(block[1]), l2(bz), l2(block[0] * block[1] * bz),
        l2(block[0] * spec.cx), l2(block[1] * spec.cy), l2(bz * cz),
        l2(potential_block), l2(geom.grid[0]), l2(geom.grid[1]), l2(geom.grid[2] if d3 else 1),
        *_launch_features(geom, block, plan, d3),
    ], dtype=np.float32)


def _launch_features(geom: Geometry, block, plan, d3: bool) -> list:
    threads = block[0] * block[1] * (block[2] if d3 else 1)
    occ = max(1, plan.ctas_per_sm)
    ctas = plan.grid_blocks[0] * plan.grid_blocks[1] * (plan.grid_blocks[2] if d3 else 1)
    per_wave = plan.num_sms * occ
    waves = ctas / per_wave
    tile = 1.0
    for i in range(3 if d3 else 2):
        tile *= geom.threads[i] / float(plan.grid_blocks[i] * block[i])
    return [math.log2(occ * threads / 32.0), math.log2(max(waves, 1e-3)), ctas / (math.ceil(waves) * per_wave),
            tile]


def candidate_features(st: Stencil, geom: Geometry, blocks) -> tuple:
    """(runnable blocks, their feature matrix): blocks the direct kernel cannot launch are dropped."""
    pot = st.max_potential_block_size()
    keep, rows = [], []
    for b in blocks:
        try:
            plan = st.plan(geom, Launch(block=tuple(b), variant="direct"))
        except _lib.TcsError:
            continue
        keep.append(tuple(b))
        rows.append(features(st.spec, geom, b, pot, plan))
    return keep, (np.stack(rows) if rows else np.zeros((0, len(FEATURES)), np.float32))


def corpus_grid(spec: StencilSpec) -> tuple:
    """Grid extents of a corpus configuration: one buffer of about GRID_BYTES."""
    pts = GRID_BYTES // spec.itemsize
    if spec.dimension == 2:
        s = int(math.sqrt(pts))
        return (s, s, 1)
    s = int(round(pts ** (1.0 / 3.0)))
    return (s, s, s)


def sample_configs(n: int, seed: int = 7) -> list:
    """Seeded parameter sets: dim 2/3, Box/Star, range 1-8, Jacobi/Variable, FP64/FP32,
    coarsening 1-8 per axis, Row orientation, no alignment; sets whose unrolled work per thread
    (stencil points x outputs) exceeds TERM_BUDGET are redrawn."""
    rng = np.random.default_rng(seed)
    out = []
    seen = set()
    while len(out) < n:
        d = int(rng.choice([2, 3]))
        spec = StencilSpec(dimension=d, neighbourhood=str(rng.choice(["Box", "Star"])), orientation="Row",
                           coefficients=str(rng.choice(["Jacobi", "Variable"])), range=int(rng.integers(1, 9)),
                           cx=int(rng.integers(1, 9)), cy=int(rng.integers(1, 9)),
                           cz=int(rng.integers(1, 9)) if d == 3 else 1,
                           precision=str(rng.choice(["f64", "f32"])))
        ne = spec.cx * spec.cy * spec.cz
        if ne > 512 or spec.stencil_size * ne > TERM_BUDGET:
            continue
        key = repr(spec)
        if key in seen:
            continue
        seen.add(key)
        out.append(spec)
    return out


# ---- timing -----------------------------------------------------------------------------------
def time_block(st: Stencil, geom: Geometry, x, y, block, sweeps: int = 2) -> float | None:
    """GLup/s of the direct kernel with this block (one warm-up sweep, then ``sweeps`` timed with
    CUDA events), or None when the kernel cannot run the shape."""
    launch = Launch(block=tuple(block), variant="direct")
    try:
        st.update_grid(geom, x, y, launch)
        ms = st.time_sweeps(geom, x, y, sweeps, launch)
    except _lib.TcsError:
        return None
    if ms <= 0:
        return None
    return geom.interior_points * sweeps / (ms / 1e3) / 1e9


def exhaustive(st: Stencil, geom: Geometry, x, y, blocks, sweeps: int = 2) -> list:
    """[(block, GLup/s)] for every block the kernel can run, in candidate order."""
    out = []
    for b in blocks:
        g = time_block(st, geom, x, y, b, sweeps)
        if g is not None:
            out.append((tuple(b), g))
    return out


# ---- the cost model on the GPU ----------------------------------------------------------------
class CostModel:
    """3-layer perceptron on standardised features, predicting log GLup/s (tcs_mlp_* kernels)."""

    def __init__(self, n_in: int | None = None, hidden: int = HIDDEN, max_batch: int = 4096,
                 params: np.ndarray | None = None, seed: int = 0, features: list | None = None):
        self.features = list(features or FEATURES)
        n_in = n_in or len(self.features)
        self._lib = _lib.load()
        self.n_in, self.hidden, self.max_batch = n_in, hidden, max_batch
        h = ctypes.c_void_p()
        _lib.check(self._lib.tcs_mlp_create(n_in, hidden, max_batch, ctypes.byref(h)))
        self._h = h
        c = ctypes.c_uint()
        _lib.check(self._lib.tcs_mlp_param_count(self._h, ctypes.byref(c)))
        self.n_params = c.value
        self.x_mean = np.zeros(n_in, np.float32)
        self.x_std = np.ones(n_in, np.float32)
        self.y_mean, self.y_std = 0.0, 1.0
        self.feature_lo = np.full(n_in, -np.inf, np.float32)
        self.feature_hi = np.full(n_in, np.inf, np.float32)
        self.set_params(params if params is not None else init_params(n_in, hidden, seed))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.tcs_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        _lib.check(self._lib.tcs_mlp_set_params(self._h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), p.size))

    def params(self) -> np.ndarray:
        p = np.empty(self.n_params, np.float32)
        _lib.check(self._lib.tcs_mlp_get_params(self._h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), p.size))
        return p

    # raw network on device tensors (standardised inputs and targets)
    def forward_raw(self, x_dev, y_dev, stream=None) -> None:
        n = int(x_dev.shape[0])
        _lib.check(self._lib.tcs_mlp_forward(self._h, _ptr(x_dev), n, _ptr(y_dev), _stream(stream)))

    def gradient_raw(self, x_dev, t_dev, grad_dev=None, stream=None) -> float:
        loss = ctypes.c_float()
        _lib.check(self._lib.tcs_mlp_gradient(self._h, _ptr(x_dev), _ptr(t_dev), int(x_dev.shape[0]),
                                              None if grad_dev is None else _ptr(grad_dev), ctypes.byref(loss),
                                              _stream(stream)))
        return loss.value

    def adam_step_raw(self, x_dev, t_dev, lr: float, want_loss: bool = False, stream=None,
                      beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8) -> float | None:
        loss = ctypes.c_float()
        _lib.check(self._lib.tcs_mlp_adam_step(self._h, _ptr(x_dev), _ptr(t_dev), int(x_dev.shape[0]), lr, beta1,
                                               beta2, eps, ctypes.byref(loss) if want_loss else None,
                                               _stream(stream)))
        return loss.value if want_loss else None

    # standardised interface
    def fit(self, X: np.ndarray, y: np.ndarray, groups: np.ndarray | None = None, epochs: int = 150,
            batch: int = 1024, lr: float = 2e-3, seed: int = 0, log=None) -> list:
        """Train on features X [n x n_in] and targets y = log GLup/s [n] (centred per group when
        ``groups`` gives each row's parameter set); returns the per-epoch mean training loss
        (standardised units)."""
        import torch

        X = np.asarray(X, np.float32)
        y = np.asarray(y, np.float32).copy()
        if groups is not None:
            for gid in np.unique(groups):
                sel = groups == gid
                y[sel] -= y[sel].mean()
        self.x_mean = X.mean(axis=0)
        self.x_std = np.where(X.std(axis=0) > 1e-6, X.std(axis=0), 1.0).astype(np.float32)
        self.y_mean, self.y_std = float(y.mean()), float(y.std() or 1.0)
        self.feature_lo, self.feature_hi = X.min(axis=0), X.max(axis=0)
        Xs = torch.from_numpy((X - self.x_mean) / self.x_std).cuda()
        ys = torch.from_numpy((y - self.y_mean) / self.y_std).cuda()
        n = Xs.shape[0]
        batch = min(batch, self.max_batch, n)
        rng = np.random.default_rng(seed)
        history = []
        for ep in range(epochs):
            perm = torch.from_numpy(rng.permutation(n)).cuda()
            Xp, yp = Xs[perm].contiguous(), ys[perm].contiguous()
            lr_ep = lr * 0.5 * (1 + math.cos(math.pi * ep / epochs))  # cosine decay
            losses = []
            nb = n // batch
            for b in range(nb):
                want = b == nb - 1 or b % 16 == 0
                l = self.adam_step_raw(Xp[b * batch:(b + 1) * batch], yp[b * batch:(b + 1) * batch], lr_ep,
                                       want_loss=want)
                if l is not None:
                    losses.append(l)
            history.append(float(np.mean(losses)))
            if log and (ep % 10 == 0 or ep == epochs - 1):
                log("epoch %d loss %.4f" % (ep, history[-1]))
        return history

    def predict(self, X: np.ndarray) -> np.ndarray:
        """Predicted log GLup/s for features X [n x n_in] (inference on the GPU)."""
        import torch

        X = np.asarray(X, np.float32)
        xs = torch.from_numpy((X - self.x_mean) / self.x_std).cuda()
        out = torch.empty(X.shape[0], dtype=torch.float32, device="cuda")
        self.forward_raw(xs, out)
        torch.cuda.synchronize()
        return out.cpu().numpy() * self.y_std + self.y_mean

    def in_domain(self, X: np.ndarray, slack: float = 0.1) -> bool:
        """Every feature within the training range widened by ``slack`` of its width."""
        X = np.asarray(X, np.float32)
        w = (self.feature_hi - self.feature_lo) * slack + 1e-3
        return bool(np.all(X >= self.feature_lo - w) and np.all(X <= self.feature_hi + w))

    def save(self, path: Path = MODEL_PATH, **meta) -> None:
        path.parent.mkdir(parents=True, exist_ok=True)
        np.savez_compressed(path, params=self.params(), x_mean=self.x_mean, x_std=self.x_std,
                            y_mean=self.y_mean, y_std=self.y_std, feature_lo=self.feature_lo,
                            feature_hi=self.feature_hi, hidden=self.hidden, features=np.array(self.features),
                            meta=json.dumps(meta))

    @classmethod
    def load(cls, path: Path = MODEL_PATH, features: list | None = None) -> "CostModel":
        d = np.load(path, allow_pickle=False)
        names = list(features or FEATURES)
        if list(d["features"]) != names:
            raise ValueError("cost model was trained on another feature set")
        m = cls(n_in=len(names), hidden=int(d["hidden"]), params=d["params"], features=names)
        m.x_mean, m.x_std = d["x_mean"], d["x_std"]
        m.y_mean, m.y_std = float(d["y_mean"]), float(d["y_std"])
        m.feature_lo, m.feature_hi = d["feature_lo"], d["feature_hi"]
        return m


def init_params(n_in: int, hidden: int, seed: int) -> np.ndarray:
    """He-normal weights (fan-in), zero biases."""
    rng = np.random.default_rng(seed)
    parts = [rng.standard_normal((n_in, hidden)) * math.sqrt(2.0 / n_in), np.zeros(hidden),
             rng.standard_normal((hidden, hidden)) * math.sqrt(2.0 / hidden), np.zeros(hidden),
             rng.standard_normal(hidden) * math.sqrt(1.0 / hidden), np.zeros(1)]
    return np.concatenate([q.ravel() for q in parts]).astype(np.float32)


# ---- the tuner --------------------------------------------------------------------------------
@dataclass
class TuneResult:
    block: tuple
    glups: float
    timed: int                      # candidates timed
    candidates: int                 # candidates that exist
    fell_back: bool                 # exhaustive sweep ran
    seconds: float                  # wall time of the tuning
    reason: str = ""
    predicted: dict = field(default_factory=dict)  # block -> predicted relative log GLup/s (timed ones)
    measured: dict = field(default_factory=dict)   # block -> measured GLup/s
    model_error: float | None = None               # largest gap between measured and predicted differences


class Autotuner:
    """Picks the direct kernel's block for (stencil, grid): model-ranked top-k, exhaustive fallback."""

    def __init__(self, model: CostModel | None = None, top_k: int = 5, tolerance: float = 0.25,
                 sweeps: int = 2, space: str = "pow2"):
        self.model = model
        self.space = space  # candidate blocks: "pow2" or the reference's whole enumeration
        self.top_k = top_k
        # allowed gap between measured and predicted log-throughput differences of the timed blocks
        self.tolerance = tolerance
        self.sweeps = sweeps

    def rank(self, st: Stencil, geom: Geometry, blocks: list) -> tuple:
        """(runnable blocks, features, predicted relative log GLup/s)."""
        keep, X = candidate_features(st, geom, blocks)
        return keep, X, self.model.predict(X)

    def tune(self, st: Stencil, geom: Geometry, x, y) -> TuneResult:
        t0 = time.perf_counter()
        blocks = blocks_of(self.space, st.spec.dimension)
        if self.model is None:
            return self._exhaustive(st, geom, x, y, blocks, t0, "no model")
        keep, X, pred = self.rank(st, geom, blocks)
        if not keep:
            raise _lib.UnsupportedLaunch(_lib.TCS_ERR_UNSUPPORTED, "no candidate block runs this parameter set")
        if not self.model.in_domain(X):
            return self._exhaustive(st, geom, x, y, keep, t0, "parameter set outside the training corpus")
        order = np.argsort(-pred)
        timed, measured, predicted = 0, {}, {}
        for i in order:
            if timed >= self.top_k:
                break
            g = time_block(st, geom, x, y, keep[i], self.sweeps)
            if g is None:
                continue
            timed += 1
            measured[keep[i]] = g
            predicted[keep[i]] = float(pred[i])
        if not measured:
            return self._exhaustive(st, geom, x, y, keep, t0, "no predicted candidate runs")
        best, err = self._model_error(measured, predicted)
        if err > self.tolerance:
            # A timing over a couple of sweeps can be off by more than the tolerance on its own:
            # before giving up on the model, time the same candidates again over twice the sweeps.
            # Interference and clock dips only ever slow a run down, so each block keeps the
            # faster of its two timings.
            for b in list(measured):
                g = time_block(st, geom, x, y, b, 2 * self.sweeps)
                if g is not None:
                    measured[b] = max(measured[b], g)
            best, err = self._model_error(measured, predicted)
        if err > self.tolerance:
            r = self._exhaustive(st, geom, x, y, keep, t0, "prediction error %.2f (log) above %.2f" % (
                err, self.tolerance))
            r.predicted = predicted
            r.model_error = err
            return r
        return TuneResult(best, measured[best], timed, len(keep), False, time.perf_counter() - t0,
                          "model top-%d" % self.top_k, predicted, measured, err)

    @staticmethod
    def _model_error(measured: dict, predicted: dict) -> tuple:
        """(best timed block, largest gap between the measured and the predicted log-throughput
        difference of a timed block to the best one)."""
        best = max(measured, key=measured.get)
        err = max(abs((predicted[b] - predicted[best]) - math.log(measured[b] / measured[best])) for b in measured)
        return best, err

    def _exhaustive(self, st, geom, x, y, blocks, t0, reason) -> TuneResult:
        res = exhaustive(st, geom, x, y, blocks, self.sweeps)
        if not res:
            raise _lib.UnsupportedLaunch(_lib.TCS_ERR_UNSUPPORTED, "no candidate block runs this parameter set")
        best = max(res, key=lambda r: r[1])
        return TuneResult(best[0], best[1], len(res), len(blocks), True, time.perf_counter() - t0, reason,
                          {}, dict(res))


# ---- corpus / training / evaluation entry points ----------------------------------------------
def _alloc(spec: StencilSpec, geom: Geometry, seed: int):
    import torch

    dt = torch.float64 if spec.precision == "f64" else torch.float32
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    x = torch.rand(geom.shape, dtype=dt, device="cuda", generator=g)
    return x, x.clone()


def build_corpus(n_configs: int, seed: int, out: Path, sweeps: int = 2, log=print, start: int = 0,
                 time_budget_s: float | None = None) -> dict:
    """Time every candidate block of ``n_configs`` sampled parameter sets on ~1 GB grids."""
    import torch

    specs = sample_configs(n_configs, seed)
    rows, cfg_rows = [], []
    if out.exists() and start > 0:
        d = np.load(out)
        rows = [tuple(r) for r in d["samples"]]
    t_start = time.perf_counter()
    for ci in range(start, len(specs)):
        if time_budget_s is not None and time.perf_counter() - t_start > time_budget_s:
            log("time budget reached after %d configurations" % ci)
            break
        spec = specs[ci]
        geom = spec.geometry(*corpus_grid(spec))
        st = Stencil(spec)
        if spec.coefficients == "Variable":
            st.copy_mask(np.random.default_rng(ci).standard_normal(spec.stencil_size) / spec.stencil_size)
        x, y = _alloc(spec, geom, ci)
        blocks, F = candidate_features(st, geom, candidate_blocks(spec.dimension))
        fmap = dict(zip(blocks, F))
        t0 = time.perf_counter()
        res = exhaustive(st, geom, x, y, blocks, sweeps)
        if st.device_status() != 0:
            raise RuntimeError("device status word set during the corpus sweep")
        for b, g in res:
            rows.append((ci, *fmap[b], math.log(g)))
        log("config %d/%d %s: %d blocks, best %.1f GLup/s (%.1fs)" % (
            ci + 1, len(specs), _spec_str(spec), len(res), max(g for _, g in res) if res else 0.0,
            time.perf_counter() - t0))
        st.close()
        del x, y
        torch.cuda.empty_cache()
        if ci % 20 == 19 or ci == len(specs) - 1:
            _save_corpus(out, rows, n_configs, seed)
    _save_corpus(out, rows, n_configs, seed)
    return {"samples": len(rows)}


def _spec_str(s: StencilSpec) -> str:
    return "%dD %s %s r%d c%dx%dx%d %s" % (s.dimension, s.neighbourhood, s.coefficients, s.range, s.cx, s.cy,
                                          s.cz if s.dimension == 3 else 1, s.precision)


def _save_corpus(out: Path, rows, n_configs, seed) -> None:
    out.parent.mkdir(parents=True, exist_ok=True)
    a = np.array(rows, dtype=np.float32).reshape(-1, len(FEATURES) + 2)
    np.savez_compressed(out, samples=a, features=np.array(FEATURES), n_configs=n_configs, seed=seed)


def load_corpus(path: Path = CORPUS_PATH):
    """(config id [n], features [n x F], log GLup/s [n])."""
    d = np.load(path)
    a = d["samples"]
    return a[:, 0].astype(np.int64), a[:, 1:-1], a[:, -1]


def split(cfg: np.ndarray, n_holdout: int = 50, seed: int = 11):
    """Held-out configuration ids (seeded) and the training mask."""
    ids = np.unique(cfg)
    rng = np.random.default_rng(seed)
    hold = set(rng.choice(ids, size=min(n_holdout, len(ids) // 4), replace=False).tolist())
    return sorted(hold), np.array([c not in hold for c in cfg])


def evaluate(model: CostModel, cfg, X, y, ids, top_k: int = 3, seed: int = 3) -> dict:
    """Quality on configurations ``ids`` using the corpus timings: best of the model's top-k vs the
    exhaustive best, against (a) k random candidates and (b) the first k candidates in sweep order
    (the method without a model, given the same timing budget)."""
    rng = np.random.default_rng(seed)
    ratios, rnd, first, within = [], [], [], 0
    for c in ids:
        sel = cfg == c
        g = np.exp(y[sel])
        best = g.max()
        pred = model.predict(X[sel])
        top = np.argsort(-pred)[:top_k]
        r = g[top].max() / best
        ratios.append(r)
        within += r >= 0.95
        rnd.append(np.mean([g[rng.choice(len(g), size=min(top_k, len(g)), replace=False)].max() / best
                            for _ in range(20)]))
        first.append(g[:top_k].max() / best)
    n = max(1, len(ids))
    return {"configs": len(ids), "top_k": top_k, "mean_ratio_to_best": float(np.mean(ratios)),
            "within_5pct": within / n, "min_ratio": float(np.min(ratios)),
            "random_k_mean_ratio": float(np.mean(rnd)), "first_k_mean_ratio": float(np.mean(first)),
            "timed_fraction": top_k / float(np.mean([np.sum(cfg == c) for c in ids]))}


def live(model: CostModel, ids, n_configs: int = 400, seed: int = 7, log=print, space: str = "pow2") -> dict:
    """Tune held-out parameter sets on the GPU twice -- the learned tuner (model top-5, fallback)
    and the exhaustive sweep, both over the candidate space `space` -- and compare the chosen
    blocks re-timed with 10 sweeps each, and the wall time each method spent."""
    import torch

    specs = sample_configs(n_configs, seed)
    tuner = Autotuner(model, space=space)
    rows = []
    for cid in ids:
        spec = specs[int(cid)]
        geom = spec.geometry(*corpus_grid(spec))
        st = Stencil(spec)
        if spec.coefficients == "Variable":
            st.copy_mask(np.random.default_rng(int(cid)).standard_normal(spec.stencil_size) / spec.stencil_size)
        x, y = _alloc(spec, geom, int(cid))
        learned = tuner.tune(st, geom, x, y)
        full = Autotuner(None, space=space).tune(st, geom, x, y)
        g_l = time_block(st, geom, x, y, learned.block, 10)
        g_f = time_block(st, geom, x, y, full.block, 10)
        rows.append({"config": int(cid), "spec": _spec_str(spec), "learned_block": list(learned.block),
                     "exhaustive_block": list(full.block), "ratio": g_l / g_f, "learned_s": learned.seconds,
                     "exhaustive_s": full.seconds, "fell_back": learned.fell_back, "reason": learned.reason,
                     "timed": learned.timed, "candidates": full.timed})
        log(json.dumps(rows[-1]))
        st.close()
        del x, y
        torch.cuda.empty_cache()
    r = np.array([q["ratio"] for q in rows])
    return {"configs": len(rows), "mean_ratio": float(r.mean()), "min_ratio": float(r.min()),
            "within_5pct": float(np.mean(r >= 0.95)),
            "time_fraction": float(sum(q["learned_s"] for q in rows) / sum(q["exhaustive_s"] for q in rows)),
            "fallbacks": int(sum(q["fell_back"] for q in rows))}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m threadcoarsenedstencilgenerator_b200.autotune")
    sub = ap.add_subparsers(dest="cmd", required=True)
    c = sub.add_parser("corpus", help="time every candidate block of sampled parameter sets (GPU)")
    c.add_argument("--configs", type=int, default=400)
    c.add_argument("--seed", type=int, default=7)
    c.add_argument("--start", type=int, default=0)
    c.add_argument("--out", type=Path, default=CORPUS_PATH)
    c.add_argument("--budget", type=float, default=None, help="stop after this many seconds")
    c.add_argument("--precompile", action="store_true", help="only instantiate the kernels (NVRTC, no GPU)")
    t = sub.add_parser("train", help="train the cost model on the corpus (GPU)")
    t.add_argument("--corpus", type=Path, default=CORPUS_PATH)
    t.add_argument("--out", type=Path, default=MODEL_PATH)
    t.add_argument("--epochs", type=int, default=150)
    e = sub.add_parser("evaluate", help="held-out quality of the trained model (GPU)")
    e.add_argument("--corpus", type=Path, default=CORPUS_PATH)
    e.add_argument("--model", type=Path, default=MODEL_PATH)
    e.add_argument("--live", type=int, default=0, help="also tune this many held-out sets live on the GPU")
    e.add_argument("--space", default="pow2", choices=["pow2", "reference"],
                   help="live candidate blocks: power-of-two shapes or the reference's whole enumeration")
    a = ap.parse_args(argv)
    if a.cmd == "corpus":
        if a.precompile:
            import multiprocessing as mp
            import os

            from .stencil import precompile

            specs = sample_configs(a.configs, a.seed)
            # NVRTC compiles one program at a time per process: use processes
            with mp.get_context("spawn").Pool(os.cpu_count() or 4) as pool:
                pool.map(precompile, specs, chunksize=1)
            print("precompiled %d parameter sets" % len(specs))
            return 0
        print(json.dumps(build_corpus(a.configs, a.seed, a.out, start=a.start, time_budget_s=a.budget)))
        return 0
    cfg, X, y = load_corpus(a.corpus if a.cmd == "train" else a.corpus)
    hold, train_mask = split(cfg)
    if a.cmd == "train":
        m = CostModel()
        t0 = time.perf_counter()
        hist = m.fit(X[train_mask], y[train_mask], groups=cfg[train_mask], epochs=a.epochs, log=print)
        dt = time.perf_counter() - t0
        m.save(a.out, epochs=a.epochs, train_seconds=dt, final_loss=hist[-1], holdout=hold)
        print(json.dumps({"train_seconds": dt, "final_loss": hist[-1], **evaluate(m, cfg, X, y, hold)}))
        return 0
    m = CostModel.load(a.model)
    out = {"corpus": evaluate(m, cfg, X, y, hold)}
    if a.live:
        out["live"] = live(m, hold[:a.live], space=a.space)
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
