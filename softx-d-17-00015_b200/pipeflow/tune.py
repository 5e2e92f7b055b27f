"""Autotuner of the fused timestep's launch choices.

No counterpart in the reference: its only tuning is FFTW's own plan search
(FFTW_PATIENT, transform.fftw3.f90:36-57), which picks radices per transform
length.  Here the choices are those pf_ctx_set_tuning exposes:

  ld_solver  the banded solves stream the stored LU factors from HBM
             (PF_LD_STREAMED), share the Helmholtz rings of a mode between
             its real and imaginary lanes (PF_LD_WARPRING), pair the modes k
             and -k on one factor stream (PF_LD_PAIRED), or rebuild the
             Helmholtz factors on chip (PF_LD_REBUILT, for factorisations
             that did not pivot);
  nl_fused   in mixed precision, the three-pass transforms (0) or those of
             one radial point in one block (1);
  nl_mc      columns (azimuthal modes m) per block of the z transform passes
             (not timed where one block per radial point runs);
  nl_zc      z rows per block of the theta pass (two rows per complex FFT;
             the candidates include the tiles whose rows fill the passes of
             the four-step row transform);
  worklist   (a batch as a whole) the transform stages as one launch per
             stage and transform length, or one persistent launch per stage
             over a work list of every pipe's tiles (pf_batch_set_worklist).

Every choice gives the same numbers bit for bit, so the tuner only times
them.  A candidate replaces a knob's current choice only when it is faster by
more than a margin (0.5% by default), so timing noise does not move choices.  It times timesteps in the steporbit form (exactly one corrector per
step, so every candidate does the same work), by coordinate descent: the
solver first, then the z tile, then the theta tile, each with the others
held (then the transform form, then the tiles).  A pipe is tuned on its own; a batch is tuned shape by shape (pipes of
one (N, K, M, Mp, precision) share a choice) while the whole batch steps,
since the kernels of different shapes share the GPU, and then the form of its
transform stages.  Choices are cached in
a JSON file (PIPEFLOW_TUNE_CACHE, default ~/.cache/pipeflow_b200/tuning.json)
keyed by the pipe shape, or by the batch's shape multiset.

The tuner advances the flow while it times; it restores every pipe's state
and time-stepping counters afterwards.
"""
from __future__ import annotations

import json
import os
import time
from pathlib import Path

from . import _lib as L
from .api import PipeflowError

ZC_CANDIDATES = (0, 4, 8, 16, 32)
LD_CANDIDATES = (L.PF_LD_AUTO, L.PF_LD_WARPRING, L.PF_LD_REBUILT, L.PF_LD_PAIRED)
KNOBS = ("ld_solver", "nl_fused", "nl_mc", "nl_zc")
DEFAULT = {"ld_solver": L.PF_LD_AUTO, "nl_mc": 0, "nl_zc": 0, "nl_fused": 0}
WORKLIST_KEY = "batch"  # batch-wide choices in a batch's cache entry


def _candidates(knob: str, shape) -> tuple:
    if knob == "ld_solver":
        return LD_CANDIDATES
    if knob == "nl_fused":
        return (0, 1) if shape[4] == L.PF_PREC_MIXED else (0,)
    if knob == "nl_mc":
        return tuple(_mc_candidates(shape[2]))
    return _zc_candidates(3 * shape[2])


def _fft4_l1(L: int) -> int:
    """The first factor of the four-step split of a length-L row FFT (the
    kernels' fft4_l1): L itself up to 32, else the largest divisor d with
    d * d <= L and L / d <= 32."""
    if L <= 32:
        return L
    best = 0
    for d in range(1, 33):
        if L % d == 0 and L // d <= 32 and (best == 0 or (d * d <= L and d > best) or (best * best > L and d < best)):
            best = d
    return best


def _zc_candidates(Th: int) -> tuple:
    """Theta-pass tiles to time: the fixed set, plus the even tiles whose
    3 * ZC complex rows fill one, two or three passes of the four-step
    transform's two steps (a 256-thread block takes 256 // L2 rows at a time
    in the first step and 256 // L1 in the second), so no pass runs part-empty."""
    out = set(ZC_CANDIDATES)
    L1 = _fft4_l1(Th)
    per_pass = {256 // (Th // L1), 256 // L1} if L1 < Th else {256}
    for per in per_pass:
        for passes in (1, 2, 3):
            zc = (per * passes // 3) // 2 * 2
            if 2 <= zc <= 32:
                out.add(zc)
    return tuple(sorted(out))


def _fused_applies(pipe, cur: dict) -> bool:
    """Whether asking for one block per radial point changes anything for
    this pipe (mixed precision, a built (Z, Th) pair, a plane that fits)."""
    if not hasattr(pipe, "nl_passes"):
        return True
    pipe.set_tuning(**dict(cur, nl_fused=1))
    ok = pipe.nl_passes == 1
    pipe.set_tuning(**cur)
    return ok


def _one_pass(pipe) -> bool:
    """Whether the pipe's nonlinear terms run as one block per radial point
    with its current choices (the z-pass tile is then unused)."""
    return getattr(pipe, "nl_passes", 3) == 1


def _mc_candidates(M: int):
    out = {0, M}
    for d in (2, 3, 4, 6, 8):
        out.add(max(1, -(-M // d)))
    return sorted(out)


def shape_of(pipe) -> tuple:
    return (pipe.N, pipe.K, pipe.M, pipe.Mp, int(getattr(pipe.cfg, "precision", 0)))


def _shape_key(shape) -> str:
    N, K, M, Mp, prec = shape
    return f"N{N}K{K}M{M}Mp{Mp}{'mixed' if prec == L.PF_PREC_MIXED else 'fp64'}"


def default_cache_path() -> Path:
    env = os.environ.get("PIPEFLOW_TUNE_CACHE")
    if env:
        return Path(env)
    return Path.home() / ".cache" / "pipeflow_b200" / "tuning.json"


class _Snapshot:
    """Host copies of pipes' states and time-stepping counters."""

    def __init__(self, pipes):
        self.items = [(p, p.get_state(), p.tim) for p in pipes]

    def restore(self):
        for p, st, tim in self.items:
            p.set_state(*st)
            p.set_tim(tim)


class Tuner:
    def __init__(self, cache_path=None, steps: int = 6, reps: int = 2, use_cache: bool = True,
                 margin: float = 0.005):
        self.cache_path = Path(cache_path) if cache_path else default_cache_path()
        self.steps = steps
        self.reps = reps
        self.use_cache = use_cache
        # a candidate replaces the first option of a knob (the current choice)
        # only when it is faster by more than this fraction: one shape's choice
        # moves a batch step by well under a percent, about the timing noise
        self.margin = margin
        self.log = []  # (what, choice, seconds) of every timing taken

    # ------------------------------------------------------------ cache
    def _load(self) -> dict:
        try:
            return json.loads(self.cache_path.read_text())
        except (OSError, ValueError):
            return {}

    def _store(self, key: str, value) -> None:
        data = self._load()
        data[key] = value
        try:
            self.cache_path.parent.mkdir(parents=True, exist_ok=True)
            tmp = self.cache_path.with_suffix(".tmp")
            tmp.write_text(json.dumps(data, indent=1, sort_keys=True))
            tmp.replace(self.cache_path)
        except OSError:
            pass  # a read-only home is not an error: the choice still applies

    # ---------------------------------------------------------- timing
    def _best(self, options, apply, run):
        """Apply each option, time run() (min over reps), keep the fastest;
        the first option that runs stays unless another beats it by more
        than the margin."""
        best, best_t, first_t = None, float("inf"), None
        for opt in options:
            try:
                apply(opt)
            except PipeflowError:  # a tile over the shared-memory cap
                continue
            t = min(run() for _ in range(self.reps))
            self.log.append((opt, t))
            if first_t is None:
                best, best_t, first_t = opt, t, t
            elif t < best_t and t < first_t * (1.0 - self.margin):
                best, best_t = opt, t
        apply(best)
        return best, best_t

    # ------------------------------------------------------------ a pipe
    def tune_pipe(self, pipe) -> dict:
        """Choose the launch choices of one pipe by timing it alone."""
        key = "pipe:" + _shape_key(shape_of(pipe))
        if self.use_cache:
            hit = self._load().get(key)
            if hit:
                pipe.set_tuning(**hit)
                return hit
        snap = _Snapshot([pipe])
        cur = dict(DEFAULT)

        def run():
            pipe.steporbit(2)
            pipe.sync()
            t0 = time.perf_counter()
            pipe.steporbit(self.steps)
            pipe.sync()
            return time.perf_counter() - t0

        for knob in KNOBS:
            if (knob == "nl_mc" and _one_pass(pipe)) or (knob == "nl_fused" and not _fused_applies(pipe, cur)):
                continue
            def apply(v, knob=knob):
                pipe.set_tuning(**dict(cur, **{knob: v}))
                cur[knob] = v
            self._best(_candidates(knob, shape_of(pipe)), apply, run)
        snap.restore()
        self._store(key, dict(cur))
        return dict(cur)

    # ----------------------------------------------------------- a batch
    def tune_batch(self, batch) -> dict:
        """Choose the launch choices of every pipe shape of a batch by timing
        whole batch steps; returns {shape key: choice}."""
        shapes = {}
        for p in batch.pipes:
            shapes.setdefault(shape_of(p), []).append(p)
        sig = "batch:" + ",".join(f"{_shape_key(s)}x{len(v)}" for s, v in sorted(shapes.items()))
        if self.use_cache:
            hit = self._load().get(sig)
            if hit and set(hit) - {WORKLIST_KEY} == {_shape_key(s) for s in shapes}:
                for s, pipes in shapes.items():
                    for p in pipes:
                        p.set_tuning(**hit[_shape_key(s)])
                if WORKLIST_KEY in hit and hasattr(batch, "set_worklist"):
                    batch.set_worklist(bool(hit[WORKLIST_KEY]["worklist"]))
                return hit
        snap = _Snapshot(batch.pipes)
        choice = {s: dict(DEFAULT) for s in shapes}

        def run():
            batch.step(3, orbit=True)  # rebuild after a change: direct step, capture, replay
            batch.sync()
            t0 = time.perf_counter()
            batch.step(self.steps, orbit=True)
            batch.sync()
            return time.perf_counter() - t0

        # largest shapes first: they carry most of the step
        order = sorted(shapes, key=lambda s: -s[0] * s[1] * s[2] * len(shapes[s]))
        for knob in KNOBS:
            for s in order:
                if knob == "nl_mc" and _one_pass(shapes[s][0]):
                    continue
                if knob == "nl_fused" and not _fused_applies(shapes[s][0], choice[s]):
                    continue
                values = _candidates(knob, s)

                def apply(v, s=s, knob=knob):
                    new = dict(choice[s], **{knob: v})
                    for p in shapes[s]:
                        p.set_tuning(**new)
                    choice[s] = new
                self._best(values, apply, run)
        # the batch-wide form of the transform stages, with every shape's
        # choices held: per-length launches or one work-list launch per stage
        if hasattr(batch, "set_worklist"):
            self._best((False, True), batch.set_worklist, run)
        snap.restore()
        out = {_shape_key(s): c for s, c in choice.items()}
        if hasattr(batch, "set_worklist"):
            out[WORKLIST_KEY] = {"worklist": int(batch.worklist)}
        self._store(sig, out)
        return out
