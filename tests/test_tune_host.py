"""Host logic of the autotuner (pipeflow/tune.py) without a GPU: candidate
tiles, shape keys, the JSON cache, and that a batch is tuned shape by shape
with the fastest candidate kept and the states restored.  The timings come
from a fake pipe whose step time depends on its launch choices."""
import json

import pipeflow as P
from pipeflow import tune as T


def test_tile_candidates_cover_the_built_in_and_the_whole_range():
    for M in (4, 12, 24, 32, 48):
        c = T._mc_candidates(M)
        assert c[0] == 0 and M in c and all(1 <= x <= M for x in c[1:])
        assert c == sorted(set(c))
    assert 0 in T.ZC_CANDIDATES and all(z % 2 == 0 for z in T.ZC_CANDIDATES)
    # the kernels' four-step split, and theta tiles that fill its passes
    assert [T._fft4_l1(L) for L in (12, 36, 72, 96, 144, 192, 288)] == [12, 6, 8, 8, 12, 12, 16]
    assert T._zc_candidates(36) == (0, 4, 8, 14, 16, 28, 32)
    for Th in (36, 48, 72, 96, 144, 192):
        c = T._zc_candidates(Th)
        assert set(T.ZC_CANDIDATES) <= set(c) and all(z % 2 == 0 and 0 <= z <= 32 for z in c)


class _Cfg:
    def __init__(self, precision):
        self.precision = precision


class FakePipe:
    """Stands in for pipeflow.Pipe: records its tuning and state, and makes
    the tuner's clock advance by a cost that depends on the tuning."""

    clock = [0.0]

    def __init__(self, N, K, M, precision, best):
        self.N, self.K, self.M, self.Mp = N, K, M, 1
        self.cfg = _Cfg(precision)
        self.best = best
        self.tuning = {"ld_solver": 0, "nl_mc": 0, "nl_zc": 0, "nl_fused": 0}
        self.state = [("s", N)]
        self.steps = 0
        self._tim = {"step": 0}

    # the parts of Pipe the tuner uses
    def set_tuning(self, ld_solver=0, nl_mc=0, nl_zc=0, nl_fused=0):
        if nl_zc % 2:
            raise P.PipeflowError(-1, "odd theta tile")
        self.tuning = {"ld_solver": ld_solver, "nl_mc": nl_mc, "nl_zc": nl_zc, "nl_fused": nl_fused}

    def cost(self):
        return sum(abs(self.tuning[k] - self.best[k]) for k in self.tuning) + 1.0

    def get_state(self):
        return list(self.state)

    def set_state(self, *st):
        self.state = list(st)

    @property
    def tim(self):
        return dict(self._tim)

    def set_tim(self, t):
        self._tim = dict(t)


class FakeBatch:
    def __init__(self, pipes):
        self.pipes = pipes

    def step(self, n, orbit=False):
        for p in self.pipes:
            p.state = [("stepped", p.N)]
            p._tim["step"] += n
        FakePipe.clock[0] += n * sum(p.cost() for p in self.pipes)

    def sync(self):
        pass


class FakeWorklistBatch(FakeBatch):
    """A batch whose work-list form of the transform stages is faster."""

    def __init__(self, pipes):
        super().__init__(pipes)
        self.worklist = False

    def set_worklist(self, on):
        self.worklist = bool(on)

    def step(self, n, orbit=False):
        super().step(n, orbit)
        if not self.worklist:
            FakePipe.clock[0] += n * 5.0


def test_batch_tuning_times_the_work_list_form_and_caches_it(tmp_path, monkeypatch):
    monkeypatch.setattr(T.time, "perf_counter", lambda: FakePipe.clock[0])
    best = {"ld_solver": P.PF_LD_AUTO, "nl_mc": 0, "nl_zc": 16, "nl_fused": 0}
    batch = FakeWorklistBatch([FakePipe(48, 32, 24, 0, best), FakePipe(48, 32, 24, 0, best)])
    cache = tmp_path / "tuning.json"
    choice = T.Tuner(cache_path=cache, steps=2, reps=1).tune_batch(batch)
    assert choice == {"N48K32M24Mp1fp64": best, "batch": {"worklist": 1}} and batch.worklist
    batch.set_worklist(False)
    again = T.Tuner(cache_path=cache, steps=2, reps=1)
    assert again.tune_batch(batch) == choice and again.log == [] and batch.worklist


def test_split_is_only_tried_in_mixed_precision_and_the_one_pass_kernel_skips_the_z_tile():
    assert T._candidates("nl_fused", (32, 16, 12, 1, P.PF_PREC_MIXED)) == (0, 1)
    assert T._candidates("nl_fused", (32, 16, 12, 1, P.PF_PREC_FP64)) == (0,)

    class OnePass:
        nl_passes = 1
    assert T._one_pass(OnePass()) and not T._one_pass(object())


def test_batch_tuning_picks_each_shapes_fastest_choice_and_caches_it(tmp_path, monkeypatch):
    monkeypatch.setattr(T.time, "perf_counter", lambda: FakePipe.clock[0])
    best_a = {"ld_solver": P.PF_LD_REBUILT, "nl_mc": 6, "nl_zc": 8, "nl_fused": 1}
    best_b = {"ld_solver": P.PF_LD_AUTO, "nl_mc": 0, "nl_zc": 16, "nl_fused": 0}
    pipes = [FakePipe(32, 16, 12, 1, best_a), FakePipe(32, 16, 12, 1, best_a), FakePipe(48, 32, 24, 0, best_b)]
    batch = FakeBatch(pipes)
    cache = tmp_path / "tuning.json"
    tuner = T.Tuner(cache_path=cache, steps=2, reps=1)
    choice = tuner.tune_batch(batch)
    assert choice == {"N32K16M12Mp1mixed": best_a, "N48K32M24Mp1fp64": best_b}
    assert [p.tuning for p in pipes] == [best_a, best_a, best_b]
    # states and counters restored after the timed steps
    assert all(p.state == [("s", p.N)] and p.tim == {"step": 0} for p in pipes)
    data = json.loads(cache.read_text())
    assert list(data.values()) == [choice]
    # a second tuner reads the cache and times nothing
    for p in pipes:
        p.set_tuning()
    again = T.Tuner(cache_path=cache, steps=2, reps=1)
    assert again.tune_batch(batch) == choice and again.log == []
    assert [p.tuning for p in pipes] == [best_a, best_a, best_b]


def test_a_candidate_within_the_margin_keeps_the_current_choice(monkeypatch):
    clock = [0.0]
    monkeypatch.setattr(T.time, "perf_counter", lambda: clock[0])
    cost = {"a": 1.000, "b": 0.998, "c": 0.90}
    chosen = []

    def apply(v):
        chosen.append(v)

    tuner = T.Tuner(cache_path="/nonexistent/tuning.json", reps=1, margin=0.005)

    def run():
        clock[0] += cost[chosen[-1]]
        return cost[chosen[-1]]

    assert tuner._best(["a", "b"], apply, run)[0] == "a"      # 0.2% faster: kept the first
    assert tuner._best(["a", "b", "c"], apply, run)[0] == "c"  # 10% faster: taken
