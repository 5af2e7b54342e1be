"""Autotuner logic on the CPU: candidate tiles, the choice rule, and the
cache round trip (the measurement itself is a GPU test)."""
from anns_fhe_b200 import autotune as A
from anns_fhe_b200.driver import CkksParams


def test_chunk_candidates():
    c = A.chunk_candidates(296, 148)
    assert c == sorted(set(c)) and c[-1] == 296 and 148 in c and 37 in c
    assert all(1 <= x <= 296 for x in c)
    assert A.chunk_candidates(8, 148) == [8]
    # multiples of the one-kernel key switch's capacity (full waves of clusters)
    c = A.chunk_candidates(256, 148, capacity=32)
    assert {32, 64, 96, 128, 160, 192, 224, 256} <= set(c) and c[-1] == 256


def test_pick_prefers_fastest_then_larger_chunk_then_fused():
    t = {(True, 148): 2.0, (True, 296): 1.5, (False, 296): 1.5, (False, 148): 1.9}
    assert A.pick(t) == (True, 296)
    assert A.pick({(True, 64): 3.0, (False, 64): 2.0}) == (False, 64)
    # within the tie band the larger tile wins even if a hair slower
    assert A.pick({(True, 148): 0.78, (True, 296): 0.84, (False, 296): 1.49}) == (True, 296)
    # outside it, speed wins
    assert A.pick({(True, 148): 0.70, (True, 296): 0.84}) == (True, 148)
    # 16 values per thread only where it wins by more than SHAPE_TIE; slices by speed
    assert A.pick({(True, 296, 8, 13): 1.00, (True, 296, 16, 13): 0.98}) == (True, 296, 8, 13)
    assert A.pick({(True, 296, 8, 13): 1.00, (True, 296, 16, 13): 0.95}) == (True, 296, 16, 13)
    assert A.pick({(True, 256, 8, 13): 1.00, (True, 256, 8, 12): 0.98}) == (True, 256, 8, 12)


def test_cache_round_trip(tmp_path):
    prm = CkksParams.generate(10, 3, 40, 1, 45, 1)
    path = str(tmp_path / "t.json")
    ch = {3: A.KsChoice(True, 296, 1.25), 2: A.KsChoice(False, 148, 0.9)}
    ntt = {"plan": 1, "us_per_limb": {"0": 2.0, "1": 1.5}, "describe": {"0": "a", "1": "b"}}
    A.save(path, prm, ch, 296, ntt)
    assert A.load(path, 296) == ch
    assert A.load_full(path, 296) == (ch, ntt)
    assert A.load(path, 128) is None            # tuned for another batch size
    assert A.load(str(tmp_path / "absent.json"), 296) is None


def test_fused_crossover_picks_the_count_from_which_the_one_kernel_path_wins(monkeypatch):
    """fused_crossover: the smallest tried count from which the one-kernel key
    switch is at least as fast as the multi-kernel pipeline at every larger
    count; the context's options come back as they were."""
    from anns_fhe_b200 import _lib as L

    class Ctx:
        def __init__(self):
            self.o = {L.OPT_FUSED_MIN: 18, L.OPT_KS_FUSED: 1}

        def get_option(self, k):
            return self.o[k]

        def set_option(self, k, v):
            self.o[k] = v

    def times(one, multi):
        def t(ctx, level, count, reps=3):
            return (one if ctx.o[L.OPT_KS_FUSED] else multi)[count]
        return t
    ctx = Ctx()
    one = {1: 9.0, 2: 5.0, 4: 3.0, 8: 2.0, 16: 1.0, 32: 0.6, 64: 0.5, 128: 0.4}
    multi = {1: 4.0, 2: 3.0, 4: 2.5, 8: 2.2, 16: 2.0, 32: 2.0, 64: 2.0, 128: 2.0}
    monkeypatch.setattr(A, "time_rotations", times(one, multi))
    assert A.fused_crossover(ctx, 3, 256) == 8
    assert ctx.o == {L.OPT_FUSED_MIN: 18, L.OPT_KS_FUSED: 1}
    # a count where the one-kernel path loses again above a win does not count
    one[32] = 2.5
    assert A.fused_crossover(ctx, 3, 256) == 64
    # never faster within the lanes: beyond the largest count tried
    monkeypatch.setattr(A, "time_rotations", times({c: 9.0 for c in one}, multi))
    assert A.fused_crossover(ctx, 3, 16) == 32
    assert A.fused_crossover(ctx, 3, 1) == 2
