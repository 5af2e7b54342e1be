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
