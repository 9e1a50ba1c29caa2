"""The ensemble batch-size autotuner's host logic (no GPU): every candidate
steps every member exactly once per timed step, in consecutive batches of
that size; rates add up over the batches; the fastest candidate is chosen;
candidates above the member count are skipped."""
import numpy as np
import pytest

from hydra_b200 import ensemble_tune as et


class FakeEnsemble:
    made = []

    def __init__(self, n, members, **kw):
        self.members = members
        FakeEnsemble.made.append(members)

    def initialise_members(self, fields, levels):
        assert len(fields) == self.members == len(levels)

    def step(self, k):
        pass

    def close(self):
        pass


def test_tuner_covers_every_member_and_picks_the_fastest(monkeypatch):
    monkeypatch.setattr(et, "CaslEnsemble", FakeEnsemble)
    FakeEnsemble.made = []
    fields = [np.zeros((16, 16)) for _ in range(100)]
    levels = [20] * 100

    def timer(e, k):
        # per-member cost falls with the batch up to 64 members, then rises
        per = 1.0 + abs(e.members - 64) / 64.0
        return per * e.members * k, 1000.0 * e.members * k

    rates, best = et.tune_batch(fields, levels, candidates=(16, 32, 64, 128), steps=3, timer=timer)
    assert set(rates) == {16, 32, 64}          # 128 > 100 members: skipped
    assert best == 64
    # batches of 16: 6 of 16 and one of 4; of 32: 3 of 32 and one of 4; of 64: 64 + 36
    assert FakeEnsemble.made == [16] * 6 + [4] + [32] * 3 + [4] + [64, 36]


def test_tuner_refuses_when_nothing_fits(monkeypatch):
    monkeypatch.setattr(et, "CaslEnsemble", FakeEnsemble)
    with pytest.raises(ValueError):
        et.tune_batch([np.zeros((16, 16))] * 4, [20] * 4, candidates=(8, 16),
                      timer=lambda e, k: (1.0, 1.0))
