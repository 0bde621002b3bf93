"""Scene groups of the batched build (host logic, no GPU): a batch of 8M
triangles or more is built as two groups of whole scenes, the first holding
about 30 % of the triangles, so its short upload starts the first build
while the rest crosses PCIe; smaller batches stay one group;
RTB200_BATCH_GROUPS overrides the count (clamped to 1..8 and to the number
of scenes), each group keeping at least one scene."""
import numpy as np
import pytest

from rtb200 import lib, scenes


def _offsets(sizes):
    return np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)


def test_the_256_scene_workload_splits_at_thirty_percent(monkeypatch):
    monkeypatch.delenv("RTB200_BATCH_GROUPS", raising=False)
    ntri, _ = scenes.batched_sizes()
    off = _offsets(ntri)
    assert off[-1] >= 8 << 20
    b = lib.batch_groups(off)
    assert len(b) == 3 and b[0] == 0 and b[2] == len(ntri)
    k = b[1]
    # the first scene boundary at or past 30 % of the triangles
    assert off[k] >= 0.3 * off[-1] > off[k - 1]


def test_small_batches_and_single_scenes_stay_one_group(monkeypatch):
    monkeypatch.delenv("RTB200_BATCH_GROUPS", raising=False)
    assert lib.batch_groups(_offsets([1000, 5000, 70000])) == [0, 3]
    assert lib.batch_groups(_offsets([9 << 20])) == [0, 1]


@pytest.mark.parametrize("forced, scenes_n, expect", [("4", 40, 4), ("1", 40, 1), ("0", 40, 1), ("12", 40, 8),
                                                       ("8", 3, 3), ("3", 3, 3)])
def test_forced_group_counts(monkeypatch, forced, scenes_n, expect):
    monkeypatch.setenv("RTB200_BATCH_GROUPS", forced)
    rng = np.random.default_rng(int(forced) * 100 + scenes_n)
    sizes = rng.integers(1, 50_000, scenes_n)
    b = lib.batch_groups(_offsets(sizes))
    assert len(b) == expect + 1 and b[0] == 0 and b[-1] == scenes_n
    assert all(x < y for x, y in zip(b, b[1:]))  # every group holds a scene


def test_bad_offsets_are_rejected():
    with pytest.raises(lib.RtError):
        lib.batch_groups(np.array([0, 5, 5, 9], np.int32))  # an empty scene
    with pytest.raises(lib.RtError):
        lib.batch_groups(np.array([1, 5], np.int32))  # not starting at 0
