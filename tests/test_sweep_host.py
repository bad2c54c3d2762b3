"""Host-side planning of the partial-wave sweep: size classes, merges, memory splits."""

from __future__ import annotations

from pyticc_b200.propagation.sweep import class_channels, plan_launches, size_class


def test_size_classes():
    assert [size_class(n, "inelastic") for n in (1, 64, 65, 128, 129, 1984)] == [64, 64, 128, 128, 256, 2048]
    assert [size_class(n, "capture") for n in (32, 33, 64, 65)] == [64, 128, 128, 256]
    assert class_channels(256, "inelastic") == 256 and class_channels(256, "capture") == 128


def test_empty_blocks_are_skipped_and_classes_kept_apart():
    sizes = [0, 10, 100, 120, 300, 0, 60]
    plans = plan_launches(sizes, "inelastic", {}, lambda n, count: count, budget=1e9)
    assert sorted(i for p in plans for i in p.members) == [1, 2, 3, 4, 6]
    by_n = {p.n: sorted(p.members) for p in plans}
    assert by_n == {64: [1, 6], 128: [2, 3], 384: [4]}


def test_merged_classes_run_padded_in_the_next_class():
    sizes = [10, 100, 300]
    plans = plan_launches(sizes, "inelastic", {64: True, 128: True}, lambda n, count: count, budget=1e9)
    assert len(plans) == 1 and plans[0].n == 384 and sorted(plans[0].members) == [0, 1, 2]
    plans = plan_launches(sizes, "inelastic", {64: True}, lambda n, count: count, budget=1e9)
    assert {p.n: sorted(p.members) for p in plans} == {128: [0, 1], 384: [2]}


def test_launches_split_at_the_memory_budget():
    sizes = [100] * 7
    plans = plan_launches(sizes, "inelastic", {}, lambda n, count: 10 * count, budget=30)
    assert [len(p.members) for p in plans] == [3, 3, 1]
    assert sorted(i for p in plans for i in p.members) == list(range(7))
