"""Host logic of the learned sector widths: runs, aligned merges, labels (no GPU)."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import learned as oracle
from pyticc_b200.propagation.grid import RadialSector, build_radial_sectors
from pyticc_b200.propagation.learned import N_PARAM, OPEN_PHASE_LIMIT, labels_from_errors, merge_groups, merge_sectors, sector_runs


def test_param_count_matches_the_packed_layout():
    assert N_PARAM == 1377
    assert oracle.split_params(np.zeros(N_PARAM))["W2"].shape == (32, 32)


def test_runs_split_at_intervals_and_shortened_sectors():
    sectors = build_radial_sectors([2.0, 3.0, 4.05], [0.1, 0.2])
    runs = sector_runs(sectors)
    assert runs[0] == 0 and np.all(runs[:5] == 0)
    # second interval: 1.05 / 0.4 -> two full sectors then a shortened one
    assert len(set(runs[5:7].tolist())) == 1 and runs[5] == 1 and runs[7] == 2


@pytest.mark.parametrize("seed", range(6))
def test_merge_groups_match_the_oracle_and_tile_the_grid(seed):
    rng = np.random.default_rng(seed)
    sectors = build_radial_sectors([2.0, 5.0, 9.0, 9.33], [0.01, 0.02, 0.05])
    runs = sector_runs(sectors)
    levels = rng.uniform(-1.0, 7.0, len(sectors))
    phase = rng.uniform(0.0, 0.05, len(sectors))
    for ph in (None, phase):
        ours = merge_groups(levels, runs, 6, ph)
        assert ours == oracle.merge_groups(levels, runs, 6, ph, OPEN_PHASE_LIMIT)
        covered = [s for start, m in ours for s in range(start, start + m)]
        assert covered == list(range(len(sectors)))
        for start, m in ours:
            assert runs[start] == runs[start + m - 1]
            assert m == 1 or levels[start : start + m].min() >= np.log2(m)


def test_merged_sectors_keep_their_points_on_the_grid():
    sectors = build_radial_sectors([2.5, 6.5], [0.02])
    grid = np.concatenate([[sectors[0].radial_start], [p for s in sectors for p in (s.radial_mid, s.radial_end)]])
    merged = merge_sectors(sectors, np.full(len(sectors), 3.2), 4)
    assert len(sectors) == 100 and len(merged) == 13  # 12 groups of 8, then one of 4
    for s in merged:
        for point in (s.radial_start, s.radial_mid, s.radial_end):
            assert np.abs(grid - point).min() <= 1e-12
    assert merged[-1].radial_end == sectors[-1].radial_end


def test_phase_cap_limits_the_merge():
    sectors = build_radial_sectors([0.0, 6.4], [0.1])
    merged = merge_sectors(sectors, np.full(len(sectors), 8.0), 8, np.full(len(sectors), 0.4))
    assert all(abs(s.radial_half_step / 0.1 - 4.0) < 1e-9 for s in merged)  # 8 * 0.4 >= 2.8 > 4 * 0.4


def test_labels_from_errors():
    errors = np.array([[1e-14, 1e-14, 1e-11, 1e-11], [1e-12, 1e-12, 1e-12, 1e-12], [np.nan, np.nan, np.nan, np.nan]])
    errors[1] = [1e-8, 1e-8, 1e-8, 1e-8]
    labels = labels_from_errors(errors, tol=1e-9, order=5.0)
    assert labels[0] == pytest.approx(2.0 + np.log2(1e-1) / 5.0)
    assert labels[2] == pytest.approx(min(1.0 + np.log2(1e2) / 5.0, 2.0 + np.log2(1e-1) / 5.0))
    forbidden = np.array([[1e-14], [np.inf]])
    assert labels_from_errors(forbidden)[0] == 1.0


def test_labels_take_both_bounds():
    open_block = np.array([[1e-14, 1e-10], [1e-14, 1e-8]])
    all_channels = np.array([[1e-6, 1e-14], [1e-4, 1e-14]])
    labels = labels_from_errors(np.stack([open_block, all_channels]), tol=1e-9, closed_tol=1e-5)
    assert labels[0] == pytest.approx(2.0 + np.log2(1e-1) / 5.0)  # closed bound at level 2
    assert labels[1] == pytest.approx(2.0 + np.log2(1e-1) / 5.0)  # open bound at level 2


def test_propagation_steps_are_validated():
    from pyticc_b200 import Propagation

    assert Propagation(steps="learned").steps == "learned"
    with pytest.raises(ValueError, match="steps must be 'fixed' or 'learned'"):
        Propagation(steps="adaptive")


def test_packaged_proposer_loads():
    from pyticc_b200.propagation.learned import DEFAULT_PROPOSER, StepProposer

    proposer = StepProposer.load(DEFAULT_PROPOSER)
    assert proposer.params.shape == (N_PARAM,) and proposer.params.dtype == np.float32
    assert proposer.norm.shape == (16,) and np.all(np.isfinite(proposer.params))
    assert proposer.max_level == 8 and proposer.margin == 0.5
