"""The ensemble autotuner's final choice among stream counts (host logic, no
GPU): the fewest streams whose step time is within 1% of the best schedule's,
other settings unchanged."""

from __future__ import annotations


def _trials(ms_by_streams, **others):
    base = dict(lw_chunk=131072, sw_chunk=262144, sw_split_max=4096, lw_split_max=2048, gemm_tile=256)
    base.update(others)
    return [dict(base, streams=s, ms=ms) for s, ms in ms_by_streams.items()]


def test_fewer_streams_within_tolerance_win(pkg):
    from wrf_jax_b200.ensemble import prefer_fewer_streams
    trials = _trials({1: 312.0, 2: 311.5, 4: 310.0})
    best = {k: v for k, v in trials[2].items() if k != "ms"}
    pick, ms = prefer_fewer_streams(best, 310.0, trials)
    assert pick["streams"] == 1 and ms == 312.0
    assert {k: v for k, v in pick.items() if k != "streams"} == {k: v for k, v in best.items() if k != "streams"}


def test_slower_fewer_streams_lose(pkg):
    from wrf_jax_b200.ensemble import prefer_fewer_streams
    trials = _trials({1: 330.0, 2: 312.0, 4: 310.0})
    best = {k: v for k, v in trials[2].items() if k != "ms"}
    pick, ms = prefer_fewer_streams(best, 310.0, trials)
    assert pick["streams"] == 2 and ms == 312.0


def test_trials_with_other_settings_are_not_candidates(pkg):
    from wrf_jax_b200.ensemble import prefer_fewer_streams
    trials = _trials({4: 310.0}) + _trials({1: 300.0}, gemm_tile=128)
    best = {k: v for k, v in trials[0].items() if k != "ms"}
    pick, ms = prefer_fewer_streams(best, 310.0, trials)
    assert pick == best and ms == 310.0
