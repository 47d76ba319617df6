"""Continuous batching server (GPU).

A request's waveform must not depend on what else shares the batched step:
each result is compared with the same solve run alone through the
single-pipeline calls (1e-12 relative: mixing solves of other shapes changes
the zero padding of the transform tiles, which may reorder a few FP64 sums),
while requests arrive during the run, wait for memory, and leave at
different times.
"""
import dataclasses

import numpy as np
import pytest

import teuk_b200 as tb
from cases import CASES, pulse_for, relative_error, step_size

pytestmark = pytest.mark.gpu

TOL = 1e-12

# linear solves of different shapes, discretizations and reductions
MIX = [
    ("kerr_d105", 7, 12),
    ("schw_d84", 8, 20),
    ("kerr_d42_sc", 9, 9),
    ("nonparent", 10, 15),
    ("kerr_d105", 11, 5),
]


def _alone(config, pulse, dt, steps):
    p = tb.Pipeline(config)
    p.initialize_gaussian(pulse)
    p.step(0.0, dt, steps)
    return p.sample_endpoint()


def _values(records):
    return np.array([r["endpoint"] for r in records])


def _keys(records):
    return [(r["boundary"], r["order"], r["m"], r["ell"]) for r in records]


def _check_same(records, alone):
    assert _keys(records) == _keys(alone)
    assert relative_error(_values(records), _values(alone)) < TOL


def test_results_in_the_mix_match_results_alone(require_gpu):
    server = tb.Server(hbm_budget_bytes=8 << 30)
    jobs = []
    # two requests up front, the rest arrive while the batch is running
    for i, (name, seed, steps) in enumerate(MIX):
        config = CASES[name]
        pulse = pulse_for(config, seed)
        dt = step_size(config)
        rid = server.submit(config, pulse, dt, steps)
        jobs.append((rid, config, pulse, dt, steps))
        if i >= 1:
            server.advance(3)
    while server.advance(4) > 0:
        pass
    st = server.stats()
    assert st.finished == len(MIX) and st.active == 0 and st.queued == 0
    expected_updates = sum(
        steps * len(c.modes) * c.radial_points * c.theta_nodes
        for _, c, _, _, steps in jobs)
    assert st.grid_point_updates == expected_updates
    for rid, config, pulse, dt, steps in jobs:
        records, latency = server.result(rid)
        assert latency > 0.0
        _check_same(records, _alone(config, pulse, dt, steps))


def test_budget_admits_one_solve_at_a_time(require_gpu):
    config = CASES["kerr_d105"]
    one = tb.footprint_bytes(config)
    server = tb.Server(hbm_budget_bytes=one + one // 2)
    dt = step_size(config)
    ids = [server.submit(config, pulse_for(config, s), dt, 4) for s in (1, 2, 3)]
    active = server.advance(1)
    assert active == 1 and server.stats().queued == 2
    with pytest.raises(tb.InvalidArgument, match="not finished"):
        server.result(ids[2])
    while server.advance(2) > 0:
        pass
    for rid, seed in zip(ids, (1, 2, 3)):
        records, _ = server.result(rid)
        _check_same(records, _alone(config, pulse_for(config, seed), dt, 4))


def test_server_rejects_what_it_cannot_run(require_gpu):
    server = tb.Server(hbm_budget_bytes=1 << 20)
    config = CASES["kerr_d105"]
    with pytest.raises(tb.InvalidArgument, match="exceeds the server HBM budget"):
        server.submit(config, pulse_for(config, 1), step_size(config), 2)
    big = tb.Server(hbm_budget_bytes=8 << 30)
    second = dataclasses.replace(CASES["nonparent"],
                                 source_mode=tb.SOURCE_UNRESTRICTED)
    with pytest.raises(tb.Unsupported):
        big.submit(second, pulse_for(second, 1), step_size(second), 2)
    with pytest.raises(tb.InvalidArgument, match="unknown request id"):
        big.result(12345)
