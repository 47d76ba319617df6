"""Continuous batching server (GPU).

A request's waveform must not depend on what else shares the batched step:
each result is compared with the same solve run alone through the
single-pipeline calls (1e-12 relative: mixing solves of other shapes changes
the zero padding of the transform tiles, which may reorder a few FP64 sums),
while requests arrive during the run, wait for memory, and leave at
different times.  Second-order (quadratic-source) requests run their own
nodal pipelines beside the batch in every server step; their records must
equal the same solve alone bit for bit (nothing they compute depends on the
mix).
"""

import numpy as np
import pytest

import teuk_b200 as tb
from cases import CASES, pulse_for, relative_error, step_size

pytestmark = pytest.mark.gpu

TOL = 1e-12

SECOND_ORDER = {
    "so_unrestricted_d84": tb.SolveConfig(
        mass=1.0, spin=0.7, compactification_length=1.2, radial_points=48,
        theta_nodes=9, ell_max_first=4, ell_max_second=8,
        modes=(-4, -2, 0, 2, 4), parents=(-2, 2), targets=(-4, 0, 4),
        dissipation=0.003, discretization=tb.D84,
        source_mode=tb.SOURCE_UNRESTRICTED, source_start_time=0.0),
    "so_constraint_d42": tb.SolveConfig(
        mass=1.0, spin=0.5, compactification_length=1.5, radial_points=40,
        theta_nodes=10, ell_max_first=4, ell_max_second=6,
        modes=(-4, -3, -2, -1, 0, 1, 2, 3, 4), parents=(-2, -1, 1, 2),
        targets=(-3, -2, -1, 0, 1, 2, 3), dissipation=0.01,
        discretization=tb.D42, reduction=tb.STAGE_CONSTRAINED,
        source_mode=tb.SOURCE_CONSTRAINT_AWARE,
        normalized_constraint_tolerance=1e30, required_consecutive_passes=2),
}

# near-extremal linear solve with bands on the wide streaming kernel
# (ell <= 24, 37 nodes)
WIDE = {
    "kerr_wide": tb.SolveConfig(
        mass=1.0, spin=0.99, compactification_length=1.0, radial_points=160,
        theta_nodes=37, ell_max_first=24, ell_max_second=24,
        modes=(-2, -1, 0, 1, 2), dissipation=0.005, discretization=tb.D105),
}

# linear solves of different shapes, discretizations and reductions
MIX = [
    ("kerr_d105", 7, 12),
    ("schw_d84", 8, 20),
    ("kerr_d42_sc", 9, 9),
    ("nonparent", 10, 15),
    ("kerr_d105", 11, 5),
    ("so_unrestricted_d84", 12, 6),
    ("so_constraint_d42", 13, 4),
    ("kerr_wide", 14, 7),
]


def test_second_order_requests_match_alone_exactly(require_gpu):
    """Only second-order requests: every record bit-identical to the solve
    run alone (the nodal pipelines do not share buffers or launches)."""
    server = tb.Server(hbm_budget_bytes=8 << 30)
    jobs = []
    for name, seed, steps in (("so_unrestricted_d84", 3, 5),
                              ("so_constraint_d42", 4, 3)):
        config = SECOND_ORDER[name]
        pulse = pulse_for(config, seed)
        dt = step_size(config)
        jobs.append((server.submit(config, pulse, dt, steps), config, pulse,
                     dt, steps))
    while server.advance(2) > 0:
        pass
    for rid, config, pulse, dt, steps in jobs:
        records, _ = server.result(rid)
        alone = _alone(config, pulse, dt, steps)
        assert _keys(records) == _keys(alone)
        assert np.array_equal(_values(records), _values(alone))


def _config(name):
    for table in (CASES, SECOND_ORDER, WIDE):
        if name in table:
            return table[name]
    raise KeyError(name)


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
        config = _config(name)
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
    with pytest.raises(tb.InvalidArgument, match="finite positive"):
        big.submit(config, pulse_for(config, 1), 0.0, 2)
    with pytest.raises(tb.InvalidArgument, match="unknown request id"):
        big.result(12345)


def test_split_precision_server_matches_split_alone(require_gpu):
    """A split-precision server: every request's records equal the same
    solve run alone with split-precision transforms (second-order requests
    bit for bit, linear ones to 1e-12 as above)."""
    split = tb.LaunchOptions(precision=tb.PRECISION_SPLIT)
    server = tb.Server(hbm_budget_bytes=8 << 30, precision=tb.PRECISION_SPLIT)
    jobs = []
    for i, (name, seed, steps) in enumerate([("kerr_d105", 21, 6),
                                             ("so_unrestricted_d84", 22, 4),
                                             ("nonparent", 23, 5)]):
        config = _config(name)
        pulse = pulse_for(config, seed)
        dt = step_size(config)
        jobs.append((server.submit(config, pulse, dt, steps), config, pulse,
                     dt, steps))
        server.advance(2)
    while server.advance(3) > 0:
        pass
    for rid, config, pulse, dt, steps in jobs:
        records, _ = server.result(rid)
        p = tb.Pipeline(config, split)
        p.initialize_gaussian(pulse)
        p.step(0.0, dt, steps)
        alone = p.sample_endpoint()
        if config.source_mode != tb.SOURCE_DISABLED:
            assert _keys(records) == _keys(alone)
            assert np.array_equal(_values(records), _values(alone))
        else:
            _check_same(records, alone)


def test_replicated_second_order_requests_match_alone_exactly(require_gpu):
    """Same-configuration Unrestricted requests share one replicated nodal
    pipeline: members join while others run (the pipeline's room grows from
    two to four replicas, moving the members' states on the device), leave
    at different steps (the last replica moves into the freed slot), and
    every record equals the solve alone bit for bit."""
    config = SECOND_ORDER["so_unrestricted_d84"]
    dt = step_size(config)
    server = tb.Server(hbm_budget_bytes=8 << 30)
    plan = [(31, 7), (32, 3), (33, 5), (34, 2), (35, 6)]
    jobs = []
    for i, (seed, steps) in enumerate(plan):
        pulse = pulse_for(config, seed)
        jobs.append((server.submit(config, pulse, dt, steps), pulse, steps))
        server.advance(1)
    while server.advance(1) > 0:
        pass
    for rid, pulse, steps in jobs:
        records, _ = server.result(rid)
        alone = _alone(config, pulse, dt, steps)
        assert _keys(records) == _keys(alone)
        assert np.array_equal(_values(records), _values(alone)), rid
