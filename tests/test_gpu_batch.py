"""Batched solves (GPU): every instance of an uneven batch evolves exactly
as the same solve alone, with or without CUDA-graph replay, and the batched
endpoint gather equals each instance's own waveform records."""
import numpy as np
import pytest

import teuk_b200 as tb
from cases import CASES, pulse_for, relative_error, step_size

pytestmark = pytest.mark.gpu


def _uneven_configs():
    base = CASES["kerr_d105"]
    spun = tb.SolveConfig(**{**base.__dict__, "spin": 0.31,
                             "radial_points": 130})
    return [CASES["schw_d84"], base, CASES["kerr_d42_sc"], CASES["nonparent"],
            spun]


def test_batch_instances_equal_solo(require_gpu):
    configs = _uneven_configs()
    batch = tb.Batch(configs)
    dts = [step_size(c) for c in configs]
    solos = []
    for i, c in enumerate(configs):
        pulse = pulse_for(c, 100 + i)
        batch.initialize_gaussian(i, pulse)
        solo = tb.Pipeline(c)
        solo.initialize_gaussian(pulse)
        solos.append(solo)
    batch.step(dts, steps=12, graph=True)
    for i, (c, solo) in enumerate(zip(configs, solos)):
        solo.step(0.0, dts[i], 12)
        assert np.array_equal(batch.get_state(i), solo.get_state()), i


def test_graph_replay_equals_eager(require_gpu):
    configs = _uneven_configs()
    a, b = tb.Batch(configs), tb.Batch(configs)
    for i, c in enumerate(configs):
        pulse = pulse_for(c, 200 + i)
        a.initialize_gaussian(i, pulse)
        b.initialize_gaussian(i, pulse)
    dts = [step_size(c) for c in configs]
    a.step(dts, steps=7, graph=True)
    b.step(dts, steps=7, graph=False)
    for i in range(len(configs)):
        assert np.array_equal(a.get_state(i), b.get_state(i))


def test_batched_endpoint_gather(require_gpu):
    configs = _uneven_configs()
    batch = tb.Batch(configs)
    for i, c in enumerate(configs):
        batch.initialize_gaussian(i, pulse_for(c, 300 + i))
    batch.step([step_size(c) for c in configs], steps=3)
    gathered = batch.endpoint_modal()
    assert gathered.size == batch.endpoint_modal_count()
    assert np.all(np.isfinite(gathered))
    # each instance's first-order scri records appear in the gather
    for i in range(len(configs)):
        records = [r for r in batch.sample_endpoint(i)
                   if r["order"] == 1 and r["boundary"] == "scri"]
        values = np.array([r["rescaled"] for r in records])
        for v in values:
            assert np.min(np.abs(gathered - v)) == 0.0


def test_launch_accounting(require_gpu):
    batch = tb.Batch(_uneven_configs())
    # one launch per RK stage per (discretization, reduction) group
    assert batch.launches_per_step() == 4 * 3
