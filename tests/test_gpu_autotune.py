"""Strip-length autotuner of the streaming stage kernel (GPU).

``LaunchOptions(autotune=True)`` times one RK4 step of every streaming
launch group for each candidate strip length at batch build and keeps the
fastest.  Strips only decide which CTA streams which radial rows, and every
row gets the same sums in the same order, so the evolved states must be
bit-identical for the tuned, the built-in and any forced strip length.
"""
from dataclasses import replace

import numpy as np
import pytest

import teuk_b200 as tb
from cases import CASES, pulse_for, step_size

pytestmark = pytest.mark.gpu

CANDIDATES = {64, 96, 128, 192, 256, 384, 512, 768, 1024, 1536, 2048, 4096}


def _configs():
    base = replace(CASES["kerr_d105"], radial_points=300)
    return [base,
            replace(base, radial_points=1025, spin=0.5),
            replace(base, radial_points=777, spin=0.9, ell_max_first=12,
                    ell_max_second=12),
            replace(CASES["schw_d84"], radial_points=513, dissipation=0.002)]


def _run(options):
    configs = _configs()
    batch = tb.Batch(configs, options)
    for i, c in enumerate(configs):
        batch.initialize_gaussian(i, pulse_for(c, 41 + i))
    batch.step([step_size(c, 0.1) for c in configs], 6)
    states = [batch.get_state(i) for i in range(len(configs))]
    return batch, states


def test_tuned_strips_give_bit_identical_states(require_gpu):
    tuned, a = _run(tb.LaunchOptions(autotune=True))
    rows = tuned.strip_rows()
    streaming = [r for r in rows if r > 0]
    assert streaming and all(r in CANDIDATES for r in streaming), rows
    default, b = _run(None)
    forced, c = _run(tb.LaunchOptions(strip_rows=64))
    assert all(r == 64 for r in forced.strip_rows() if r > 0)
    for i in range(len(a)):
        assert np.array_equal(a[i], b[i]), i
        assert np.array_equal(a[i], c[i]), i


def test_tuned_choice_is_cached_and_reused(require_gpu):
    first, _ = _run(tb.LaunchOptions(autotune=True))
    second, _ = _run(tb.LaunchOptions(autotune=True))
    assert first.strip_rows() == second.strip_rows()
