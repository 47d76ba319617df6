"""Device selection of the engine (GPU).

The engine carries its own CUDA runtime, so a process picks the engine's
device with ``teuk_b200_set_device``.  Launch set-up (shared-memory opt-in,
SM counts, register checks) is kept per device, so pipelines on a second
device in the same process must step like those on the first.
"""
import numpy as np
import pytest

import teuk_b200 as tb
from cases import CASES, pulse_for, step_size

pytestmark = pytest.mark.gpu


def test_device_selection_round_trip(require_gpu):
    tb.set_device(0)
    assert tb.get_device() == 0
    with pytest.raises(tb.InvalidArgument, match="out of range"):
        tb.set_device(1 << 20)
    assert tb.get_device() == 0


def _evolve(config, seed):
    p = tb.Pipeline(config)
    p.initialize_gaussian(pulse_for(config, seed))
    p.step(0.0, step_size(config, 0.1), 4)
    state = p.get_state()
    p.close()
    return state


def test_pipelines_on_two_devices_step_alike(require_gpu):
    import torch

    if torch.cuda.device_count() < 2:
        pytest.skip("needs two CUDA devices in this process")
    config = CASES["kerr_d105"]
    states = []
    try:
        for device in (0, 1):
            tb.set_device(device)
            states.append(_evolve(config, 3))
    finally:
        tb.set_device(0)
    assert np.array_equal(states[0], states[1])
