"""Pipeline checkpoint format v5 (include/teuk/pipeline_checkpoint.hpp).

CPU: the reference build writes and reloads its own checkpoints and rejects
a corrupted state (pins the behaviour the GPU tests rely on).
GPU: checkpoints cross between the engine and the reference in both
directions; every metadata line except the state checksum is byte-identical
between the two writers; a restart from a checkpoint continues the run.
"""
import dataclasses

import numpy as np
import pytest

import teuk_b200 as tb
from cases import CASES, pulse_for, relative_error, step_size
from oracle_bindings import RefError, RefPipeline


def _ref_pair(name="kerr_d105", seed=5):
    config = CASES[name]
    ref = RefPipeline(config)
    ref.initialize_gaussian(pulse_for(config, seed))
    return config, ref


def test_reference_checkpoint_round_trip(tmp_path):
    config, ref = _ref_pair("schw_d84")
    dt = step_size(config)
    ref.step(0.0, dt, 3)
    before = ref.get_state()
    ref.checkpoint_write(tmp_path / "ck", dt, 3 * dt, 3)
    meta = (tmp_path / "ck" / "metadata.txt").read_text().splitlines()
    assert meta[0] == "format=teuk-kokkos-pipeline-checkpoint"
    assert meta[1] == "version=5"
    other = RefPipeline(config)
    t, n = other.checkpoint_load(tmp_path / "ck", dt)
    assert (t, n) == (3 * dt, 3)
    assert np.array_equal(other.get_state(), before)
    with pytest.raises(RefError, match="already exists"):
        ref.checkpoint_write(tmp_path / "ck", dt, 3 * dt, 3)
    with pytest.raises(RefError, match="numerical configuration"):
        other.checkpoint_load(tmp_path / "ck", 2 * dt)
    raw = bytearray((tmp_path / "ck" / "state.bin").read_bytes())
    raw[100] ^= 0x01
    (tmp_path / "ck" / "state.bin").write_bytes(bytes(raw))
    with pytest.raises(RefError, match="checksum mismatch"):
        other.checkpoint_load(tmp_path / "ck", dt)


def _metadata_without_checksum(directory):
    lines = (directory / "metadata.txt").read_text().splitlines()
    return [l for l in lines if not l.startswith("state_checksum_fnv1a64=")]


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["kerr_d105", "kerr_d42_sc", "nonparent"])
def test_engine_checkpoint_loads_in_reference(require_gpu, tmp_path, name):
    config = CASES[name]
    gpu = tb.Pipeline(config)
    pulse = pulse_for(config, 9)
    gpu.initialize_gaussian(pulse)
    dt = step_size(config)
    gpu.step(0.0, dt, 4)
    gpu.checkpoint_write(tmp_path / "gpu", dt, 4 * dt, 4)
    ref = RefPipeline(config)
    assert ref.checkpoint_load(tmp_path / "gpu", dt) == (4 * dt, 4)
    assert relative_error(ref.get_state(), gpu.get_state()) < 1e-15
    # the reference writes the same metadata for the same pipeline
    ref.checkpoint_write(tmp_path / "ref", dt, 4 * dt, 4)
    assert _metadata_without_checksum(tmp_path / "gpu") == \
        _metadata_without_checksum(tmp_path / "ref")


@pytest.mark.gpu
def test_reference_checkpoint_restarts_engine(require_gpu, tmp_path):
    config, ref = _ref_pair("kerr_d105")
    dt = step_size(config)
    ref.step(0.0, dt, 5)
    ref.checkpoint_write(tmp_path / "ck", dt, 5 * dt, 5)
    gpu = tb.Pipeline(config)
    assert gpu.checkpoint_load(tmp_path / "ck", dt) == (5 * dt, 5)
    assert relative_error(gpu.get_state(), ref.get_state()) < 1e-12
    gpu.step(5 * dt, dt, 10)
    ref.step(5 * dt, dt, 10)
    assert relative_error(gpu.get_state(), ref.get_state()) < 1e-10


@pytest.mark.gpu
def test_engine_restart_continues_the_run(require_gpu, tmp_path):
    config = CASES["kerr_d105"]
    pulse = pulse_for(config, 13)
    dt = step_size(config)
    straight = tb.Pipeline(config)
    straight.initialize_gaussian(pulse)
    straight.step(0.0, dt, 10)
    first = tb.Pipeline(config)
    first.initialize_gaussian(pulse)
    first.step(0.0, dt, 5)
    first.checkpoint_write(tmp_path / "half", dt, 5 * dt, 5)
    second = tb.Pipeline(config)
    second.checkpoint_load(tmp_path / "half", dt)
    second.step(5 * dt, dt, 5)
    assert relative_error(second.get_state(), straight.get_state()) < 1e-13


@pytest.mark.gpu
def test_second_order_checkpoint_carries_the_latch(require_gpu, tmp_path):
    config = dataclasses.replace(CASES["nonparent"],
                                 source_mode=tb.SOURCE_CONSTRAINT_AWARE,
                                 normalized_constraint_tolerance=1e30,
                                 required_consecutive_passes=2)
    gpu = tb.Pipeline(config)
    gpu.initialize_gaussian(pulse_for(config, 3))
    dt = step_size(config)
    gpu.step(0.0, dt, 2)
    assert gpu.activation().active == 1
    gpu.checkpoint_write(tmp_path / "so", dt, 2 * dt, 2)
    ref = RefPipeline(config)
    ref.checkpoint_load(tmp_path / "so", dt)
    a, b = gpu.activation(), ref.activation()
    assert (a.active, a.activation_time, a.consecutive_passes,
            a.last_eligibility_time) == (b.active, b.activation_time,
                                         b.consecutive_passes,
                                         b.last_eligibility_time)
    gpu.step(2 * dt, dt, 3)
    ref.step(2 * dt, dt, 3)
    g, r = gpu.get_state(), ref.get_state()
    for f in range(tb.FIELD_COUNT):
        assert relative_error(g[:, f], r[:, f]) < 1e-10, f"field {f}"


@pytest.mark.gpu
def test_engine_rejects_corrupted_or_foreign_checkpoints(require_gpu, tmp_path):
    config, ref = _ref_pair("schw_d84")
    dt = step_size(config)
    ref.checkpoint_write(tmp_path / "ck", dt, 0.0, 0)
    gpu = tb.Pipeline(config)
    with pytest.raises(tb.TeukError, match="numerical configuration"):
        gpu.checkpoint_load(tmp_path / "ck", 2 * dt)
    other = tb.Pipeline(dataclasses.replace(config, spin=0.1))
    with pytest.raises(tb.TeukError, match="does not match"):
        other.checkpoint_load(tmp_path / "ck", dt)
    with pytest.raises(tb.TeukError, match="already exists"):
        gpu.checkpoint_write(tmp_path / "ck", dt, 0.0, 0)
    raw = bytearray((tmp_path / "ck" / "state.bin").read_bytes())
    raw[64] ^= 0x10
    (tmp_path / "ck" / "state.bin").write_bytes(bytes(raw))
    before = gpu.get_state()
    with pytest.raises(tb.TeukError, match="checksum mismatch"):
        gpu.checkpoint_load(tmp_path / "ck", dt)
    assert np.array_equal(gpu.get_state(), before)
