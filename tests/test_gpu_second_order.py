"""Second-order (quadratic source) pipeline vs the reference (GPU).

The ConstraintAware and Unrestricted source policies run the full stage
graph of SpatialPipeline::evaluate_rhs_at_time: first-order Teukolsky,
metric reconstruction and its stage tangent, the independent constraints,
the Jet1 ordered-pair source, the outer source and the forced second-order
Teukolsky block, advanced by RK4 with the source-activation latch.  Every
case compares all 13 fields against the reference build on the same state,
with 1e-10 relative tolerance per field (relative to that field's max norm),
and compares the activation records exactly.
"""
import dataclasses

import numpy as np
import pytest

import teuk_b200 as tb
from cases import pulse_for, relative_error, step_size
from oracle_bindings import RefPipeline

pytestmark = pytest.mark.gpu

TOL = 1e-10

SO_CASES = {
    # stored modes {-4..4 even}, parents +-2, targets {-4, 0, 4}; Kerr a=0.7
    "so_unrestricted_d84": tb.SolveConfig(
        mass=1.0, spin=0.7, compactification_length=1.2, radial_points=48,
        theta_nodes=9, ell_max_first=4, ell_max_second=8,
        modes=(-4, -2, 0, 2, 4), parents=(-2, 2), targets=(-4, 0, 4),
        dissipation=0.003, discretization=tb.D84,
        source_mode=tb.SOURCE_UNRESTRICTED),
    # odd and even parents, stage-constrained reduction, D4-2
    "so_constraint_d42_sc": tb.SolveConfig(
        mass=1.0, spin=0.5, compactification_length=1.5, radial_points=40,
        theta_nodes=10, ell_max_first=4, ell_max_second=6,
        modes=(-4, -3, -2, -1, 0, 1, 2, 3, 4), parents=(-2, -1, 1, 2),
        targets=(-3, -2, -1, 0, 1, 2, 3), dissipation=0.01,
        discretization=tb.D42, reduction=tb.STAGE_CONSTRAINED,
        source_mode=tb.SOURCE_CONSTRAINT_AWARE,
        normalized_constraint_tolerance=1e30, required_consecutive_passes=2),
    # near-extremal spin, D10-5, source switched on inside a step
    "so_kerr_d105_start": tb.SolveConfig(
        mass=1.0, spin=0.9, compactification_length=1.0, radial_points=48,
        theta_nodes=12, ell_max_first=4, ell_max_second=8,
        modes=(-4, -2, 0, 2, 4), parents=(-2, 2), targets=(-4, 0, 4),
        dissipation=0.002, discretization=tb.D105,
        source_mode=tb.SOURCE_UNRESTRICTED),
}


def _pair(config, seed=11):
    gpu = tb.Pipeline(config)
    ref = RefPipeline(config)
    pulse = pulse_for(config, seed)
    gpu.initialize_gaussian(pulse)
    ref.initialize_gaussian(pulse)
    return gpu, ref


def _generic_state(ref, seed, amplitude=1e-3):
    """Initial data plus seeded perturbations of all 13 fields, projected
    onto each field's retained band by the reference itself, so the
    reconstruction fields and the quadratic source are generic."""
    state = ref.get_state()
    rng = np.random.Generator(np.random.PCG64(seed))
    noise = amplitude * (rng.standard_normal(state.shape) +
                         1j * rng.standard_normal(state.shape))
    return ref.project_to_bands(state + noise)


def _compare_fields(g, r, tol=TOL):
    for f in range(tb.FIELD_COUNT):
        assert relative_error(g[:, f], r[:, f]) < tol, f"field {f}"


def _activation_tuple(a):
    return (a.active, a.activation_time, a.consecutive_passes,
            a.last_eligibility_time)


@pytest.mark.parametrize("name", sorted(SO_CASES))
def test_second_order_initial_state(require_gpu, name):
    config = SO_CASES[name]
    gpu, ref = _pair(config)
    assert gpu.shape == ref.shape
    assert relative_error(gpu.get_state(), ref.get_state()) < 1e-12
    assert _activation_tuple(gpu.activation()) == \
        _activation_tuple(ref.activation())


@pytest.mark.parametrize("name", sorted(SO_CASES))
def test_second_order_rhs(require_gpu, name):
    config = SO_CASES[name]
    gpu, ref = _pair(config)
    state = _generic_state(ref, 23)
    g = gpu.evaluate_rhs(state, time=0.0)
    r = ref.evaluate_rhs(state, 0.0)
    _compare_fields(g, r)
    if config.source_mode == tb.SOURCE_UNRESTRICTED:
        # the forcing reaches the second-order block
        assert np.max(np.abs(r[:, 10])) > 0.0


def test_second_order_rhs_with_active_constraint_aware_source(require_gpu):
    """ConstraintAware activates after two accepted checks; the RHS then
    carries the forcing."""
    config = SO_CASES["so_constraint_d42_sc"]
    gpu, ref = _pair(config)
    dt = step_size(config)
    gpu.step(0.0, dt, 2)
    ref.step(0.0, dt, 2)
    assert gpu.activation().active == 1
    assert _activation_tuple(gpu.activation()) == \
        _activation_tuple(ref.activation())
    state = _generic_state(ref, 29)
    g = gpu.evaluate_rhs(state, time=2 * dt)
    r = ref.evaluate_rhs(state, 2 * dt)
    assert np.max(np.abs(r[:, 10])) > 0.0
    _compare_fields(g, r)


@pytest.mark.parametrize("name", sorted(SO_CASES))
def test_second_order_steps(require_gpu, name):
    config = SO_CASES[name]
    gpu, ref = _pair(config)
    state = _generic_state(ref, 31)
    gpu.set_state(state)
    ref.set_state(state)
    dt = step_size(config)
    gpu.step(0.0, dt, 8)
    ref.step(0.0, dt, 8)
    _compare_fields(gpu.get_state(), ref.get_state())
    assert _activation_tuple(gpu.activation()) == \
        _activation_tuple(ref.activation())


def test_source_start_inside_a_step(require_gpu):
    """source_start_time = 1.5 dt: the second step is split at the start
    time, the latch flips there, and the rest of the step carries the
    forcing (SpatialPipeline::step)."""
    base = SO_CASES["so_kerr_d105_start"]
    dt = step_size(base)
    config = dataclasses.replace(base, source_start_time=1.5 * dt)
    gpu, ref = _pair(config)
    state = _generic_state(ref, 37)
    gpu.set_state(state)
    ref.set_state(state)
    assert gpu.activation().active == 0
    gpu.step(0.0, dt, 3)
    ref.step(0.0, dt, 3)
    a = gpu.activation()
    assert a.active == 1 and a.activation_time == 1.5 * dt
    assert _activation_tuple(a) == _activation_tuple(ref.activation())
    _compare_fields(gpu.get_state(), ref.get_state())


def test_constraint_aware_latch_never_passes_at_zero_tolerance(require_gpu):
    base = SO_CASES["so_constraint_d42_sc"]
    config = dataclasses.replace(base, normalized_constraint_tolerance=0.0)
    gpu, ref = _pair(config)
    dt = step_size(config)
    gpu.step(0.0, dt, 3)
    ref.step(0.0, dt, 3)
    a = gpu.activation()
    assert a.active == 0 and a.consecutive_passes == 0
    assert _activation_tuple(a) == _activation_tuple(ref.activation())
    g, r = gpu.get_state(), ref.get_state()
    _compare_fields(g, r)
    # no forcing while latched off: the second-order block stays at rest
    assert np.all(g[:, 10:] == 0)


def test_activation_restore_and_reset(require_gpu):
    config = SO_CASES["so_constraint_d42_sc"]
    gpu, ref = _pair(config)
    a = tb.Activation()
    a.active, a.activation_time = 1, 0.25
    a.consecutive_passes, a.last_eligibility_time = 2, 0.25
    gpu.restore_activation(a)
    assert _activation_tuple(gpu.activation()) == (1, 0.25, 2, 0.25)
    bad = tb.Activation()
    bad.active, bad.activation_time = 0, 0.5
    bad.consecutive_passes, bad.last_eligibility_time = 0, -1.0
    with pytest.raises(tb.InvalidArgument,
                       match="invalid second-order source activation state"):
        gpu.restore_activation(bad)
    gpu.reset_activation()
    assert _activation_tuple(gpu.activation()) == (0, -1.0, 0, -1.0)


@pytest.mark.parametrize("name", sorted(SO_CASES))
def test_second_order_waveforms(require_gpu, name):
    config = SO_CASES[name]
    gpu, ref = _pair(config)
    state = _generic_state(ref, 41)
    gpu.set_state(state)
    ref.set_state(state)
    dt = step_size(config)
    gpu.step(0.0, dt, 4)
    ref.step(0.0, dt, 4)
    g, r = gpu.sample_endpoint(), ref.sample_endpoint()
    key = [(x["boundary"], x["order"], x["m"], x["ell"]) for x in g]
    assert key == [(x["boundary"], x["order"], x["m"], x["ell"]) for x in r]
    for order in (1, 2):
        gv = np.array([x["endpoint"] for x in g if x["order"] == order])
        rv = np.array([x["endpoint"] for x in r if x["order"] == order])
        assert relative_error(gv, rv) < TOL


def test_batch_of_identical_second_order_solves(require_gpu):
    """Identical Unrestricted solves from t = 0 form one batch: the replicas
    of one nodal pipeline, stepped by shared launches.  Each replica's
    13-field state and waveform records equal those of the solve alone bit
    for bit, and one replica is checked against the reference build."""
    config = SO_CASES["so_unrestricted_d84"]
    dt = step_size(config)
    seeds = (21, 22, 23)
    batch = tb.Batch([config] * len(seeds))
    assert len(batch) == 3 and batch.strip_rows() == []
    assert batch.stage_kernels() == (0, 0)
    for i, seed in enumerate(seeds):
        batch.initialize_gaussian(i, pulse_for(config, seed))
    ref = RefPipeline(config)
    ref.initialize_gaussian(pulse_for(config, seeds[1]))
    batch.step(dt, 3)
    batch.step(dt, 2)
    ref.step(0.0, dt, 5)
    _compare_fields(batch.get_state(1), ref.get_state())
    for i, seed in enumerate(seeds):
        alone = tb.Pipeline(config)
        alone.initialize_gaussian(pulse_for(config, seed))
        alone.step(0.0, dt, 5)
        assert np.array_equal(batch.get_state(i), alone.get_state()), i
        assert batch.sample_endpoint(i) == alone.sample_endpoint(), i
    # a state written into one replica changes only that replica
    state = _generic_state(ref, 43)
    before = batch.get_state(2)
    batch.set_state(0, state)
    assert np.array_equal(batch.get_state(0), state)
    assert np.array_equal(batch.get_state(2), before)
    with pytest.raises(tb.Unsupported):
        batch.endpoint_modal()
    with pytest.raises(IndexError):
        batch.get_state(3)


def test_batch_rejects_other_second_order_mixes(require_gpu):
    """Second-order batches other than identical Unrestricted-from-zero
    solves stay with one pipeline each."""
    un = SO_CASES["so_unrestricted_d84"]
    cases = [
        [SO_CASES["so_constraint_d42_sc"]] * 2,
        [un, SO_CASES["so_kerr_d105_start"]],
        [un, dataclasses.replace(un, source_mode=tb.SOURCE_DISABLED)],
        [dataclasses.replace(un, source_start_time=0.5)] * 2,
    ]
    for configs in cases:
        with pytest.raises(tb.Unsupported):
            tb.Batch(configs)
