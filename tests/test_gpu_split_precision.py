"""Split-precision tensor-core transforms against the FP64 reference (GPU).

With ``LaunchOptions(precision=PRECISION_SPLIT)`` the transforms multiply
through BF16 digit slices with FP32 accumulation and FP64 recombination
(split_precision.cuh): in the second-order pipeline the angular operators
(project, Laplacian, eth, eth'), in the linear streaming kernel the synthesis
and analysis of the implicit Kerr ell-coupling; everything else stays FP64.  The stated
bound for this path is 1e-9 relative to each field's maximum modulus against
the reference build (the plain FP64 path is held to 1e-10 elsewhere), with
activation records exact.
"""
from dataclasses import replace

import numpy as np
import pytest

import teuk_b200 as tb
from teuk_b200 import workloads as wl
from cases import relative_error
from oracle_bindings import RefPipeline

pytestmark = pytest.mark.gpu

SPLIT_TOL = 1e-9
SPLIT = tb.LaunchOptions(precision=tb.PRECISION_SPLIT)


def _activation(a):
    return (a.active, a.activation_time, a.consecutive_passes,
            a.last_eligibility_time)


def _field_errors(a, b, fields):
    return [relative_error(a[:, f], b[:, f]) for f in fields]


def test_split_quadratic_source_full_shape(require_gpu):
    """a 0.9, nr 1025, ntheta 48, ell <= 10 / 20, source switched on inside
    the run: all 13 fields within 1e-9 of the reference after 12 steps."""
    base, pulse, dt = wl.second_order_self_coupling()
    config = replace(base, source_start_time=5.5 * dt)
    split = tb.Pipeline(config, SPLIT)
    fp64 = tb.Pipeline(config)
    ref = RefPipeline(config, threads=True)
    for p in (split, fp64, ref):
        p.initialize_gaussian(pulse)
    t = 0.0
    for block in (4, 4, 4):
        for p in (split, fp64, ref):
            p.step(t, dt, block)
        t += block * dt
        assert _activation(split.activation()) == _activation(ref.activation())
    r = ref.get_state()
    errors = _field_errors(split.get_state(), r, range(13))
    assert max(errors) < SPLIT_TOL, errors
    # the FP64 path of the same engine stays at its own tighter bound
    assert max(_field_errors(fp64.get_state(), r, range(13))) < 1e-10


def test_split_rhs_of_a_generic_state(require_gpu):
    """One right-hand side of a seeded state with all 13 fields populated
    (projected onto each field's band by the reference): every field of the
    split-precision RHS within 1e-9 of the reference's."""
    config = tb.SolveConfig(
        mass=1.0, spin=0.7, compactification_length=1.2, radial_points=64,
        theta_nodes=24, ell_max_first=6, ell_max_second=12,
        modes=(-4, -2, 0, 2, 4), parents=(-2, 2), targets=(-4, 0, 4),
        dissipation=0.003, discretization=tb.D84,
        source_mode=tb.SOURCE_UNRESTRICTED)
    ref = RefPipeline(config)
    rng = np.random.Generator(np.random.PCG64(5))
    shape = config.shape()
    state = ref.project_to_bands(1e-3 * (rng.standard_normal(shape) +
                                         1j * rng.standard_normal(shape)))
    split = tb.Pipeline(config, SPLIT)
    split.set_state(state)
    ref.set_state(state)
    g = split.evaluate_rhs(state)
    r = ref.evaluate_rhs(state)
    errors = _field_errors(g, r, range(13))
    assert max(errors) < SPLIT_TOL, errors


def test_split_precision_is_rejected_above_64_nodes(require_gpu):
    config = tb.SolveConfig(
        mass=1.0, spin=0.5, compactification_length=1.0, radial_points=40,
        theta_nodes=66, ell_max_first=4, ell_max_second=8,
        modes=(-4, -2, 0, 2, 4), parents=(-2, 2), targets=(-4, 0, 4),
        discretization=tb.D42, source_mode=tb.SOURCE_UNRESTRICTED)
    with pytest.raises(tb.InvalidArgument, match="at most 64 theta nodes"):
        tb.Pipeline(config, SPLIT)


def test_split_kerr_ringdown_nr1025_100_steps(require_gpu):
    """The linear Kerr ringdown at its full shape (a 0.7, nr 1025, D10-5,
    m = -4..4, ell <= 16) on the streaming kernel with split-precision
    transforms: within 1e-9 of the reference after 100 steps."""
    config, pulse, dt = wl.kerr_ringdown()
    ref = RefPipeline(config, threads=True)
    ref.initialize_gaussian(pulse)
    state = ref.get_state() + ref.project_to_bands(wl.band_noise(config, 7))
    ref.set_state(state)
    split = tb.Pipeline(config, SPLIT)
    split.set_state(state)
    split.step(0.0, dt, 100)
    ref.step(0.0, dt, 100)
    errors = _field_errors(split.get_state(), ref.get_state(), range(3))
    assert max(errors) < SPLIT_TOL, errors


@pytest.mark.parametrize("reduction", [tb.FREE_DAMPED, tb.STAGE_CONSTRAINED])
def test_split_linear_rhs_and_steps(require_gpu, reduction):
    """Both reductions of the streaming kernel (D8-4, several strips)."""
    config = tb.SolveConfig(
        mass=1.0, spin=0.8, compactification_length=1.0, radial_points=300,
        theta_nodes=25, ell_max_first=16, ell_max_second=16,
        modes=tuple(range(-4, 5)), dissipation=0.003,
        discretization=tb.D84, reduction=reduction)
    ref = RefPipeline(config)
    from cases import pulse_for, step_size
    pulse = pulse_for(config, 3)
    ref.initialize_gaussian(pulse)
    split = tb.Pipeline(config, SPLIT)
    split.initialize_gaussian(pulse)
    dt = step_size(config, 0.1)
    split.step(0.0, dt, 20)
    ref.step(0.0, dt, 20)
    errors = _field_errors(split.get_state(), ref.get_state(), range(3))
    assert max(errors) < SPLIT_TOL, errors


def test_split_batch_member_equals_solo(require_gpu):
    """Split-precision results depend only on each row's own data: a solve
    in a mixed batch equals the same solve alone, bit for bit."""
    from cases import pulse_for, step_size
    base = tb.SolveConfig(
        mass=1.0, spin=0.7, compactification_length=1.0, radial_points=300,
        theta_nodes=25, ell_max_first=16, ell_max_second=16,
        modes=tuple(range(-4, 5)), dissipation=0.005, discretization=tb.D105)
    configs = [base, replace(base, radial_points=129, spin=0.3),
               replace(base, radial_points=513, spin=0.9, ell_max_first=12,
                       ell_max_second=12, theta_nodes=19)]
    pulses = [pulse_for(c, 31 + i) for i, c in enumerate(configs)]
    dts = [step_size(c, 0.1) for c in configs]
    batch = tb.Batch(configs, SPLIT)
    for i, p in enumerate(pulses):
        batch.initialize_gaussian(i, p)
    batch.step(dts, 5)
    for i, c in enumerate(configs):
        solo = tb.Pipeline(c, SPLIT)
        solo.initialize_gaussian(pulses[i])
        solo.step(0.0, dts[i], 5)
        assert np.array_equal(batch.get_state(i), solo.get_state()), i


def test_split_batch_runs_wide_bands_in_fp64(require_gpu):
    """Bands on the wide streaming kernel transform in FP64 in every
    precision: in a split-precision batch, a solve whose bands are all wide
    equals the same solve in an FP64 batch bit for bit, beside a narrow
    split-precision solve."""
    from cases import pulse_for, step_size
    narrow = tb.SolveConfig(
        mass=1.0, spin=0.7, compactification_length=1.0, radial_points=200,
        theta_nodes=25, ell_max_first=16, ell_max_second=16,
        modes=tuple(range(-4, 5)), dissipation=0.005, discretization=tb.D105)
    wide = replace(narrow, radial_points=240, spin=0.95, theta_nodes=37,
                   ell_max_first=24, ell_max_second=24, modes=(-2, 2))
    configs = [narrow, wide]
    pulses = [pulse_for(c, 41 + i) for i, c in enumerate(configs)]
    dts = [step_size(c, 0.1) for c in configs]
    states = []
    for options in (SPLIT, None):
        batch = tb.Batch(configs, options)
        assert batch.stage_kernels() == (2, 0)  # narrow and wide groups
        for i, p in enumerate(pulses):
            batch.initialize_gaussian(i, p)
        batch.step(dts, 6)
        states.append([batch.get_state(i) for i in range(2)])
    assert np.array_equal(states[0][1], states[1][1])
    assert not np.array_equal(states[0][0], states[1][0])
    assert relative_error(states[0][0][:, :3], states[1][0][:, :3]) < SPLIT_TOL


def test_split_second_order_checkpoint_loads_into_the_reference(require_gpu, tmp_path):
    """Projections run the FP64 two-GEMM path in every precision, so a
    split-precision pipeline's state stays band limited to the reference's
    checkpoint tolerance (5e-11 per radial line) and the reference loads it."""
    config = tb.SolveConfig(
        mass=1.0, spin=0.7, compactification_length=1.2, radial_points=48,
        theta_nodes=9, ell_max_first=4, ell_max_second=8,
        modes=(-4, -2, 0, 2, 4), parents=(-2, 2), targets=(-4, 0, 4),
        dissipation=0.0, discretization=tb.D84,
        source_mode=tb.SOURCE_CONSTRAINT_AWARE,
        normalized_constraint_tolerance=1e30, required_consecutive_passes=2)
    from cases import pulse_for, step_size
    split = tb.Pipeline(config, SPLIT)
    split.initialize_gaussian(pulse_for(config, 3))
    dt = step_size(config)
    split.step(0.0, dt, 3)
    split.checkpoint_write(tmp_path / "split", dt, 3 * dt, 3)
    ref = RefPipeline(config)
    ref.checkpoint_load(tmp_path / "split", dt)
    errors = _field_errors(split.get_state(), ref.get_state(), range(13))
    assert max(errors) < 1e-12, errors
