"""Split-precision tensor-core transforms against the FP64 reference (GPU).

With ``LaunchOptions(precision=PRECISION_SPLIT)`` the angular operators
(project, Laplacian, eth, eth') multiply through BF16 digit slices with FP32
accumulation and FP64 recombination; everything else stays FP64.  The stated
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
