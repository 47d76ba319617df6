"""Streaming stage kernel on shapes that split every segment into several
radial strips, against the reference build and against the tile kernel.

The engine runs launch groups with n_ell <= 16 and at most 32 Gauss-Legendre
nodes through the streaming kernel (persistent CTAs, bulk-copy ring), and
free-damped groups with n_ell <= 24 and at most 48 nodes through its wide
form (8-row chunks, two transform groups); LaunchOptions(stage_kernel=
KERNEL_TILE) makes a pipeline use the tile kernel instead.  Segments of one launch differ in n_ell (m = -4..4), so
the ring also changes its row stride between strips.
Tolerance: 1e-10 relative to the field's max norm against the reference;
the two engine kernels agree to 1e-12 (they differ in summation order only).
"""
from dataclasses import replace

import numpy as np
import pytest

import teuk_b200 as tb
from cases import CASES, pulse_for, relative_error, step_size
from oracle_bindings import RefPipeline
from test_gpu_parity import _generic_band_state

pytestmark = pytest.mark.gpu

TOL = 1e-10

LONG = {
    # D10-5 free-damped Kerr, 300 radial points: strips of 64-75 rows
    "kerr_d105_long": replace(CASES["kerr_d105"], radial_points=300),
    # D8-4 stage-constrained Kerr with odd m (n_ell 3..5)
    "kerr_d84_sc_long": replace(CASES["kerr_d42_sc"], discretization=tb.D84,
                                radial_points=260, dissipation=0.005),
    # Schwarzschild D4-2 (pointwise psi_t)
    "schw_d42_long": replace(CASES["schw_d84"], discretization=tb.D42,
                             radial_points=203, dissipation=0.01),
    # D10-5 stage-constrained Kerr (effective-Q lag of 2 x 5 rows)
    "kerr_d105_sc_long": replace(CASES["kerr_d105"], radial_points=280,
                                 reduction=tb.STAGE_CONSTRAINED,
                                 theta_nodes=21, ell_max_first=10,
                                 ell_max_second=10),
    # D8-4 free-damped Schwarzschild without dissipation, odd nr
    "schw_d84_long": replace(CASES["schw_d84"], radial_points=331,
                             dissipation=0.0),
    # wide kernel: D10-5 Kerr, ell <= 20 (n_ell 17..19 for m = -4..4)
    "kerr_d105_wide": replace(CASES["kerr_d105"], radial_points=260,
                              theta_nodes=31, ell_max_first=20,
                              ell_max_second=20),
    # wide kernel: near-extremal D8-4 Kerr, ell <= 24, 37 nodes
    "kerr_d84_wide48": replace(CASES["kerr_d105"], discretization=tb.D84,
                               spin=0.99, radial_points=240, theta_nodes=37,
                               ell_max_first=24, ell_max_second=24,
                               modes=(-2, -1, 0, 1, 2)),
    # wide kernel: Schwarzschild D4-2 (pointwise psi_t), ell <= 22
    "schw_d42_wide": replace(CASES["schw_d84"], discretization=tb.D42,
                             radial_points=203, theta_nodes=34,
                             ell_max_first=22, ell_max_second=22,
                             dissipation=0.01),
}


def _pair(name, seed=11):
    config = LONG[name]
    gpu = tb.Pipeline(config)
    ref = RefPipeline(config)
    pulse = pulse_for(config, seed)
    gpu.initialize_gaussian(pulse)
    ref.initialize_gaussian(pulse)
    return config, gpu, ref


@pytest.mark.parametrize("name", sorted(LONG))
def test_long_rhs_matches_reference(require_gpu, name):
    config, gpu, ref = _pair(name)
    state = _generic_band_state(ref, 23)
    g = gpu.evaluate_rhs(state)
    r = ref.evaluate_rhs(state)
    for f in range(3):
        assert relative_error(g[:, f], r[:, f]) < TOL, f"field {f}"
    assert np.all(g[:, 3:] == 0)


@pytest.mark.parametrize("name", sorted(LONG))
def test_long_rk4_matches_reference(require_gpu, name):
    config, gpu, ref = _pair(name)
    dt = step_size(config, 0.1)
    gpu.step(0.0, dt, 6)
    ref.step(0.0, dt, 6)
    g, r = gpu.get_state(), ref.get_state()
    for f in range(3):
        assert relative_error(g[:, f], r[:, f]) < TOL, f"field {f}"
    assert np.array_equal(g[:, 3:], r[:, 3:])


@pytest.mark.parametrize("name", sorted(LONG) + ["kerr_d105", "kerr_d42_sc"])
def test_stream_kernel_equals_tile_kernel(require_gpu, name):
    config = LONG.get(name, CASES.get(name))
    pulse = pulse_for(config, 5)
    stream = tb.Batch([config])
    tile = tb.Batch([config], tb.LaunchOptions(stage_kernel=tb.KERNEL_TILE))
    assert stream.stage_kernels() == (1, 0)
    assert tile.stage_kernels() == (0, 1)
    for p in (stream, tile):
        p.initialize_gaussian(0, pulse)
    dt = step_size(config, 0.1)
    stream.step([dt], 12)
    tile.step([dt], 12)
    a, b = stream.get_state(0), tile.get_state(0)
    for f in range(3):
        assert relative_error(a[:, f], b[:, f]) < 1e-12, f"field {f}"


def test_mixed_batch_matches_solo(require_gpu):
    """Solves of different radial sizes, spins and n_ell share launches; each
    result equals the same solve run alone (the streaming kernel's rows do
    not depend on how segments are split into strips)."""
    base = LONG["kerr_d105_long"]
    configs = [base,
               replace(base, radial_points=129, spin=0.3),
               replace(base, radial_points=777, spin=0.9, ell_max_first=12,
                       ell_max_second=12),
               replace(base, radial_points=64, spin=0.0),
               # bands with n_ell 17..19 (wide kernel) and 37 nodes
               replace(base, radial_points=301, spin=0.6, theta_nodes=31,
                       ell_max_first=20, ell_max_second=20),
               replace(base, radial_points=150, spin=0.95, theta_nodes=37,
                       ell_max_first=24, ell_max_second=24, modes=(-2, 2))]
    pulses = [pulse_for(c, 31 + i) for i, c in enumerate(configs)]
    dts = [step_size(c, 0.1) for c in configs]
    batch = tb.Batch(configs)
    assert batch.stage_kernels() == (2, 0)  # narrow and wide groups
    for i, p in enumerate(pulses):
        batch.initialize_gaussian(i, p)
    batch.step(dts, 5)
    for i, c in enumerate(configs):
        solo = tb.Pipeline(c)
        solo.initialize_gaussian(pulses[i])
        solo.step(0.0, dts[i], 5)
        assert np.array_equal(batch.get_state(i), solo.get_state()), i


def test_solve_split_between_stage_kernels(require_gpu):
    """Stage-constrained, ell <= 18 with m = -4..4: the m = +-2, +-1, 0 bands
    (n_ell >= 17; the wide kernel is free-damped only) run the tile kernel,
    the m = +-3, +-4 bands the streaming kernel, in the same step; the result
    matches the reference."""
    config = replace(CASES["kerr_d105"], radial_points=220, theta_nodes=29,
                     ell_max_first=18, ell_max_second=18,
                     reduction=tb.STAGE_CONSTRAINED)
    batch = tb.Batch([config])
    assert batch.stage_kernels() == (1, 1)
    ref = RefPipeline(config)
    pulse = pulse_for(config, 13)
    batch.initialize_gaussian(0, pulse)
    ref.initialize_gaussian(pulse)
    dt = step_size(config, 0.1)
    batch.step([dt], 6)
    ref.step(0.0, dt, 6)
    g, r = batch.get_state(0), ref.get_state()
    for f in range(3):
        assert relative_error(g[:, f], r[:, f]) < TOL, f"field {f}"


def test_stage_wait_timeout_is_reported(require_gpu):
    """Failure detection without a GPU fault: with the test hook
    teuk_b200_test_withhold_chunk the producer of one CTA never loads a chunk in
    stage-1 launches, so the transform warps' bounded wait runs out (2 s),
    every warp role leaves its loop, and the step reports the timeout.  The
    device context stays usable: a new pipeline then steps like the
    reference."""
    config = LONG["kerr_d105_long"]
    dt = step_size(config, 0.1)
    tb.test_withhold_chunk(2)
    try:
        broken = tb.Pipeline(config)
    finally:
        tb.test_withhold_chunk(-1)
    broken.initialize_gaussian(pulse_for(config, 19))
    with pytest.raises(tb.TeukError, match="timed out"):
        broken.step(0.0, dt, 1)
    broken.close()
    config, gpu, ref = _pair("kerr_d105_long")
    gpu.step(0.0, dt, 2)
    ref.step(0.0, dt, 2)
    g, r = gpu.get_state(), ref.get_state()
    for f in range(3):
        assert relative_error(g[:, f], r[:, f]) < TOL, f"field {f}"
