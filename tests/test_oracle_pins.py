"""Pins of the C oracle (CPU, no GPU).

1. Known-answer properties the reference's own tests hold
   (tests/test_sbp.cpp, test_sbp84.cpp, test_sbp105.cpp:75-135; test_angular.cpp):
   the SBP identity H D + D^T H = diag(-1, 0, ..., 0, 1), polynomial
   exactness of the interior/boundary rows, Gauss-Legendre exactness and
   orthonormality of the analysis/synthesis pair.
2. Bit-level agreement of the oracle's tables with the reference compiled
   from its own headers (oracle/_ref): SBP matrices, Gauss-Legendre nodes.
3. RHS and RK4 agreement of the oracle with the reference pipeline on the
   shared seeded cases (the reference builds the initial data).
"""
import numpy as np
import pytest

import teuk_b200 as tb
from cases import CASES, pulse_for, relative_error, step_size
from oracle_bindings import (OraclePipeline, RefPipeline, oracle_gauss_legendre,
                             oracle_sbp_matrix, ref_available,
                             ref_gauss_legendre, ref_sbp_matrix,
                             ref_transform_matrices)

needs_ref = pytest.mark.skipif(not ref_available(),
                               reason="oracle/_ref not built (reference absent)")

ORDERS = {tb.D42: (2, 4), tb.D84: (4, 8), tb.D105: (5, 10)}


@pytest.mark.parametrize("disc,n", [(tb.D42, 20), (tb.D84, 40), (tb.D105, 50)])
def test_sbp_identity_and_exactness(disc, n):
    D, H = oracle_sbp_matrix(disc, n)
    Hm = np.diag(H)
    B = Hm @ D + D.T @ Hm
    expected = np.zeros((n, n))
    expected[0, 0] = -1.0
    expected[-1, -1] = 1.0
    assert np.max(np.abs(B - expected)) < 5e-13
    h = 1.0 / (n - 1)
    x = np.linspace(0.0, 1.0, n)
    boundary_order, interior_order = ORDERS[disc]
    closure = {tb.D42: 4, tb.D84: 8, tb.D105: 11}[disc]
    half = interior_order // 2
    for k in range(boundary_order + 1):
        exact = h * k * x ** (k - 1) if k else 0 * x
        assert np.max(np.abs(D @ x ** k - exact)) < 1e-11
    interior = slice(closure + half, n - closure - half)
    for k in range(interior_order + 1):
        exact = h * k * x ** (k - 1) if k else 0 * x
        assert np.max(np.abs((D @ x ** k - exact)[interior])) < 1e-11


@pytest.mark.parametrize("n", [7, 13, 25, 48])
def test_gauss_legendre_exactness(n):
    x, w = oracle_gauss_legendre(n)
    assert np.all(np.diff(x) > 0)
    for k in range(2 * n):
        exact = 0.0 if k % 2 else 2.0 / (k + 1)
        assert abs(np.dot(w, x ** k) - exact) < 1e-13


@needs_ref
@pytest.mark.parametrize("disc,n", [(tb.D42, 20), (tb.D84, 40), (tb.D105, 50)])
def test_sbp_tables_bitwise_equal_reference(disc, n):
    Do, Ho = oracle_sbp_matrix(disc, n)
    Dr, Hr = ref_sbp_matrix(disc, n)
    assert np.array_equal(Do, Dr)
    assert np.array_equal(Ho, Hr)


@needs_ref
@pytest.mark.parametrize("n", [7, 10, 13, 25, 48])
def test_gauss_legendre_bitwise_equal_reference(n):
    xo, wo = oracle_gauss_legendre(n)
    xr, wr = ref_gauss_legendre(n)
    assert np.array_equal(xo, xr)
    assert np.array_equal(wo, wr)


@needs_ref
@pytest.mark.parametrize("m,ell_max,nodes", [(2, 8, 13), (-4, 16, 25),
                                             (0, 20, 48)])
def test_transform_orthonormality(m, ell_max, nodes):
    S, A = ref_transform_matrices(-2, m, ell_max, nodes)
    # The reference evaluates the basis in long double; at ell = 20 the
    # quadrature pair is orthonormal to ~4e-13.
    assert np.max(np.abs(A @ S - np.eye(S.shape[1]))) < 1e-12


def _oracle_and_ref(name, seed=5):
    config = CASES[name]
    ref = RefPipeline(config)
    ref.initialize_gaussian(pulse_for(config, seed))
    orc = OraclePipeline(config)
    orc.set_state(ref.get_state())
    return config, orc, ref


@needs_ref
@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_rhs_matches_reference(name):
    config, orc, ref = _oracle_and_ref(name)
    state = ref.get_state()
    rng = np.random.Generator(np.random.PCG64(23))
    noise = np.zeros_like(state)
    noise[:, :3] = np.max(np.abs(state[:, 2])) * (
        rng.standard_normal(state[:, :3].shape) +
        1j * rng.standard_normal(state[:, :3].shape))
    state = ref.project_to_bands(state + noise)
    o = orc.evaluate_rhs(state)
    r = ref.evaluate_rhs(state)
    for f in range(3):
        assert relative_error(o[:, f], r[:, f]) < 1e-13, f"field {f}"
    assert np.all(o[:, 3:] == 0)


@needs_ref
@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_steps_match_reference(name):
    config, orc, ref = _oracle_and_ref(name)
    dt = step_size(config)
    orc.step(0.0, dt, 5)
    ref.step(0.0, dt, 5)
    o, r = orc.get_state(), ref.get_state()
    for f in range(3):
        assert relative_error(o[:, f], r[:, f]) < 1e-13, f"field {f}"
