"""Seeded solve configurations shared by the parity tests and smoke().

Shapes are small versions of the benchmark configurations (the full sizes
run in bench.py and in the size-independent property tests):

* ``schw_d84``   Schwarzschild, D8-4, m = +-2, ell <= 8 (the 2000-step CPU
                 configuration at reduced nr)
* ``kerr_d105``  Kerr a = 0.7, D10-5, m = -4..4, ell <= 16, ntheta = 25 (the
                 Kerr ringdown configuration at reduced nr)
* ``kerr_d42_sc`` Kerr a = 0.5, D4-2, stage-constrained reduction
* ``nonparent``  stored modes {-4,-2,0,2,4} with parents {-2,2}: the
                 non-parent first-order fields stay frozen
"""
from __future__ import annotations

import numpy as np

import teuk_b200 as tb


def pulse_for(config: tb.SolveConfig, seed: int, center_fraction: float = 0.3,
              width_fraction: float = 0.06, amplitude: float = 1e-3,
              extra_modes: bool = True) -> tb.GaussianPulse:
    """Seeded complex amplitudes (numpy PCG64) on ell = 2 of every parent
    m >= 2 plus, optionally, a smaller ell = 3 component."""
    rng = np.random.Generator(np.random.PCG64(seed))
    modes = []
    for m in sorted(config.parent_list()):
        if abs(m) > 2 or m == 0 and not extra_modes:
            continue
        ell = max(2, abs(m))
        amp = amplitude * complex(rng.standard_normal(), rng.standard_normal())
        modes.append((ell, m, amp))
        if extra_modes and ell + 1 <= config.ell_max_first:
            amp3 = 0.3 * amplitude * complex(rng.standard_normal(),
                                             rng.standard_normal())
            modes.append((ell + 1, m, amp3))
    R_H = config.horizon_radius
    return tb.GaussianPulse(center=center_fraction * R_H,
                            width=width_fraction * R_H, modes=modes)


CASES = {
    "schw_d84": tb.SolveConfig(
        mass=1.0, spin=0.0, compactification_length=1.0, radial_points=64,
        theta_nodes=13, ell_max_first=8, ell_max_second=8, modes=(-2, 2),
        dissipation=0.005, discretization=tb.D84),
    "kerr_d105": tb.SolveConfig(
        mass=1.0, spin=0.7, compactification_length=1.0, radial_points=96,
        theta_nodes=25, ell_max_first=16, ell_max_second=16,
        modes=tuple(range(-4, 5)), dissipation=0.005,
        discretization=tb.D105),
    "kerr_d42_sc": tb.SolveConfig(
        mass=1.0, spin=0.5, compactification_length=1.5, radial_points=40,
        theta_nodes=10, ell_max_first=6, ell_max_second=6,
        modes=(-3, -2, -1, 0, 1, 2, 3), dissipation=0.01,
        discretization=tb.D42, reduction=tb.STAGE_CONSTRAINED),
    "nonparent": tb.SolveConfig(
        mass=1.0, spin=0.7, compactification_length=1.2, radial_points=48,
        theta_nodes=9, ell_max_first=4, ell_max_second=8,
        modes=(-4, -2, 0, 2, 4), parents=(-2, 2), targets=(-4, 0, 4),
        dissipation=0.0, discretization=tb.D84),
}


def step_size(config: tb.SolveConfig, ratio: float = 0.02) -> float:
    return ratio * config.spacing


def relative_error(value: np.ndarray, reference: np.ndarray) -> float:
    scale = np.max(np.abs(reference))
    if scale == 0.0:
        return float(np.max(np.abs(value)))
    return float(np.max(np.abs(value - reference)) / scale)
