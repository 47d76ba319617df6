"""Seeded synthetic workloads with the benchmark configurations' shapes, and
the run-driver arithmetic the reference uses to size a time step.

* ``maximum_coordinate_speed`` restates solver_driver.hpp:36-57 with the
  characteristic speeds of boundary.hpp:23-37;
* ``dissipation_bound`` restates radial_discretization.hpp:20-59.

Boyer-Lindquist radii map to the compactified coordinate by R = L^2 / r
(docs/CONVENTIONS.md of the reference); a width dr maps to L^2 dr / r^2
(linearised at the pulse centre).
"""
from __future__ import annotations

import math
from dataclasses import replace

import numpy as np

from . import (D42, D84, D105, FIELD_COUNT, GaussianPulse, SolveConfig)

SPECTRAL_BOUND = {D42: 64.0, D84: 1371.0, D105: 5500.0}
RK4_NEGATIVE_AXIS = 2.785293563405282
SAFETY = 0.8


def _gauss_legendre(n: int):
    x, w = np.polynomial.legendre.leggauss(n)
    return x, w


def maximum_coordinate_speed(config: SolveConfig) -> float:
    """max |(K +- sqrt(K^2 + C_T H_R)) / C_T| over the (R, theta) grid."""
    M, a, L = config.mass, config.spin, config.compactification_length
    x, _ = _gauss_legendre(config.theta_nodes)
    theta = np.arccos(x)
    R = config.spacing * np.arange(config.radial_points)
    L2, L4 = L * L, L ** 4
    a2 = a * a
    mrl = M * R / L2
    c_t = (8.0 * M * (2.0 * M - a2 * R / L2) * (1.0 + 2.0 * mrl))[:, None] - \
        a2 * np.sin(theta)[None, :] ** 2
    K = (L2 - (8.0 * M * M - a2) * R ** 2 / L2 + 4.0 * a2 * M * R ** 3 / L4)[:, None]
    HR = (R ** 2 / L4 * (L4 - 2.0 * L2 * M * R + a2 * R ** 2))[:, None]
    root = np.sqrt(K * K + c_t * HR)
    return float(max(np.max(np.abs((K - root) / c_t)),
                     np.max(np.abs((K + root) / c_t))))


def cfl_time_step(config: SolveConfig, cfl: float) -> float:
    """The reference driver's upper bound on the step
    (solver_driver.hpp:117-125): dt <= cfl h / v_max."""
    return cfl * config.spacing / maximum_coordinate_speed(config)


# Step of the workloads, in radial spacings.  At CFL 0.25 the driver's bound
# allows dt of about 2 h, where the semi-discrete system is unstable: in the
# reference build itself the Schwarzschild D8-4 state grows by 1e42 within
# 400 steps at dt = 0.2 h and stays bounded at 0.15 h; the Kerr D10-5 shapes
# are stable at 0.2 h.  0.1 h sits inside every measured limit and far
# inside the CFL bound, so the configurations' CFL 0.25 holds as the
# driver's check.
STEP_OVER_SPACING = 0.1


def time_step(config: SolveConfig, cfl: float) -> float:
    """Step of a workload: 0.1 h, or the CFL bound if that is smaller."""
    return min(cfl_time_step(config, cfl), STEP_OVER_SPACING * config.spacing)


def dissipation_bound(discretization: int, step_over_spacing: float) -> float:
    """Largest sigma with dt/h <= 0.8 * 2.785 / (sigma * rho)."""
    return SAFETY * RK4_NEGATIVE_AXIS / (SPECTRAL_BOUND[discretization] *
                                          step_over_spacing)


def compactified(config: SolveConfig, r_center: float, r_width: float):
    L2 = config.compactification_length ** 2
    return L2 / r_center, L2 * r_width / (r_center * r_center)


def kerr_ringdown(seed: int = 20260101, radial_points: int = 1025,
                  cfl: float = 0.25):
    """Plain FP64 linear Kerr ringdown: a = 0.7, M = 1, D10-5, m = -4..4,
    ell <= 16 (ntheta 25 by the exact-product rule), Gaussian pulses
    (centre 8M, width 0.8M, amplitude 1e-3) in ell = 2, m = +-2 with seeded
    complex amplitudes.  Returns (config, pulse, dt)."""
    base = SolveConfig(mass=1.0, spin=0.7, compactification_length=1.0,
                       radial_points=radial_points, theta_nodes=25,
                       ell_max_first=16, ell_max_second=16,
                       modes=tuple(range(-4, 5)), reduction_damping=0.1,
                       dissipation=0.0, discretization=D105)
    dt = time_step(base, cfl)
    sigma = min(0.005, 0.9 * dissipation_bound(D105, dt / base.spacing))
    config = replace(base, dissipation=sigma)
    rng = np.random.Generator(np.random.PCG64(seed))
    center, width = compactified(config, 8.0, 0.8)
    modes = []
    for m in (-2, 2):
        amp = 1e-3 * complex(rng.standard_normal(), rng.standard_normal())
        modes.append((2, m, amp))
    return config, GaussianPulse(center=center, width=width, modes=modes), dt


def schwarzschild_quadrupole(seed: int = 20260101):
    """Plain FP64 linear Schwarzschild, nr = 257, D8-4, m = +-2 (closure),
    ell = 2..8, ntheta 13; ell = 2, m = 2 pulse of amplitude
    1e-3 (N(0,1) + i N(0,1)) at r = 10M, width 1M; CFL 0.25."""
    base = SolveConfig(mass=1.0, spin=0.0, compactification_length=1.0,
                       radial_points=257, theta_nodes=13, ell_max_first=8,
                       ell_max_second=8, modes=(-2, 2), reduction_damping=0.1,
                       dissipation=0.0, discretization=D84)
    dt = time_step(base, 0.25)
    sigma = min(0.005, 0.9 * dissipation_bound(D84, dt / base.spacing))
    config = replace(base, dissipation=sigma)
    rng = np.random.Generator(np.random.PCG64(seed))
    center, width = compactified(config, 10.0, 1.0)
    amp = 1e-3 * complex(rng.standard_normal(), rng.standard_normal())
    return config, GaussianPulse(center=center, width=width,
                                 modes=[(2, 2, amp)]), dt


def second_order_self_coupling(seed: int = 20260101, radial_points: int = 1025,
                               cfl: float = 0.25, source_start_time: float = 0.0):
    """Quadratic-source run: a = 0.9, M = 1, D10-5, parents m = +-2 with
    ell <= 10, targets m in {-4, 0, 4} with ell <= 20, ntheta 48, source
    Unrestricted from `source_start_time`; seeded Gaussian parents in
    ell = 2 (centre 10M, width 1M, amplitude 1e-2).  Returns
    (config, pulse, dt)."""
    from . import SOURCE_UNRESTRICTED

    base = SolveConfig(mass=1.0, spin=0.9, compactification_length=1.0,
                       radial_points=radial_points, theta_nodes=48,
                       ell_max_first=10, ell_max_second=20,
                       modes=(-4, -2, 0, 2, 4), parents=(-2, 2),
                       targets=(-4, 0, 4), reduction_damping=0.1,
                       dissipation=0.0, discretization=D105,
                       source_mode=SOURCE_UNRESTRICTED,
                       source_start_time=source_start_time)
    dt = time_step(base, cfl)
    sigma = min(0.005, 0.9 * dissipation_bound(D105, dt / base.spacing))
    config = replace(base, dissipation=sigma)
    rng = np.random.Generator(np.random.PCG64(seed))
    center, width = compactified(config, 10.0, 1.0)
    modes = [(2, m, 1e-2 * complex(rng.standard_normal(), rng.standard_normal()))
             for m in (-2, 2)]
    return config, GaussianPulse(center=center, width=width, modes=modes), dt


def uneven_instance(rng: np.random.Generator, cfl: float = 0.25):
    """One solve of the batched uneven-instance mix: spin U[0, 0.95],
    nr from {257, 513, 1025, 2049}, D10-5, ell_max U{8..20}, m = -2..2
    (ntheta by the exact-product rule), a Gaussian in ell = 2, m = +-2 with
    centre U[6M, 14M], width U[0.5M, 1.5M] and amplitude 1e-3."""
    spin = float(rng.uniform(0.0, 0.95))
    nr = int(rng.choice([257, 513, 1025, 2049]))
    ell = int(rng.integers(8, 21))
    base = SolveConfig(mass=1.0, spin=spin, compactification_length=1.0,
                       radial_points=nr, theta_nodes=(3 * ell + 2) // 2,
                       ell_max_first=ell, ell_max_second=ell,
                       modes=(-2, -1, 0, 1, 2), reduction_damping=0.1,
                       dissipation=0.0, discretization=D105)
    dt = time_step(base, cfl)
    sigma = min(0.005, 0.9 * dissipation_bound(D105, dt / base.spacing))
    config = replace(base, dissipation=sigma)
    center, width = compactified(config, float(rng.uniform(6.0, 14.0)),
                                 float(rng.uniform(0.5, 1.5)))
    modes = [(2, m, 1e-3 * complex(rng.standard_normal(), rng.standard_normal()))
             for m in (-2, 2)]
    return config, GaussianPulse(center=center, width=width, modes=modes), dt


def extremal_kerr(seed: int = 20260101, cfl: float = 0.25):
    """Near-extremal linear Kerr solve of the serving mix: a = 0.99, M = 1,
    nr = 4097, D10-5, m = -4..4, ell <= 24 (ntheta 37 by the exact-product
    rule), Gaussian pulses (centre 8M, width 0.8M, amplitude 1e-3) in
    ell = 2, m = +-2; CFL 0.25."""
    base = SolveConfig(mass=1.0, spin=0.99, compactification_length=1.0,
                       radial_points=4097, theta_nodes=37, ell_max_first=24,
                       ell_max_second=24, modes=tuple(range(-4, 5)),
                       reduction_damping=0.1, dissipation=0.0,
                       discretization=D105)
    dt = time_step(base, cfl)
    sigma = min(0.005, 0.9 * dissipation_bound(D105, dt / base.spacing))
    config = replace(base, dissipation=sigma)
    rng = np.random.Generator(np.random.PCG64(seed))
    center, width = compactified(config, 8.0, 0.8)
    modes = [(2, m, 1e-3 * complex(rng.standard_normal(), rng.standard_normal()))
             for m in (-2, 2)]
    return config, GaussianPulse(center=center, width=width, modes=modes), dt


SERVING_KINDS = ("schwarzschild", "kerr_ringdown", "second_order", "extremal")


def serving_mix(count: int, seed: int = 20260101):
    """Request stream of the serving configuration: 40 % Schwarzschild
    quadrupoles (nr 257, D8-4), 30 % Kerr ringdowns (a 0.7, nr 1025), 20 %
    quadratic-source solves (a 0.9, nr 1025, ntheta 48, ell <= 10 / 20, the
    source active from t = 0) and 10 % near-extremal Kerr solves (a 0.99,
    nr 4097, ell <= 24); each entry (kind, config, pulse, dt)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i in range(count):
        u = rng.uniform()
        if u < 0.4:
            config, pulse, dt = schwarzschild_quadrupole(seed + i)
            out.append(("schwarzschild", config, pulse, dt))
        elif u < 0.7:
            config, pulse, dt = kerr_ringdown(seed + i)
            out.append(("kerr_ringdown", config, pulse, dt))
        elif u < 0.9:
            config, pulse, dt = second_order_self_coupling(seed + i)
            out.append(("second_order", config, pulse, dt))
        else:
            config, pulse, dt = extremal_kerr(seed + i)
            out.append(("extremal", config, pulse, dt))
    return out


def uneven_batch(count: int = 256, seed: int = 20260101):
    """The batched uneven-instance configuration: `count` solves drawn by
    ``uneven_instance`` from one seeded stream; each (config, pulse, dt)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return [uneven_instance(rng) for _ in range(count)]


def band_noise(config: SolveConfig, seed: int, scale: float = 1e-6):
    """Seeded complex N(0,1) * scale nodal noise on the first-order psi field
    of every parent mode; set_state projects it onto each fixed-m band."""
    rng = np.random.Generator(np.random.PCG64(seed))
    noise = np.zeros(config.shape(), dtype=np.complex128)
    modes = list(config.modes)
    for m in config.parent_list():
        i = modes.index(m)
        shape = (config.radial_points, config.theta_nodes)
        noise[i, 2] = scale * (rng.standard_normal(shape) +
                               1j * rng.standard_normal(shape))
    return noise


def grid_points(config: SolveConfig) -> int:
    """Reference grid-point count per step: modes * nr * ntheta
    (solver_driver.hpp:323-341)."""
    return len(config.modes) * config.radial_points * config.theta_nodes


def modal_values(config: SolveConfig) -> int:
    """Evolved complex values of one solve in band storage:
    3 fields * nr * sum over parent m of n_ell(m)."""
    total = 0
    for m in config.parent_list():
        total += config.ell_max_first - max(2, abs(m)) + 1
    return 3 * config.radial_points * total


def state_bytes(config: SolveConfig) -> int:
    return 16 * len(config.modes) * FIELD_COUNT * config.radial_points * \
        config.theta_nodes
