"""Python host binding of the B200 teuk-kokkos RK4 engine (ctypes over the
C ABI declared in include/teuk_b200.h).

The classes mirror the reference's C++ interface: ``Pipeline`` is
``teuk::SpatialPipeline`` (include/teuk/spatial_pipeline.hpp:144-1364) for one
solve and ``Batch`` packs many solves into one set of stage launches.  State
arrays are complex128 in the reference's (mode, field, radial, theta) order.
Arrays may be numpy (host) or torch CUDA tensors (device).  There is no CPU
fallback: the first call into the engine (``library()``, creating a
``Pipeline``, ``Batch`` or ``Server``) fails when libteuk_b200.so is missing.
The structures and configuration classes load nothing, so host-only code can
describe solves without mapping the engine.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from pathlib import Path
from typing import Iterable, Sequence

import threading

import numpy as np

_PACKAGE = Path(__file__).resolve().parent.parent
LIBRARY_PATH = _PACKAGE / "lib" / "libteuk_b200.so"

OK = 0
ERR_INVALID_ARGUMENT = -1
ERR_RUNTIME = -2
ERR_CUDA = -3
ERR_UNSUPPORTED = -4
ERR_OUT_OF_MEMORY = -5

HOST = 0
DEVICE = 1

D42, D84, D105 = 0, 1, 2
FREE_DAMPED, STAGE_CONSTRAINED = 0, 1
SOURCE_DISABLED, SOURCE_CONSTRAINT_AWARE, SOURCE_UNRESTRICTED = 0, 1, 2
FIELD_COUNT = 13
SCRI, HORIZON = 0, 1

DISCRETIZATION_NAMES = {"d4-2": D42, "d8-4": D84, "d10-5": D105}


class TeukError(RuntimeError):
    """Raised for any non-zero status; ``status`` holds the code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


class InvalidArgument(TeukError, ValueError):
    """std::invalid_argument in the reference."""


class Unsupported(TeukError):
    """A valid reference input that the B200 path does not run yet."""


class _Config(ctypes.Structure):
    _fields_ = [
        ("abi_version", ctypes.c_int),
        ("mass", ctypes.c_double),
        ("spin", ctypes.c_double),
        ("compactification_length", ctypes.c_double),
        ("radial_points", ctypes.c_int),
        ("theta_nodes", ctypes.c_int),
        ("ell_max_first", ctypes.c_int),
        ("ell_max_second", ctypes.c_int),
        ("mode_count", ctypes.c_int),
        ("modes", ctypes.POINTER(ctypes.c_int)),
        ("parent_count", ctypes.c_int),
        ("parents", ctypes.POINTER(ctypes.c_int)),
        ("target_count", ctypes.c_int),
        ("targets", ctypes.POINTER(ctypes.c_int)),
        ("reduction_damping", ctypes.c_double),
        ("dissipation", ctypes.c_double),
        ("reduction", ctypes.c_int),
        ("discretization", ctypes.c_int),
        ("source_mode", ctypes.c_int),
        ("source_start_time", ctypes.c_double),
        ("normalized_constraint_tolerance", ctypes.c_double),
        ("required_consecutive_passes", ctypes.c_int),
    ]


class Activation(ctypes.Structure):
    _fields_ = [
        ("active", ctypes.c_int),
        ("activation_time", ctypes.c_double),
        ("consecutive_passes", ctypes.c_int),
        ("last_eligibility_time", ctypes.c_double),
    ]


class _ServerOptions(ctypes.Structure):
    _fields_ = [
        ("abi_version", ctypes.c_int),
        ("hbm_budget_bytes", ctypes.c_size_t),
        ("max_active", ctypes.c_int),
        ("graph", ctypes.c_int),
        ("precision", ctypes.c_int),
    ]


class ServerStats(ctypes.Structure):
    _fields_ = [
        ("queued", ctypes.c_int),
        ("active", ctypes.c_int),
        ("finished", ctypes.c_int),
        ("steps", ctypes.c_longlong),
        ("grid_point_updates", ctypes.c_double),
        ("device_seconds", ctypes.c_double),
        ("resident_bytes", ctypes.c_size_t),
        ("rebuilds", ctypes.c_int),
        ("rebuild_seconds", ctypes.c_double),
    ]


class _GaussianMode(ctypes.Structure):
    _fields_ = [
        ("ell", ctypes.c_int),
        ("m", ctypes.c_int),
        ("amplitude_real", ctypes.c_double),
        ("amplitude_imag", ctypes.c_double),
    ]


class _Gaussian(ctypes.Structure):
    _fields_ = [
        ("center", ctypes.c_double),
        ("width", ctypes.c_double),
        ("compact_support", ctypes.c_int),
        ("mode_count", ctypes.c_int),
        ("modes", ctypes.POINTER(_GaussianMode)),
    ]


MAX_MODES = 64
MAX_SEEDS = 64
PATH_CAPACITY = 1024


class RunConfig(ctypes.Structure):
    """teuk_b200_run_config: a parsed and validated .cfg run."""
    _fields_ = [
        ("abi_version", ctypes.c_int),
        ("mass", ctypes.c_double),
        ("spin", ctypes.c_double),
        ("compactification_length", ctypes.c_double),
        ("radial_points", ctypes.c_int),
        ("theta_nodes", ctypes.c_int),
        ("ell_max_first", ctypes.c_int),
        ("ell_max_second", ctypes.c_int),
        ("mode_count", ctypes.c_int),
        ("modes", ctypes.c_int * MAX_MODES),
        ("parent_count", ctypes.c_int),
        ("parents", ctypes.c_int * MAX_MODES),
        ("target_count", ctypes.c_int),
        ("targets", ctypes.c_int * MAX_MODES),
        ("reduction_damping", ctypes.c_double),
        ("dissipation", ctypes.c_double),
        ("reduction", ctypes.c_int),
        ("discretization", ctypes.c_int),
        ("source_mode", ctypes.c_int),
        ("source_start_time", ctypes.c_double),
        ("normalized_constraint_tolerance", ctypes.c_double),
        ("required_consecutive_passes", ctypes.c_int),
        ("final_time", ctypes.c_double),
        ("steps", ctypes.c_int),
        ("cfl", ctypes.c_double),
        ("time_step", ctypes.c_double),
        ("initial_data_type", ctypes.c_int),
        ("center", ctypes.c_double),
        ("width", ctypes.c_double),
        ("compact_support", ctypes.c_int),
        ("seed_count", ctypes.c_int),
        ("seeds", _GaussianMode * MAX_SEEDS),
        ("checkpoint_directory", ctypes.c_char * PATH_CAPACITY),
        ("output_directory", ctypes.c_char * PATH_CAPACITY),
        ("diagnostic_every", ctypes.c_int),
        ("checkpoint_every", ctypes.c_int),
    ]

    def solve_config(self) -> "SolveConfig":
        return SolveConfig(
            mass=self.mass, spin=self.spin,
            compactification_length=self.compactification_length,
            radial_points=self.radial_points, theta_nodes=self.theta_nodes,
            ell_max_first=self.ell_max_first, ell_max_second=self.ell_max_second,
            modes=tuple(self.modes[:self.mode_count]),
            parents=tuple(self.parents[:self.parent_count]),
            targets=tuple(self.targets[:self.target_count]),
            reduction_damping=self.reduction_damping,
            dissipation=self.dissipation, reduction=self.reduction,
            discretization=self.discretization, source_mode=self.source_mode,
            source_start_time=self.source_start_time,
            normalized_constraint_tolerance=self.normalized_constraint_tolerance,
            required_consecutive_passes=self.required_consecutive_passes)

    def pulse(self) -> "GaussianPulse":
        modes = [(s.ell, s.m, complex(s.amplitude_real, s.amplitude_imag))
                 for s in self.seeds[:self.seed_count]]
        return GaussianPulse(center=self.center, width=self.width, modes=modes,
                             compact_support=bool(self.compact_support))


def _override_array(overrides):
    items = [o.encode() for o in overrides]
    return (ctypes.c_char_p * max(len(items), 1))(*items), len(items)


class Norm(ctypes.Structure):
    _fields_ = [("rms", ctypes.c_double), ("maximum", ctypes.c_double)]


class Diagnostics(ctypes.Structure):
    """teuk_b200_diagnostics (PipelineDiagnosticsReport)."""
    _fields_ = [
        ("state", Norm * FIELD_COUNT),
        ("rhs", Norm * FIELD_COUNT),
        ("first_reduction_constraint", Norm),
        ("second_reduction_constraint", Norm),
        ("source_over_r3", Norm),
        ("forcing", Norm),
        ("independent_reconstruction_constraint_maximum", ctypes.c_double),
        ("constraint_absolute_maximum", ctypes.c_double * 3),
        ("constraint_normalized_maximum", ctypes.c_double * 3),
        ("constraint_weighted_rms", ctypes.c_double * 3),
        ("constraint_normalized_weighted", ctypes.c_double * 3),
        ("constraint_controlling_normalized", ctypes.c_double),
        ("constraints_finite", ctypes.c_int),
        ("activation", Activation),
        ("second_order_source_active", ctypes.c_int),
        ("point_count", ctypes.c_size_t),
        ("scri_finite", ctypes.c_int),
        ("horizon_finite", ctypes.c_int),
        ("all_finite", ctypes.c_int),
    ]

    def norms(self):
        """Flat list of every (rms, maximum) pair in report order."""
        out = [(n.rms, n.maximum) for n in self.state]
        out += [(n.rms, n.maximum) for n in self.rhs]
        for name in ("first_reduction_constraint", "second_reduction_constraint",
                     "source_over_r3", "forcing"):
            n = getattr(self, name)
            out.append((n.rms, n.maximum))
        return out


class WaveformRecord(ctypes.Structure):
    _fields_ = [
        ("boundary", ctypes.c_int),
        ("order", ctypes.c_int),
        ("m", ctypes.c_int),
        ("ell", ctypes.c_int),
        ("rescaled_real", ctypes.c_double),
        ("rescaled_imag", ctypes.c_double),
        ("endpoint_real", ctypes.c_double),
        ("endpoint_imag", ctypes.c_double),
    ]


ABI_VERSION = 1

KERNEL_AUTO, KERNEL_TILE = 0, 1
PRECISION_FP64, PRECISION_SPLIT = 0, 1


class _BatchOptions(ctypes.Structure):
    _fields_ = [
        ("abi_version", ctypes.c_int),
        ("stage_kernel", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("strip_rows", ctypes.c_int),
        ("autotune", ctypes.c_int),
    ]


@dataclass
class LaunchOptions:
    """teuk_b200_batch_options: stage kernel choice, transform precision,
    streaming strip length (0: built-in or tuned), autotuning."""

    stage_kernel: int = KERNEL_AUTO
    precision: int = PRECISION_FP64
    strip_rows: int = 0
    autotune: bool = False

    def to_struct(self):
        return _BatchOptions(ABI_VERSION, self.stage_kernel, self.precision,
                             self.strip_rows, int(self.autotune))


@dataclass
class SolveConfig:
    """SpatialPipeline constructor arguments + ModeRegistry lists."""

    mass: float = 1.0
    spin: float = 0.0
    compactification_length: float = 1.0
    radial_points: int = 65
    theta_nodes: int = 7
    ell_max_first: int = 4
    ell_max_second: int = 4
    modes: Sequence[int] = (-2, 2)
    parents: Sequence[int] | None = None
    targets: Sequence[int] | None = None
    reduction_damping: float = 0.1
    dissipation: float = 0.0
    reduction: int = FREE_DAMPED
    discretization: int = D42
    source_mode: int = SOURCE_DISABLED
    source_start_time: float = 0.0
    normalized_constraint_tolerance: float = 0.0
    required_consecutive_passes: int = 1

    @property
    def horizon_radius(self) -> float:
        r_plus = self.mass + math.sqrt(self.mass * self.mass - self.spin * self.spin)
        return self.compactification_length ** 2 / r_plus

    @property
    def spacing(self) -> float:
        return self.horizon_radius / (self.radial_points - 1)

    def parent_list(self):
        return list(self.modes if self.parents is None else self.parents)

    def target_list(self):
        return list(self.modes if self.targets is None else self.targets)

    def shape(self):
        return (len(self.modes), FIELD_COUNT, self.radial_points, self.theta_nodes)

    def value_count(self) -> int:
        return int(np.prod(self.shape()))

    def to_struct(self):
        """ctypes struct plus the arrays it points into (keep them alive)."""
        modes = (ctypes.c_int * len(self.modes))(*self.modes)
        parents_list = self.parent_list()
        targets_list = self.target_list()
        parents = (ctypes.c_int * len(parents_list))(*parents_list)
        targets = (ctypes.c_int * len(targets_list))(*targets_list)
        s = _Config(
            ABI_VERSION, self.mass, self.spin, self.compactification_length,
            self.radial_points, self.theta_nodes, self.ell_max_first,
            self.ell_max_second, len(self.modes), modes, len(parents_list),
            parents, len(targets_list), targets, self.reduction_damping,
            self.dissipation, self.reduction, self.discretization,
            self.source_mode, self.source_start_time,
            self.normalized_constraint_tolerance,
            self.required_consecutive_passes)
        return s, (modes, parents, targets)


@dataclass
class GaussianPulse:
    """PipelineGaussianPulse (include/teuk/pipeline_initial_data.hpp:29-57);
    center/width are compactified radii."""

    center: float
    width: float
    modes: Sequence[tuple] = field(default_factory=lambda: [(2, 2, 1e-3 + 0j)])
    compact_support: bool = False

    def to_struct(self):
        items = (_GaussianMode * len(self.modes))()
        for i, (ell, m, amp) in enumerate(self.modes):
            amp = complex(amp)
            items[i] = _GaussianMode(int(ell), int(m), amp.real, amp.imag)
        return _Gaussian(self.center, self.width, int(self.compact_support),
                         len(self.modes), items), items


def _load() -> ctypes.CDLL:
    if not LIBRARY_PATH.exists():
        raise ImportError(
            f"{LIBRARY_PATH} is missing: build it with "
            "`python teuk-kokkos_b200/build.py` (no CPU fallback exists)")
    lib = ctypes.CDLL(str(LIBRARY_PATH))
    P = ctypes.c_void_p
    D = ctypes.c_double
    I = ctypes.c_int
    SZ = ctypes.c_size_t
    DP = ctypes.POINTER(ctypes.c_double)
    sig = {
        "teuk_b200_last_error": ([], ctypes.c_char_p),
        "teuk_b200_abi_version": ([], I),
        "teuk_b200_set_device": ([I], I),
        "teuk_b200_get_device": ([ctypes.POINTER(I)], I),
        "teuk_b200_create": ([ctypes.POINTER(_Config), ctypes.POINTER(P)], I),
        "teuk_b200_create_with_options": ([ctypes.POINTER(_Config),
                                           ctypes.POINTER(_BatchOptions),
                                           ctypes.POINTER(P)], I),
        "teuk_b200_test_withhold_chunk": ([I], I),
        "teuk_b200_batch_create_with_options": ([ctypes.POINTER(_Config), I,
                                                 ctypes.POINTER(_BatchOptions),
                                                 ctypes.POINTER(P)], I),
        "teuk_b200_batch_strip_rows": ([P, ctypes.POINTER(I), I,
                                        ctypes.POINTER(I)], I),
        "teuk_b200_destroy": ([P], I),
        "teuk_b200_shape": ([P, ctypes.POINTER(SZ)], I),
        "teuk_b200_set_state": ([P, P, SZ, I], I),
        "teuk_b200_get_state": ([P, P, SZ, I], I),
        "teuk_b200_evaluate_rhs": ([P, P, P, SZ, D, I], I),
        "teuk_b200_step": ([P, D, D, I], I),
        "teuk_b200_step_static_scratch": ([P, D, D, I], I),
        "teuk_b200_initialize_gaussian": ([P, ctypes.POINTER(_Gaussian)], I),
        "teuk_b200_sample_endpoint": ([P, ctypes.POINTER(WaveformRecord), SZ,
                                       ctypes.POINTER(SZ)], I),
        "teuk_b200_get_activation": ([P, ctypes.POINTER(Activation)], I),
        "teuk_b200_restore_activation": ([P, ctypes.POINTER(Activation)], I),
        "teuk_b200_reset_activation": ([P], I),
        "teuk_b200_set_stream": ([P, P], I),
        "teuk_b200_synchronize": ([P], I),
        "teuk_b200_diagnostics_sample": ([P, ctypes.POINTER(Diagnostics)], I),
        "teuk_b200_checkpoint_write": ([P, ctypes.c_char_p, D, D,
                                        ctypes.c_uint64], I),
        "teuk_b200_checkpoint_load": ([P, ctypes.c_char_p, D, DP,
                                       ctypes.POINTER(ctypes.c_uint64)], I),
        "teuk_b200_footprint_bytes": ([ctypes.POINTER(_Config),
                                       ctypes.POINTER(SZ)], I),
        "teuk_b200_batch_create": ([ctypes.POINTER(_Config), I,
                                    ctypes.POINTER(P)], I),
        "teuk_b200_batch_destroy": ([P], I),
        "teuk_b200_batch_size": ([P, ctypes.POINTER(I)], I),
        "teuk_b200_batch_shape": ([P, I, ctypes.POINTER(SZ)], I),
        "teuk_b200_batch_set_state": ([P, I, P, SZ, I], I),
        "teuk_b200_batch_get_state": ([P, I, P, SZ, I], I),
        "teuk_b200_batch_initialize_gaussian": ([P, I,
                                                 ctypes.POINTER(_Gaussian)], I),
        "teuk_b200_batch_step": ([P, DP, I, I], I),
        "teuk_b200_batch_sample_endpoint": ([P, I,
                                             ctypes.POINTER(WaveformRecord),
                                             SZ, ctypes.POINTER(SZ)], I),
        "teuk_b200_batch_endpoint_modal": ([P, P, SZ, ctypes.POINTER(SZ), I], I),
        "teuk_b200_batch_set_stream": ([P, P], I),
        "teuk_b200_batch_synchronize": ([P], I),
        "teuk_b200_batch_launches_per_step": ([P, ctypes.POINTER(I)], I),
        "teuk_b200_batch_stage_kernels": ([P, ctypes.POINTER(I),
                                           ctypes.POINTER(I)], I),
        "teuk_b200_parse_run_config": ([ctypes.c_char_p,
                                        ctypes.POINTER(ctypes.c_char_p), I,
                                        ctypes.POINTER(RunConfig)], I),
        "teuk_b200_resolved_config": ([ctypes.c_char_p,
                                       ctypes.POINTER(ctypes.c_char_p), I,
                                       ctypes.c_char_p, SZ,
                                       ctypes.POINTER(SZ)], I),
        "teuk_b200_server_create": ([ctypes.POINTER(_ServerOptions),
                                     ctypes.POINTER(P)], I),
        "teuk_b200_server_destroy": ([P], I),
        "teuk_b200_server_submit": ([P, ctypes.POINTER(_Config),
                                     ctypes.POINTER(_Gaussian), D, I,
                                     ctypes.POINTER(ctypes.c_uint64)], I),
        "teuk_b200_server_advance": ([P, I, ctypes.POINTER(I)], I),
        "teuk_b200_server_result": ([P, ctypes.c_uint64,
                                     ctypes.POINTER(WaveformRecord), SZ,
                                     ctypes.POINTER(SZ), DP], I),
        "teuk_b200_server_stats_get": ([P, ctypes.POINTER(ServerStats)], I),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return lib


class _Library:
    """The engine library, mapped on first use.  The structures, constants
    and configuration classes above need no library, so host-only code (the
    oracle bindings, workload descriptions) can use them without mapping the
    engine into its process.  Any call into the engine loads it, and fails
    loudly when it is missing: there is no CPU fallback."""

    def __init__(self):
        self._cdll = None
        self._lock = threading.Lock()

    def load(self) -> ctypes.CDLL:
        if self._cdll is None:
            with self._lock:
                if self._cdll is None:
                    self._cdll = _load()
        return self._cdll

    def loaded(self) -> bool:
        return self._cdll is not None

    def __getattr__(self, name):
        return getattr(self.load(), name)


_lib = _Library()


def library() -> ctypes.CDLL:
    """The mapped engine library (loads it on first use)."""
    return _lib.load()


def set_device(device: int):
    """Select the CUDA device of the engine for this thread
    (teuk_b200_set_device): the engine's statically linked CUDA runtime does
    not follow torch.cuda.set_device."""
    _check(_lib.teuk_b200_set_device(int(device)))


def get_device() -> int:
    d = ctypes.c_int()
    _check(_lib.teuk_b200_get_device(ctypes.byref(d)))
    return d.value


def test_withhold_chunk(chunk: int):
    """Failure-detection test hook (teuk_b200_test_withhold_chunk): batches
    built while chunk >= 0 withhold that chunk from CTA 0 of their stage-1
    streaming launches; -1 switches it off."""
    _check(_lib.teuk_b200_test_withhold_chunk(chunk))


def _check(status: int):
    if status == OK:
        return
    message = _lib.teuk_b200_last_error().decode()
    if status == ERR_INVALID_ARGUMENT:
        raise InvalidArgument(status, message)
    if status == ERR_UNSUPPORTED:
        raise Unsupported(status, message)
    raise TeukError(status, message)


def _pointer(array, writable: bool, count: int):
    """(pointer, memory kind, keepalive) for a complex128 buffer."""
    try:
        import torch
    except ImportError:  # pragma: no cover - torch is in the image
        torch = None
    if torch is not None and isinstance(array, torch.Tensor):
        if array.dtype != torch.complex128 or not array.is_contiguous():
            raise ValueError("state tensors must be contiguous complex128")
        if array.numel() != count:
            raise ValueError("state tensor size does not match the shape")
        kind = DEVICE if array.is_cuda else HOST
        return ctypes.c_void_p(array.data_ptr()), kind, array
    arr = np.asarray(array)
    if arr.dtype != np.complex128 or not arr.flags.c_contiguous:
        raise ValueError("state arrays must be C-contiguous complex128")
    if writable and not arr.flags.writeable:
        raise ValueError("output array is read-only")
    if arr.size != count:
        raise ValueError("state array size does not match the shape")
    return ctypes.c_void_p(arr.ctypes.data), HOST, arr


def _records(buffer, count):
    out = []
    for i in range(count):
        r = buffer[i]
        out.append({
            "boundary": "scri" if r.boundary == SCRI else "horizon",
            "order": r.order, "m": r.m, "ell": r.ell,
            "rescaled": complex(r.rescaled_real, r.rescaled_imag),
            "endpoint": complex(r.endpoint_real, r.endpoint_imag),
        })
    return out


def parse_run_config(text: str, overrides=()) -> RunConfig:
    """Parse and validate a teuk_solver .cfg text (+ key=value overrides)."""
    arr, n = _override_array(overrides)
    out = RunConfig()
    _check(_lib.teuk_b200_parse_run_config(text.encode(), arr, n,
                                           ctypes.byref(out)))
    return out


def resolved_config(text: str, overrides=()) -> str:
    """resolved_config.cfg body of a .cfg text."""
    arr, n = _override_array(overrides)
    length = ctypes.c_size_t()
    _check(_lib.teuk_b200_resolved_config(text.encode(), arr, n, None, 0,
                                          ctypes.byref(length)))
    buf = ctypes.create_string_buffer(length.value + 1)
    _check(_lib.teuk_b200_resolved_config(text.encode(), arr, n, buf,
                                          length.value + 1,
                                          ctypes.byref(length)))
    return buf.value.decode()


def footprint_bytes(config: SolveConfig) -> int:
    s, keep = config.to_struct()
    out = ctypes.c_size_t()
    _check(_lib.teuk_b200_footprint_bytes(ctypes.byref(s), ctypes.byref(out)))
    return out.value


class Pipeline:
    """One solve (teuk::SpatialPipeline)."""

    def __init__(self, config: SolveConfig, options: LaunchOptions | None = None):
        self.config = config
        s, keep = config.to_struct()
        handle = ctypes.c_void_p()
        if options is None:
            _check(_lib.teuk_b200_create(ctypes.byref(s), ctypes.byref(handle)))
        else:
            o = options.to_struct()
            _check(_lib.teuk_b200_create_with_options(
                ctypes.byref(s), ctypes.byref(o), ctypes.byref(handle)))
        self._handle = handle

    def close(self):
        if getattr(self, "_handle", None):
            _lib.teuk_b200_destroy(self._handle)
            self._handle = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def shape(self):
        dims = (ctypes.c_size_t * 4)()
        _check(_lib.teuk_b200_shape(self._handle, dims))
        return tuple(int(d) for d in dims)

    def set_state(self, state):
        ptr, kind, _keep = _pointer(state, False, self.config.value_count())
        _check(_lib.teuk_b200_set_state(self._handle, ptr,
                                        self.config.value_count(), kind))

    def get_state(self, out=None):
        if out is None:
            out = np.zeros(self.shape, dtype=np.complex128)
        ptr, kind, _keep = _pointer(out, True, self.config.value_count())
        _check(_lib.teuk_b200_get_state(self._handle, ptr,
                                        self.config.value_count(), kind))
        return out

    def evaluate_rhs(self, stage, out=None, time: float = 0.0):
        if out is None:
            out = np.zeros(self.shape, dtype=np.complex128)
        src, kind, _k1 = _pointer(stage, False, self.config.value_count())
        dst, kind2, _k2 = _pointer(out, True, self.config.value_count())
        if kind != kind2:
            raise ValueError("stage and output must live in the same memory")
        _check(_lib.teuk_b200_evaluate_rhs(self._handle, src, dst,
                                           self.config.value_count(), time,
                                           kind))
        return out

    def step(self, time: float, dt: float, steps: int = 1):
        _check(_lib.teuk_b200_step(self._handle, time, dt, steps))

    def step_static_scratch(self, time: float, dt: float, steps: int = 1):
        """teuk_b200_step with the RK slopes in the library's static device
        array: no device allocation (linear pipelines up to 524,288 band
        values; calls must not overlap on one device)."""
        _check(_lib.teuk_b200_step_static_scratch(self._handle, time, dt,
                                                  steps))

    def initialize_gaussian(self, pulse: GaussianPulse):
        s, keep = pulse.to_struct()
        _check(_lib.teuk_b200_initialize_gaussian(self._handle, ctypes.byref(s)))

    def sample_endpoint(self):
        count = ctypes.c_size_t()
        cap = 4 * len(self.config.modes) * (self.config.ell_max_first +
                                             self.config.ell_max_second + 2)
        buf = (WaveformRecord * cap)()
        _check(_lib.teuk_b200_sample_endpoint(self._handle, buf, cap,
                                              ctypes.byref(count)))
        return _records(buf, count.value)

    def activation(self) -> Activation:
        a = Activation()
        _check(_lib.teuk_b200_get_activation(self._handle, ctypes.byref(a)))
        return a

    def diagnostics(self) -> Diagnostics:
        """Device-side PipelineDiagnostics sample of the current state."""
        d = Diagnostics()
        _check(_lib.teuk_b200_diagnostics_sample(self._handle, ctypes.byref(d)))
        return d

    def checkpoint_write(self, directory, time_step: float, time: float,
                         step: int):
        """Write the reference's checkpoint format v5 into `directory`."""
        _check(_lib.teuk_b200_checkpoint_write(
            self._handle, str(directory).encode(), time_step, time, step))

    def checkpoint_load(self, directory, time_step: float):
        """Verified load of a v5 checkpoint; returns (time, step)."""
        t = ctypes.c_double()
        n = ctypes.c_uint64()
        _check(_lib.teuk_b200_checkpoint_load(
            self._handle, str(directory).encode(), time_step, ctypes.byref(t),
            ctypes.byref(n)))
        return t.value, n.value

    def restore_activation(self, a: Activation):
        _check(_lib.teuk_b200_restore_activation(self._handle, ctypes.byref(a)))

    def reset_activation(self):
        _check(_lib.teuk_b200_reset_activation(self._handle))

    def set_stream(self, stream_handle: int | None):
        _check(_lib.teuk_b200_set_stream(self._handle,
                                         ctypes.c_void_p(stream_handle or 0)))

    def synchronize(self):
        _check(_lib.teuk_b200_synchronize(self._handle))


class Batch:
    """Many independent solves advanced by the same stage launches."""

    def __init__(self, configs: Iterable[SolveConfig],
                 options: LaunchOptions | None = None):
        self.configs = list(configs)
        structs = (_Config * len(self.configs))()
        keep = []
        for i, c in enumerate(self.configs):
            s, k = c.to_struct()
            structs[i] = s
            keep.append(k)
        handle = ctypes.c_void_p()
        if options is None:
            _check(_lib.teuk_b200_batch_create(structs, len(self.configs),
                                               ctypes.byref(handle)))
        else:
            o = options.to_struct()
            _check(_lib.teuk_b200_batch_create_with_options(
                structs, len(self.configs), ctypes.byref(o),
                ctypes.byref(handle)))
        self._handle = handle

    def strip_rows(self) -> list[int]:
        """Streaming strip length per launch group (0: tile-kernel group)."""
        n = ctypes.c_int()
        _check(_lib.teuk_b200_batch_strip_rows(self._handle, None, 0,
                                               ctypes.byref(n)))
        out = (ctypes.c_int * max(n.value, 1))()
        _check(_lib.teuk_b200_batch_strip_rows(self._handle, out, n.value,
                                               ctypes.byref(n)))
        return list(out[:n.value])

    def close(self):
        if getattr(self, "_handle", None):
            _lib.teuk_b200_batch_destroy(self._handle)
            self._handle = None

    __del__ = close

    def __len__(self):
        return len(self.configs)

    def set_state(self, instance: int, state):
        n = self.configs[instance].value_count()
        ptr, kind, _keep = _pointer(state, False, n)
        _check(_lib.teuk_b200_batch_set_state(self._handle, instance, ptr, n,
                                              kind))

    def get_state(self, instance: int, out=None):
        c = self.configs[instance]
        if out is None:
            out = np.zeros(c.shape(), dtype=np.complex128)
        ptr, kind, _keep = _pointer(out, True, c.value_count())
        _check(_lib.teuk_b200_batch_get_state(self._handle, instance, ptr,
                                              c.value_count(), kind))
        return out

    def initialize_gaussian(self, instance: int, pulse: GaussianPulse):
        s, keep = pulse.to_struct()
        _check(_lib.teuk_b200_batch_initialize_gaussian(self._handle, instance,
                                                        ctypes.byref(s)))

    def step(self, dt, steps: int = 1, graph: bool = True):
        dts = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, dtype=np.float64),
                                                   (len(self.configs),)))
        _check(_lib.teuk_b200_batch_step(
            self._handle, dts.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            steps, int(graph)))

    def sample_endpoint(self, instance: int):
        c = self.configs[instance]
        cap = 4 * len(c.modes) * (c.ell_max_first + c.ell_max_second + 2)
        buf = (WaveformRecord * cap)()
        count = ctypes.c_size_t()
        _check(_lib.teuk_b200_batch_sample_endpoint(self._handle, instance, buf,
                                                    cap, ctypes.byref(count)))
        return _records(buf, count.value)

    def endpoint_modal_count(self) -> int:
        count = ctypes.c_size_t()
        _check(_lib.teuk_b200_batch_endpoint_modal(self._handle, None, 0,
                                                   ctypes.byref(count), HOST))
        return count.value

    def endpoint_modal(self, out=None):
        n = self.endpoint_modal_count()
        if out is None:
            out = np.zeros(n, dtype=np.complex128)
        ptr, kind, _keep = _pointer(out, True, n)
        count = ctypes.c_size_t()
        _check(_lib.teuk_b200_batch_endpoint_modal(self._handle, ptr, n,
                                                   ctypes.byref(count), kind))
        return out

    def set_stream(self, stream_handle: int | None):
        _check(_lib.teuk_b200_batch_set_stream(
            self._handle, ctypes.c_void_p(stream_handle or 0)))

    def synchronize(self):
        _check(_lib.teuk_b200_batch_synchronize(self._handle))

    def launches_per_step(self) -> int:
        n = ctypes.c_int()
        _check(_lib.teuk_b200_batch_launches_per_step(self._handle,
                                                      ctypes.byref(n)))
        return n.value

    def stage_kernels(self) -> tuple[int, int]:
        """(launch groups on the streaming kernel, groups on the tile
        kernel)."""
        a, b = ctypes.c_int(), ctypes.c_int()
        _check(_lib.teuk_b200_batch_stage_kernels(self._handle,
                                                  ctypes.byref(a),
                                                  ctypes.byref(b)))
        return a.value, b.value


class Server:
    """Continuous batching: solves are admitted as memory allows, advance in
    one shared batched step, and leave with their waveform records."""

    def __init__(self, hbm_budget_bytes: int, max_active: int = 0,
                 graph: bool = True, precision: int = PRECISION_FP64):
        opts = _ServerOptions(ABI_VERSION, int(hbm_budget_bytes),
                              int(max_active), int(graph), int(precision))
        handle = ctypes.c_void_p()
        _check(_lib.teuk_b200_server_create(ctypes.byref(opts),
                                            ctypes.byref(handle)))
        self._handle = handle

    def close(self):
        if getattr(self, "_handle", None):
            _lib.teuk_b200_server_destroy(self._handle)
            self._handle = None

    __del__ = close

    def submit(self, config: SolveConfig, pulse: GaussianPulse, dt: float,
               steps: int) -> int:
        s, keep = config.to_struct()
        g, gkeep = pulse.to_struct()
        rid = ctypes.c_uint64()
        _check(_lib.teuk_b200_server_submit(self._handle, ctypes.byref(s),
                                            ctypes.byref(g), dt, steps,
                                            ctypes.byref(rid)))
        return rid.value

    def advance(self, steps: int = 1) -> int:
        active = ctypes.c_int()
        _check(_lib.teuk_b200_server_advance(self._handle, steps,
                                             ctypes.byref(active)))
        return active.value

    def result(self, request_id: int):
        """(waveform records, time-to-waveform seconds) of a finished
        request; raises InvalidArgument while it is queued or running."""
        count = ctypes.c_size_t()
        latency = ctypes.c_double()
        _check(_lib.teuk_b200_server_result(self._handle, request_id, None, 0,
                                            ctypes.byref(count),
                                            ctypes.byref(latency)))
        buf = (WaveformRecord * max(count.value, 1))()
        _check(_lib.teuk_b200_server_result(self._handle, request_id, buf,
                                            count.value, ctypes.byref(count),
                                            ctypes.byref(latency)))
        return _records(buf, count.value), latency.value

    def stats(self) -> ServerStats:
        st = ServerStats()
        _check(_lib.teuk_b200_server_stats_get(self._handle, ctypes.byref(st)))
        return st

