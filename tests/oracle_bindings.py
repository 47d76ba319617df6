"""ctypes bindings of the oracles (test infrastructure only).

* ``RefPipeline`` drives the unmodified teuk-kokkos SpatialPipeline compiled
  against the project-written Kokkos-API host shim
  (oracle/_ref/libteuk_ref.so, built by oracle/Makefile where the reference
  sources are present; the built library travels with the repository).
* ``OraclePipeline`` drives the plain-C restatement of the linear RK4 path
  (oracle/_build/libteuk_oracle.so).

Both expose the same methods as ``teuk_b200.Pipeline`` so parity tests call
the B200 engine and an oracle with identical arguments.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

import teuk_b200 as tb

REPO = Path(__file__).resolve().parent.parent
REF_LIBRARY = REPO / "oracle" / "_ref" / "libteuk_ref.so"
REF_THREADS_LIBRARY = REPO / "oracle" / "_ref" / "libteuk_ref_threads.so"
ORACLE_LIBRARY = REPO / "oracle" / "_build" / "libteuk_oracle.so"

_ref_cache: dict = {}


def ref_available(threads: bool = False) -> bool:
    return (REF_THREADS_LIBRARY if threads else REF_LIBRARY).exists()


def load_ref(threads: bool = False) -> ctypes.CDLL:
    path = REF_THREADS_LIBRARY if threads else REF_LIBRARY
    if path in _ref_cache:
        return _ref_cache[path]
    if not path.exists():
        raise FileNotFoundError(f"{path} is missing; run `make -C oracle`")
    lib = ctypes.CDLL(str(path))
    P, D, I, SZ = ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_size_t
    DP = ctypes.POINTER(ctypes.c_double)
    sig = {
        "teuk_ref_last_error": ([], ctypes.c_char_p),
        "teuk_ref_backend": ([], ctypes.c_char_p),
        "teuk_ref_create": ([ctypes.POINTER(tb._Config), ctypes.POINTER(P)], I),
        "teuk_ref_destroy": ([P], I),
        "teuk_ref_shape": ([P, ctypes.POINTER(SZ)], I),
        "teuk_ref_set_state": ([P, P, SZ, I], I),
        "teuk_ref_get_state": ([P, P, SZ, I], I),
        "teuk_ref_evaluate_rhs": ([P, P, P, SZ, D, I], I),
        "teuk_ref_step": ([P, D, D, I], I),
        "teuk_ref_initialize_gaussian": ([P, ctypes.POINTER(tb._Gaussian)], I),
        "teuk_ref_sample_endpoint": ([P, ctypes.POINTER(tb.WaveformRecord), SZ,
                                      ctypes.POINTER(SZ)], I),
        "teuk_ref_get_activation": ([P, ctypes.POINTER(tb.Activation)], I),
        "teuk_ref_project_to_bands": ([P, P, SZ], I),
        "teuk_ref_gauss_legendre": ([I, DP, DP], I),
        "teuk_ref_transform_matrices": ([I, I, I, I, DP, DP,
                                         ctypes.POINTER(I)], I),
        "teuk_ref_sbp_matrix": ([I, I, DP, DP], I),
        "teuk_ref_checkpoint_write": ([P, ctypes.c_char_p, D, D,
                                       ctypes.c_uint64], I),
        "teuk_ref_checkpoint_load": ([P, ctypes.c_char_p, D,
                                      ctypes.POINTER(ctypes.c_double),
                                      ctypes.POINTER(ctypes.c_uint64)], I),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _ref_cache[path] = lib
    return lib


class RefError(RuntimeError):
    pass


class RefPipeline:
    """The reference SpatialPipeline behind the shared C ABI."""

    def __init__(self, config: tb.SolveConfig, threads: bool = False):
        self.lib = load_ref(threads)
        self.config = config
        s, keep = config.to_struct()
        handle = ctypes.c_void_p()
        self._check(self.lib.teuk_ref_create(ctypes.byref(s),
                                             ctypes.byref(handle)))
        self._handle = handle

    def _check(self, status):
        if status != 0:
            raise RefError(f"[{status}] " +
                           self.lib.teuk_ref_last_error().decode())

    def close(self):
        if getattr(self, "_handle", None):
            self.lib.teuk_ref_destroy(self._handle)
            self._handle = None

    __del__ = close

    @property
    def shape(self):
        dims = (ctypes.c_size_t * 4)()
        self.lib.teuk_ref_shape(self._handle, dims)
        return tuple(int(d) for d in dims)

    def _buf(self, arr):
        arr = np.ascontiguousarray(arr, dtype=np.complex128)
        assert arr.size == self.config.value_count()
        return arr

    def set_state(self, state):
        arr = self._buf(state)
        self._check(self.lib.teuk_ref_set_state(
            self._handle, ctypes.c_void_p(arr.ctypes.data), arr.size, 0))

    def get_state(self):
        out = np.zeros(self.shape, dtype=np.complex128)
        self._check(self.lib.teuk_ref_get_state(
            self._handle, ctypes.c_void_p(out.ctypes.data), out.size, 0))
        return out

    def evaluate_rhs(self, stage, time: float = 0.0):
        arr = self._buf(stage)
        out = np.zeros(self.shape, dtype=np.complex128)
        self._check(self.lib.teuk_ref_evaluate_rhs(
            self._handle, ctypes.c_void_p(arr.ctypes.data),
            ctypes.c_void_p(out.ctypes.data), arr.size, time, 0))
        return out

    def step(self, time: float, dt: float, steps: int = 1):
        self._check(self.lib.teuk_ref_step(self._handle, time, dt, steps))

    def initialize_gaussian(self, pulse: tb.GaussianPulse):
        s, keep = pulse.to_struct()
        self._check(self.lib.teuk_ref_initialize_gaussian(self._handle,
                                                          ctypes.byref(s)))

    def sample_endpoint(self):
        c = self.config
        cap = 4 * len(c.modes) * (c.ell_max_first + c.ell_max_second + 2)
        buf = (tb.WaveformRecord * cap)()
        count = ctypes.c_size_t()
        self._check(self.lib.teuk_ref_sample_endpoint(self._handle, buf, cap,
                                                      ctypes.byref(count)))
        return tb._records(buf, count.value)

    def checkpoint_write(self, directory, time_step: float, time: float,
                         step: int):
        self._check(self.lib.teuk_ref_checkpoint_write(
            self._handle, str(directory).encode(), time_step, time, step))

    def checkpoint_load(self, directory, time_step: float):
        t = ctypes.c_double()
        n = ctypes.c_uint64()
        self._check(self.lib.teuk_ref_checkpoint_load(
            self._handle, str(directory).encode(), time_step, ctypes.byref(t),
            ctypes.byref(n)))
        return t.value, n.value

    def diagnostics(self) -> tb.Diagnostics:
        lib = self.lib
        if not hasattr(lib, "_diag_ready"):
            lib.teuk_ref_diagnostics.argtypes = [ctypes.c_void_p,
                                                 ctypes.POINTER(tb.Diagnostics)]
            lib.teuk_ref_diagnostics.restype = ctypes.c_int
            lib._diag_ready = True
        d = tb.Diagnostics()
        self._check(lib.teuk_ref_diagnostics(self._handle, ctypes.byref(d)))
        return d

    def activation(self) -> tb.Activation:
        a = tb.Activation()
        self._check(self.lib.teuk_ref_get_activation(self._handle,
                                                     ctypes.byref(a)))
        return a

    def project_to_bands(self, state):
        arr = np.array(state, dtype=np.complex128, order="C", copy=True)
        self._check(self.lib.teuk_ref_project_to_bands(
            self._handle, ctypes.c_void_p(arr.ctypes.data), arr.size))
        return arr


def ref_gauss_legendre(n: int):
    lib = load_ref()
    x = np.zeros(n)
    w = np.zeros(n)
    dp = ctypes.POINTER(ctypes.c_double)
    assert lib.teuk_ref_gauss_legendre(n, x.ctypes.data_as(dp),
                                       w.ctypes.data_as(dp)) == 0
    return x, w


def ref_transform_matrices(spin: int, m: int, ell_max: int, nodes: int):
    lib = load_ref()
    ell_min = max(abs(spin), abs(m))
    ne = ell_max - ell_min + 1
    S = np.zeros((nodes, ne))
    A = np.zeros((ne, nodes))
    count = ctypes.c_int()
    dp = ctypes.POINTER(ctypes.c_double)
    assert lib.teuk_ref_transform_matrices(
        spin, m, ell_max, nodes, S.ctypes.data_as(dp), A.ctypes.data_as(dp),
        ctypes.byref(count)) == 0
    assert count.value == ne
    return S, A


def ref_sbp_matrix(disc: int, n: int):
    lib = load_ref()
    D = np.zeros((n, n))
    H = np.zeros(n)
    dp = ctypes.POINTER(ctypes.c_double)
    assert lib.teuk_ref_sbp_matrix(disc, n, D.ctypes.data_as(dp),
                                   H.ctypes.data_as(dp)) == 0
    return D, H


# ---------------------------------------------------------------- C oracle
_oracle_cache: dict = {}


def oracle_available() -> bool:
    return ORACLE_LIBRARY.exists()


def load_oracle() -> ctypes.CDLL:
    if "lib" in _oracle_cache:
        return _oracle_cache["lib"]
    if not ORACLE_LIBRARY.exists():
        raise FileNotFoundError(f"{ORACLE_LIBRARY} is missing; run `make -C oracle`")
    lib = ctypes.CDLL(str(ORACLE_LIBRARY))
    P, D, I, SZ = ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_size_t
    DP = ctypes.POINTER(ctypes.c_double)
    sig = {
        "oracle_last_error": ([], ctypes.c_char_p),
        "oracle_create": ([ctypes.POINTER(tb._Config), ctypes.POINTER(P)], I),
        "oracle_destroy": ([P], I),
        "oracle_set_state": ([P, P, SZ], I),
        "oracle_get_state": ([P, P, SZ], I),
        "oracle_evaluate_rhs": ([P, P, P, SZ], I),
        "oracle_step": ([P, D, I], I),
        "oracle_gauss_legendre": ([I, DP, DP], I),
        "oracle_sbp_matrix": ([I, I, DP, DP], I),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _oracle_cache["lib"] = lib
    return lib


class OraclePipeline:
    """The plain-C restatement of the linear pipeline."""

    def __init__(self, config: tb.SolveConfig):
        self.lib = load_oracle()
        self.config = config
        s, keep = config.to_struct()
        handle = ctypes.c_void_p()
        self._check(self.lib.oracle_create(ctypes.byref(s), ctypes.byref(handle)))
        self._handle = handle

    def _check(self, status):
        if status != 0:
            raise RefError(f"[{status}] " + self.lib.oracle_last_error().decode())

    def close(self):
        if getattr(self, "_handle", None):
            self.lib.oracle_destroy(self._handle)
            self._handle = None

    __del__ = close

    @property
    def shape(self):
        return self.config.shape()

    def set_state(self, state):
        arr = np.ascontiguousarray(state, dtype=np.complex128)
        self._check(self.lib.oracle_set_state(
            self._handle, ctypes.c_void_p(arr.ctypes.data), arr.size))

    def get_state(self):
        out = np.zeros(self.shape, dtype=np.complex128)
        self._check(self.lib.oracle_get_state(
            self._handle, ctypes.c_void_p(out.ctypes.data), out.size))
        return out

    def evaluate_rhs(self, stage, time: float = 0.0):
        arr = np.ascontiguousarray(stage, dtype=np.complex128)
        out = np.zeros(self.shape, dtype=np.complex128)
        self._check(self.lib.oracle_evaluate_rhs(
            self._handle, ctypes.c_void_p(arr.ctypes.data),
            ctypes.c_void_p(out.ctypes.data), arr.size))
        return out

    def step(self, time: float, dt: float, steps: int = 1):
        self._check(self.lib.oracle_step(self._handle, dt, steps))


def oracle_sbp_matrix(disc: int, n: int):
    lib = load_oracle()
    D = np.zeros((n, n))
    H = np.zeros(n)
    dp = ctypes.POINTER(ctypes.c_double)
    assert lib.oracle_sbp_matrix(disc, n, D.ctypes.data_as(dp),
                                 H.ctypes.data_as(dp)) == 0
    return D, H


def oracle_gauss_legendre(n: int):
    lib = load_oracle()
    x = np.zeros(n)
    w = np.zeros(n)
    dp = ctypes.POINTER(ctypes.c_double)
    assert lib.oracle_gauss_legendre(n, x.ctypes.data_as(dp),
                                     w.ctypes.data_as(dp)) == 0
    return x, w


def _ref_config_calls():
    lib = load_ref()
    if not hasattr(lib, "_config_ready"):
        CP = ctypes.POINTER(ctypes.c_char_p)
        lib.teuk_ref_resolved_config.argtypes = [
            ctypes.c_char_p, CP, ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t,
            ctypes.POINTER(ctypes.c_size_t)]
        lib.teuk_ref_resolved_config.restype = ctypes.c_int
        lib.teuk_ref_parse_run_config.argtypes = [
            ctypes.c_char_p, CP, ctypes.c_int, ctypes.POINTER(tb.RunConfig)]
        lib.teuk_ref_parse_run_config.restype = ctypes.c_int
        lib._config_ready = True
    return lib


def ref_resolved_config(text: str, overrides=()):
    """(status, resolved text or error message) from the reference parser."""
    lib = _ref_config_calls()
    arr, n = tb._override_array(overrides)
    length = ctypes.c_size_t()
    status = lib.teuk_ref_resolved_config(text.encode(), arr, n, None, 0,
                                          ctypes.byref(length))
    if status != 0:
        return status, lib.teuk_ref_last_error().decode()
    buf = ctypes.create_string_buffer(length.value + 1)
    lib.teuk_ref_resolved_config(text.encode(), arr, n, buf, length.value + 1,
                                 ctypes.byref(length))
    return 0, buf.value.decode()


def ref_parse_run_config(text: str, overrides=()):
    lib = _ref_config_calls()
    arr, n = tb._override_array(overrides)
    out = tb.RunConfig()
    status = lib.teuk_ref_parse_run_config(text.encode(), arr, n,
                                           ctypes.byref(out))
    if status != 0:
        raise RefError(lib.teuk_ref_last_error().decode())
    return out
