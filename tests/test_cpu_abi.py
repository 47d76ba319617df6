"""The drop-in boundary on a host without a GPU.

* libteuk_b200.so loads and exports every entry point include/teuk_b200.h
  declares;
* construction-time validation reproduces the reference's
  std::invalid_argument cases before any device work;
* a valid configuration fails loudly (status TEUK_B200_ERR_CUDA) when no
  CUDA device is usable: there is no CPU fallback;
* the C++ facade (include/teuk_b200.hpp) compiles against the library and
  maps status codes to the reference's exception types.
"""
import re
import subprocess
from pathlib import Path

import pytest

import teuk_b200 as tb
from cases import CASES
from conftest import cuda_available

REPO = Path(__file__).resolve().parent.parent
HEADER = REPO / "include" / "teuk_b200.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(teuk_b200_[a-z_0-9]+)\s*\(", text)))


def test_header_symbols_are_exported():
    names = declared_functions()
    assert len(names) >= 30
    out = subprocess.run(["nm", "-D", "--defined-only", str(tb.LIBRARY_PATH)],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (teuk_b200_\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    lib = tb.library()
    for name in names:
        assert hasattr(lib, name)


def test_abi_version():
    assert tb.library().teuk_b200_abi_version() == tb.ABI_VERSION


@pytest.mark.parametrize("change,message", [
    ({"radial_points": 12, "discretization": tb.D105},
     "too small for selected discretization"),
    ({"theta_nodes": 8}, "exact-product padding"),
    ({"modes": (-2, 2, 3)}, "closed under m -> -m"),
    ({"modes": (-2, 2, 2)}, "duplicate mode"),
    ({"dissipation": -1.0}, "dissipation must be nonnegative"),
    ({"parents": (-3, 3)}, "is not stored"),
    ({"ell_max_first": 2}, "exact-product padding"),
    ({"spin": 1.5}, "Kerr parameters"),
])
def test_reference_validation_before_device_work(change, message):
    config = tb.SolveConfig(**{**CASES["schw_d84"].__dict__, **change})
    with pytest.raises(tb.InvalidArgument, match=re.escape(message)):
        tb.Pipeline(config)


SECOND_ORDER = tb.SolveConfig(**{**CASES["nonparent"].__dict__,
                                 "source_mode": tb.SOURCE_UNRESTRICTED})


@pytest.mark.skipif(cuda_available(), reason="host has a GPU")
def test_second_order_has_no_cpu_fallback():
    with pytest.raises(tb.TeukError) as info:
        tb.Pipeline(SECOND_ORDER)
    assert info.value.status == tb.ERR_CUDA


@pytest.mark.parametrize("change,message", [
    ({"targets": (-4, 0, 6)}, "is not stored"),
    ({"normalized_constraint_tolerance": -1.0}, "source policy is invalid"),
    ({"required_consecutive_passes": 0}, "source policy is invalid"),
    ({"ell_max_second": 2}, "exact-product padding"),
])
def test_second_order_validation_before_device_work(change, message):
    config = tb.SolveConfig(**{**SECOND_ORDER.__dict__, **change})
    with pytest.raises(tb.InvalidArgument, match=re.escape(message)):
        tb.Pipeline(config)


def test_second_order_footprint_counts_nodal_buffers():
    nodal = tb.footprint_bytes(SECOND_ORDER)
    points = (len(SECOND_ORDER.modes) * SECOND_ORDER.radial_points *
              SECOND_ORDER.theta_nodes)
    # at least the state, RK stage and four RK slopes of all 13 fields
    assert nodal >= 6 * 13 * points * 16
    linear = tb.footprint_bytes(CASES["nonparent"])
    assert nodal > linear


@pytest.mark.skipif(cuda_available(), reason="host has a GPU")
def test_no_cpu_fallback_without_gpu():
    with pytest.raises(tb.TeukError) as info:
        tb.Pipeline(CASES["schw_d84"])
    assert info.value.status == tb.ERR_CUDA


def test_cpp_facade_compiles_and_maps_exceptions(tmp_path):
    exe = tmp_path / "facade_check"
    subprocess.run(["g++", "-std=c++20", "-O1", "-I", str(REPO / "include"),
                    str(REPO / "tests" / "cpp" / "facade_check.cpp"),
                    str(tb.LIBRARY_PATH), f"-Wl,-rpath,{tb.LIBRARY_PATH.parent}",
                    "-o", str(exe)], check=True)
    run = subprocess.run([str(exe)], capture_output=True, text=True)
    assert run.stdout.count("invalid_argument:") == 2
    expected = 0 if cuda_available() else 3
    assert run.returncode == expected, run.stdout + run.stderr


def test_server_options_validated_before_device_work():
    with pytest.raises(tb.InvalidArgument, match="budget must be positive"):
        tb.Server(hbm_budget_bytes=0)
    with pytest.raises(tb.InvalidArgument, match="max_active"):
        tb.Server(hbm_budget_bytes=1 << 30, max_active=-1)


@pytest.mark.skipif(cuda_available(), reason="host has a GPU")
def test_server_has_no_cpu_fallback():
    with pytest.raises(tb.TeukError) as info:
        tb.Server(hbm_budget_bytes=1 << 30)
    assert info.value.status == tb.ERR_CUDA


@pytest.mark.parametrize("options,message", [
    (tb.LaunchOptions(strip_rows=32), "strip_rows must be 0 or at least 64"),
    (tb.LaunchOptions(stage_kernel=7), "unknown stage kernel choice"),
    (tb.LaunchOptions(precision=3), "unknown transform precision"),
])
def test_launch_options_are_validated_before_device_work(options, message):
    with pytest.raises(tb.InvalidArgument, match=message):
        tb.Batch([CASES["schw_d84"]], options)
    with pytest.raises(tb.InvalidArgument, match=message):
        tb.Pipeline(CASES["schw_d84"], options)


def test_test_hook_rejects_bad_chunk():
    with pytest.raises(tb.InvalidArgument, match="chunk"):
        tb.test_withhold_chunk(-2)
    tb.test_withhold_chunk(-1)
