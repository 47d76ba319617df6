"""teuk_solver .cfg schema: the engine's parser against the reference's own
(include/teuk/config.hpp compiled in oracle/_ref).  Valid configurations must
resolve to byte-identical resolved_config.cfg text and the same pipeline
mapping; invalid ones must be rejected with the reference's message."""
import pytest

import teuk_b200 as tb
from oracle_bindings import ref_parse_run_config, ref_resolved_config

KERR = """
# Kerr ringdown, seeded Gaussian pair
config_version = 1
mass = 1.0
spin = 0.7
compactification_length = 1
nr = 1025
ntheta = 25
ellmax_first = 16
ellmax_second = 16
first_order_modes = -4,-3,-2,-1,0,1,2,3,4
second_order_modes = -4, -3, -2, -1, 0, 1, 2, 3, 4
final_time = 1.1045232051503807
steps = 1000
cfl = 0.25
reduction_damping = 0.1
dissipation = 1.8806976056754497e-4
radial_discretization = d10-5
initial_data.center = 0.1556
initial_data.width = 0.0156
initial_data.seed_ell = 2
initial_data.seed_m = 2
initial_data.amplitude_real = 7.3e-4
initial_data.amplitude_imag = -2.1e-4
initial_data.add_sharp_partner = true
output.directory = runs/kerr
"""

SECOND = """
spin = 0.9
nr = 97
ntheta = 21
ellmax_first = 6
ellmax_second = 12
first_order_modes = -2,2
second_order_modes = -4,0,4
final_time = 0.01
steps = 40
dissipation = 0.002
radial_discretization = d8-4
reduction_mode = stage_constrained
second_order.enabled = 1
second_order.source_mode = unrestricted
second_order.source_start_time = 0.005
initial_data.mode.0.ell = 2
initial_data.mode.0.m = 2
initial_data.mode.0.amplitude_real = 1e-2
initial_data.mode.0.amplitude_imag = 0
initial_data.mode.1.ell = 3
initial_data.mode.1.m = -2
initial_data.mode.1.amplitude_real = -3e-3
initial_data.mode.1.amplitude_imag = 5e-3
initial_data.compact_support = false
output.checkpoint_every = 10
"""

CHECKPOINT = """
nr = 65
initial_data.type = checkpoint
initial_data.checkpoint_directory = runs/ck/checkpoint_00000100
"""

VALID = [("defaults", "", ()), ("kerr", KERR, ()), ("second", SECOND, ()),
         ("checkpoint", CHECKPOINT, ()),
         ("overrides", KERR, ("steps=2000", "spin = 0.5", "dissipation=0")),
         ("plus2_schema", SECOND,
          ("plus2.ell_max_first=5", "plus2.output.ordered_pairs=false"))]


@pytest.mark.parametrize("name,text,overrides", VALID,
                         ids=[v[0] for v in VALID])
def test_resolved_text_matches_reference(name, text, overrides):
    status, expected = ref_resolved_config(text, overrides)
    assert status == 0, expected
    assert tb.resolved_config(text, overrides) == expected


@pytest.mark.parametrize("name,text,overrides", VALID,
                         ids=[v[0] for v in VALID])
def test_pipeline_mapping_matches_reference(name, text, overrides):
    mine = tb.parse_run_config(text, overrides)
    ref = ref_parse_run_config(text, overrides)
    for field, _ in tb.RunConfig._fields_:
        a, b = getattr(mine, field), getattr(ref, field)
        if field in ("modes", "parents", "targets"):
            assert list(a) == list(b), field
        elif field == "seeds":
            n = mine.seed_count
            assert [(s.ell, s.m, s.amplitude_real, s.amplitude_imag)
                    for s in a[:n]] == \
                [(s.ell, s.m, s.amplitude_real, s.amplitude_imag) for s in b[:n]]
        else:
            assert a == b, field


INVALID = [
    ("unknown key", "nr = 65\nbogus = 1\n", ()),
    ("duplicate", "nr = 65\nnr = 66\n", ()),
    ("two equals", "nr = 6=5\n", ()),
    ("empty value", "nr = \n", ()),
    ("malformed number", "mass = 1.0x\n", ()),
    ("bad bool", "initial_data.compact_support = yes\n", ()),
    ("empty list item", "first_order_modes = -2,,2\n", ()),
    ("reduction", "reduction_mode = implicit\n", ()),
    ("discretization", "radial_discretization = d6-3\n", ()),
    ("spin", "spin = 1.5\n", ()),
    ("nr small", "nr = 12\nradial_discretization = d10-5\n", ()),
    ("ntheta", "ntheta = 5\n", ()),
    ("not closed", "first_order_modes = -2,2,3\nellmax_first=4\n", ()),
    ("above ellmax", "first_order_modes = -5,5\n", ()),
    ("daughters", "second_order.enabled = true\nsecond_order_modes = -4,4\n"
                  "ellmax_second = 4\n", ()),
    ("dissipation bound", "dissipation = 10\n", ()),
    ("steps", "steps = 0\n", ()),
    ("seed ell", "initial_data.seed_ell = 9\n", ()),
    ("seed m", "initial_data.seed_m = 1\ninitial_data.seed_ell = 2\n", ()),
    ("partial mode", "initial_data.mode.1.ell = 2\n", ()),
    ("center", "initial_data.center = 1.5\n", ()),
    ("time derivative", "initial_data.time_derivative = galerkin\n", ()),
    ("checkpoint dir", "initial_data.type = checkpoint\n", ()),
    ("policy", "second_order.required_consecutive_passes = 0\n", ()),
    ("plus2 enabled", "plus2.enabled = true\n", ()),
    ("plus2 mode", "plus2.mode = sideways\n", ()),
    ("plus2 normalization", "plus2.source_normalization.version = 1\n", ()),
    ("output dir", "output.diagnostic_every = 0\n", ()),
    ("override syntax", "", ("steps",)),
    ("override duplicate", "", ("steps=3", "steps=4")),
]


@pytest.mark.parametrize("name,text,overrides", INVALID,
                         ids=[v[0] for v in INVALID])
def test_rejections_match_reference(name, text, overrides):
    status, message = ref_resolved_config(text, overrides)
    assert status != 0
    with pytest.raises(tb.TeukError) as info:
        tb.resolved_config(text, overrides)
    assert str(info.value).split("] ", 1)[-1] == message


@pytest.mark.gpu
def test_parsed_run_drives_engine_like_reference(require_gpu):
    """A parsed .cfg maps onto the pipeline, its initial data and its step
    exactly as teuk_solver builds them (make_run_mode_registry,
    make_source_policy, expanded_gaussian_modes, final_time / steps)."""
    from cases import relative_error
    from oracle_bindings import RefPipeline

    text = KERR.replace("nr = 1025", "nr = 97")
    run = tb.parse_run_config(text, ("steps=20000",))
    config, pulse = run.solve_config(), run.pulse()
    gpu, ref = tb.Pipeline(config), RefPipeline(config)
    gpu.initialize_gaussian(pulse)
    ref.initialize_gaussian(pulse)
    gpu.step(0.0, run.time_step, 10)
    ref.step(0.0, run.time_step, 10)
    g, r = gpu.get_state(), ref.get_state()
    for f in range(3):
        assert relative_error(g[:, f], r[:, f]) < 1e-10
