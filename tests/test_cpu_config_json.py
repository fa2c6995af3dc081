"""The reference's "JSON config parsing" testsets (test/runtests.jl:
3244-3511), restated through the C ABI: draugr_amg_config_from_json parses,
draugr_b200_config_json reads every field back (where the reference's tests
read the Julia config object behind the handle), and the expected defaults
are those of AMGConfig() (src/types.jl:514-529)."""

import json

import pytest

import draugr

DEFAULTS = {
    "smoother": "l1_colored_gs", "jacobi_omega": 2.0 / 3.0, "max_levels": 20, "max_coarse_size": 50,
    "pre_smoothing_steps": 1, "post_smoothing_steps": 1, "verbose": 0, "initial_coarsening_levels": 0,
    "max_row_sum": 1.0, "cycle": "v", "strength": "absolute", "coarse_solve_on_cpu": False,
}
EXT_I_DEFAULT = {"type": "extended_i", "trunc_factor": 0.0, "max_elements": 0, "norm_p": 1,
                 "rescale": False}


@pytest.fixture(scope="module")
def lib():
    return draugr._lib.load()


def parse(lib, text):
    h = lib.draugr_amg_config_from_json(text.encode())
    assert h > 0, draugr.last_error()
    c = json.loads(lib.draugr_b200_config_json(h))
    assert lib.draugr_amg_config_free(h) == 0
    return c


def test_empty_json_gives_the_defaults(lib):
    """"empty JSON produces AMGConfig() defaults" (:3254-3271)."""
    c = parse(lib, "{}")
    for k, v in DEFAULTS.items():
        assert c[k] == pytest.approx(v), k
    assert c["coarsening"]["type"] == "hmis" and c["coarsening"]["theta"] == 0.5
    assert c["coarsening"]["interpolation"] == EXT_I_DEFAULT
    assert c["initial_coarsening"] == c["coarsening"]


def test_scalar_and_string_encoded_fields(lib):
    """"scalar fields" and "string-encoded values" (:3273-3311)."""
    c = parse(lib, """{"theta": 0.3, "max_levels": 10, "max_coarse_size": 25,
        "pre_smoothing_steps": 2, "post_smoothing_steps": 3, "jacobi_omega": 0.8, "verbose": 2,
        "initial_coarsening_levels": 3, "max_row_sum": 0.9, "coarse_solve_on_cpu": true}""")
    assert c["coarsening"]["theta"] == pytest.approx(0.3)
    assert (c["max_levels"], c["max_coarse_size"], c["pre_smoothing_steps"], c["post_smoothing_steps"],
            c["verbose"], c["initial_coarsening_levels"]) == (10, 25, 2, 3, 2, 3)
    assert c["jacobi_omega"] == pytest.approx(0.8) and c["max_row_sum"] == pytest.approx(0.9)
    assert c["coarse_solve_on_cpu"] is True
    c = parse(lib, """{"theta": "0.3", "max_levels": "10", "jacobi_omega": "0.8",
        "coarse_solve_on_cpu": "true", "verbose": "2"}""")
    assert c["coarsening"]["theta"] == pytest.approx(0.3) and c["max_levels"] == 10
    assert c["jacobi_omega"] == pytest.approx(0.8) and c["coarse_solve_on_cpu"] is True
    assert c["verbose"] == 2


@pytest.mark.parametrize("name", ["hmis", "pmis", "rs", "aggregation", "smoothed_aggregation",
                                  "aggressive_pmis", "aggressive_hmis"])
def test_coarsening_types(lib, name):
    """"coarsening types" (:3313-3329): each name selects its coarsening (the
    aggressive ones with their base)."""
    assert parse(lib, json.dumps({"coarsening": name}))["coarsening"]["type"] == name


@pytest.mark.parametrize("name", ["jacobi", "colored_gs", "serial_gs", "spai0", "spai1", "l1_jacobi",
                                  "l1_colored_gs", "l1_serial_gs", "chebyshev", "ilu0", "serial_ilu0"])
def test_smoother_types(lib, name):
    """"smoother types" (:3331-3348)."""
    assert parse(lib, json.dumps({"smoother": name}))["smoother"] == name


def test_smoother_omega_override_and_interpolation(lib):
    """"smoother with omega override" and the "interpolation" testsets
    (:3350-3400): string names, nested extended+i options, nested direct
    with a truncation factor, and nested defaults from the type's
    constructor."""
    c = parse(lib, '{"smoother": {"type": "jacobi", "omega": 0.42}}')
    assert c["smoother"] == "jacobi" and c["jacobi_omega"] == pytest.approx(0.42)
    for name in ("direct", "standard", "extended_i"):
        assert parse(lib, json.dumps({"interpolation": name}))["coarsening"]["interpolation"]["type"] == name
    ip = parse(lib, """{"interpolation": {"type": "extended_i", "trunc_factor": 0.3, "max_elements": 5,
        "norm_p": 2, "rescale": true}}""")["coarsening"]["interpolation"]
    assert ip == {"type": "extended_i", "trunc_factor": pytest.approx(0.3), "max_elements": 5, "norm_p": 2,
                  "rescale": True}
    ip = parse(lib, '{"interpolation": {"type": "direct", "trunc_factor": 0.1}}')["coarsening"]["interpolation"]
    assert ip["type"] == "direct" and ip["trunc_factor"] == pytest.approx(0.1)
    ip = parse(lib, '{"interpolation": {"type": "extended_i"}}')["coarsening"]["interpolation"]
    assert ip == EXT_I_DEFAULT


def test_strength_cycle_and_initial_coarsening(lib):
    """"strength types", "cycle types", "initial_coarsening", "initial_coarsening
    defaults to coarsening" and "unknown keys are ignored" (:3402-3436)."""
    assert parse(lib, '{"strength": "absolute"}')["strength"] == "absolute"
    assert parse(lib, '{"strength": "signed"}')["strength"] == "signed"
    assert parse(lib, '{"cycle": "v"}')["cycle"] == "v"
    assert parse(lib, '{"cycle": "w"}')["cycle"] == "w"
    c = parse(lib, '{"coarsening": "hmis", "initial_coarsening": "pmis", "initial_coarsening_levels": 2}')
    assert c["coarsening"]["type"] == "hmis" and c["initial_coarsening"]["type"] == "pmis"
    assert c["initial_coarsening_levels"] == 2
    c = parse(lib, '{"coarsening": "rs"}')
    assert c["coarsening"]["type"] == "rs" and c["initial_coarsening"]["type"] == "rs"
    c = parse(lib, '{"type": "draugr", "setup_frequency": 30, "theta": 0.4}')
    assert c["coarsening"]["theta"] == pytest.approx(0.4)


def test_invalid_input_and_handle_lifecycle(lib):
    """"invalid type names return -1", "invalid JSON returns -1", "handle
    lifecycle" and "case insensitive" (:3438-3472)."""
    for text in ('{"coarsening": "bogus"}', '{"smoother": "nope"}', '{"interpolation": "bad"}',
                 '{"strength": "wrong"}', '{"cycle": "z"}', "{not valid json"):
        assert lib.draugr_amg_config_from_json(text.encode()) == -1, text
        assert len(draugr.last_error()) > 0
    h = lib.draugr_amg_config_from_json(b"{}")
    assert h > 0 and lib.draugr_b200_config_json(h) is not None
    assert lib.draugr_amg_config_free(h) == 0
    assert lib.draugr_b200_config_json(h) is None
    assert lib.draugr_amg_config_free(h) == -1
    c = parse(lib, '{"coarsening": "HMIS", "smoother": "L1_Colored_GS", "cycle": "V"}')
    assert c["coarsening"]["type"] == "hmis" and c["smoother"] == "l1_colored_gs" and c["cycle"] == "v"


def test_python_mirror_round_trip():
    """The Python mirror's AMGConfig goes through the same parser: its
    fields read back unchanged (draugr.config_fields)."""
    cfg = draugr.AMGConfig(coarsening=draugr.PMISCoarsening(0.3, draugr.StandardInterpolation(0.1)),
                           smoother=draugr.ChebyshevSmootherType(), max_levels=7, cycle_type="W",
                           strength_type=draugr.SignedStrength(), seed=9)
    c = draugr.config_fields(cfg)
    assert c["coarsening"]["type"] == "pmis" and c["coarsening"]["theta"] == pytest.approx(0.3)
    assert c["coarsening"]["interpolation"]["type"] == "standard"
    assert c["coarsening"]["interpolation"]["trunc_factor"] == pytest.approx(0.1)
    assert (c["smoother"], c["max_levels"], c["cycle"], c["strength"], c["seed"]) == (
        "chebyshev", 7, "w", "signed", 9)


def test_full_realistic_config(lib):
    """"full realistic config" (:3474-3510)."""
    c = parse(lib, """{"coarsening": "hmis",
        "interpolation": {"type": "extended_i", "trunc_factor": 0.0, "max_elements": 5, "norm_p": 2,
                          "rescale": true},
        "smoother": "serial_gs", "strength": "absolute", "cycle": "v", "theta": 0.5,
        "jacobi_omega": 0.6666666666666666, "max_levels": 20, "max_coarse_size": 50,
        "pre_smoothing_steps": 1, "post_smoothing_steps": 1, "initial_coarsening": "aggressive_pmis",
        "initial_coarsening_levels": 1, "max_row_sum": 1.0, "coarse_solve_on_cpu": false,
        "verbose": 0}""")
    assert c["coarsening"]["type"] == "hmis" and c["coarsening"]["theta"] == pytest.approx(0.5)
    ip = c["coarsening"]["interpolation"]
    assert (ip["type"], ip["max_elements"], ip["norm_p"], ip["rescale"]) == ("extended_i", 5, 2, True)
    assert c["smoother"] == "serial_gs" and c["strength"] == "absolute" and c["cycle"] == "v"
    assert c["jacobi_omega"] == pytest.approx(2 / 3)
    assert c["initial_coarsening"]["type"] == "aggressive_pmis" and c["initial_coarsening_levels"] == 1
