"""The parameter models on the CPU, against the reference's
(src/dnsjax/parameters.py:26-211): defaults, validation bounds, the derived
values, the merge of explicitly set fields, padded sizes and TOML input."""

from math import pi

import pytest
from pydantic import ValidationError

from dnsjax_b200 import parameters as P

# Reference defaults (parameters.py:26-133); dist.platform and solver.backend
# are the two deliberate differences.
REFERENCE_DEFAULTS = {
    "dist": {"np": 1, "platform": "cpu"},
    "phys": {"re": 1000, "system": "kolmogorov", "oversampling_factor": 3,
             "oversample_y": True},
    "geo": {"lx": 4.0, "lz": 4.0, "tilt_degree": 0},
    "res": {"nx": 128, "ny": 128, "nz": 128, "fd_order": 4, "double_precision": True},
    "init": {"start_from_laminar": True, "snapshot": None, "t0": 0, "it0": 0},
    "outs": {"it_stats": None},
    "step": {"dt": 0.01, "implicitness": 0.5, "corrector_tolerance": 1e-5,
             "max_corrector_iterations": 10},
    "stop": {"max_sim_time": None, "max_wall_time": None},
    "debug": {"time_functions": True, "measure_corrections": False,
              "correct_divergence": True},
    "solver": {"backend": "banded"},
}


def test_defaults_match_the_reference():
    got = P.Parameters().model_dump()
    want = {k: dict(v) for k, v in REFERENCE_DEFAULTS.items()}
    want["dist"]["platform"] = "cuda"
    want["solver"]["backend"] = "cuda"
    assert got == want


@pytest.mark.parametrize("section,field,value", [
    ("phys", "re", 0.0), ("phys", "oversampling_factor", 1), ("phys", "system", "pipe"),
    ("geo", "lx", 0.0), ("geo", "tilt_degree", -180.0), ("geo", "tilt_degree", 181.0),
    ("res", "nx", 0), ("res", "fd_order", 1), ("step", "dt", 0.0),
    ("step", "implicitness", 1.5), ("step", "corrector_tolerance", 0.0),
    ("step", "max_corrector_iterations", 0), ("dist", "np", 0),
    ("solver", "backend", "lapack")])
def test_validation_rejects(section, field, value):
    with pytest.raises(ValidationError):
        P.Parameters(**{section: {field: value}})


@pytest.mark.parametrize("backend", ["banded", "dense", "cuda"])
def test_backends_accepted(backend):
    assert P.Parameters(solver={"backend": backend}).solver.backend == backend


@pytest.mark.parametrize("system,ly", [("kolmogorov", 4), ("waleffe", 4),
                                       ("decaying-box", 4), ("plane-couette", 2)])
def test_derived_ly(system, ly):
    assert P.derive(P.Parameters(phys={"system": system})).ly == ly


@pytest.mark.parametrize("tilt,flags", [(0.0, (False, False)), (180.0, (False, False)),
                                        (90.0, (True, True)), (-90.0, (True, True)),
                                        (30.0, (True, False)), (-45.0, (True, False))])
def test_derived_tilt(tilt, flags):
    d = P.derive(P.Parameters(geo={"tilt_degree": tilt}))
    assert (d.tilt, d.tilt_90) == flags
    assert d.tilt_rad == pi * tilt / 180


def test_update_applies_only_set_fields():
    saved = P.params.model_copy(deep=True)
    try:
        P.update_parameters(P.Parameters(phys={"system": "plane-couette", "re": 400.0}))
        P.update_parameters(P.Parameters(res={"ny": 65}))
        assert P.params.phys.system == "plane-couette" and P.params.phys.re == 400.0
        assert P.params.res.ny == 65 and P.params.res.nx == 128
        assert P.derived_params.ly == 2
    finally:
        for name in type(saved).model_fields:
            setattr(P.params, name, getattr(saved, name))
        P.derive(P.params, P.derived_params)


@pytest.mark.parametrize("sections,want", [
    ({"res": {"nx": 32, "ny": 32, "nz": 64}}, (48, 48, 96)),
    ({"res": {"nx": 32, "ny": 32, "nz": 64}, "phys": {"oversample_y": False}}, (48, 32, 96)),
    ({"res": {"nx": 128, "ny": 129, "nz": 128}, "phys": {"system": "plane-couette"}},
     (192, 129, 192)),
    ({"res": {"nx": 16, "ny": 16, "nz": 16}, "phys": {"oversampling_factor": 4}},
     (32, 32, 32)),
])
def test_padded_sizes(sections, want):
    assert P.padded_sizes(P.Parameters(**sections)) == want


def test_read_parameters_from_toml(tmp_path):
    f = tmp_path / "params.toml"
    f.write_text('[phys]\nsystem = "plane-couette"\nre = 400.0\n\n'
                 '[res]\nnx = 64\nny = 65\nnz = 64\nfd_order = 6\n\n'
                 '[step]\ndt = 0.02\n\n'
                 '[stop]\nmax_wall_time = "PT1H"\n')
    p = P.read_parameters(f)
    assert p.phys.system == "plane-couette" and p.res.fd_order == 6 and p.step.dt == 0.02
    assert p.stop.max_wall_time.total_seconds() == 3600
