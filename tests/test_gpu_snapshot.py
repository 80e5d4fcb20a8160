"""npz snapshots in the reference's formats: a state written with
save_snapshot and read back with init_state (the reference's readers,
monochromatic.py:294-314 -- ``velocity_phys`` with the base flow -- and
plane_couette.py:225-248 -- ``velocity_phys_nonexpanded``) is the same
state to rounding, and the file carries the reference's key and the
physical-grid shape."""

from math import pi

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_periodic_snapshot_round_trip(tmp_path):
    import torch

    from dnsjax_b200 import initial
    from dnsjax_b200.flows.monochromatic import TriplyPeriodicFlow
    from dnsjax_b200.parameters import Parameters

    p = Parameters(phys=dict(system="kolmogorov", re=40.0),
                   geo=dict(lx=2 * pi, lz=2 * pi), res=dict(nx=16, ny=16, nz=16),
                   init=dict(start_from_laminar=False))
    flow = TriplyPeriodicFlow(p, ly=2 * pi)
    u = torch.as_tensor(initial.periodic_field(16, 16, 16, 2 * pi, 2 * pi, 2 * pi, 3,
                                               initial.kolmogorov_spectrum_cfg0, 1e-2),
                        device="cuda")
    path = tmp_path / "snap.npz"
    flow.save_snapshot(path, u)
    with np.load(path) as z:
        assert list(z.keys()) == ["velocity_phys"]
        assert z["velocity_phys"].shape == flow.phys_shape
        # the file holds the total velocity: perturbation plus base flow
        pert = flow.spec_to_phys(u).cpu().numpy()
        np.testing.assert_array_equal(z["velocity_phys"],
                                      pert + flow.base_flow[:, :, None, None])
    back = flow.init_state(path)
    d = torch.linalg.vector_norm(back - u) / torch.linalg.vector_norm(u)
    assert float(d) < 1e-13


def test_couette_snapshot_round_trip(tmp_path):
    import torch

    from dnsjax_b200 import initial
    from dnsjax_b200.flows.plane_couette import PlaneCouetteFlow
    from dnsjax_b200.parameters import Parameters

    p = Parameters(phys=dict(system="plane-couette", re=400.0),
                   geo=dict(lx=2 * pi, lz=pi), res=dict(nx=16, ny=17, nz=16, fd_order=4),
                   init=dict(start_from_laminar=False))
    flow = PlaneCouetteFlow(p)
    u0 = torch.as_tensor(initial.couette_field(16, 17, 16, 2 * pi, pi, 4, 2, 8.0, 1e-3),
                         device="cuda")
    u = flow.phys_to_spec(flow.spec_to_phys(u0))  # a field of real velocities
    path = tmp_path / "snap.npz"
    flow.save_snapshot(path, u)
    with np.load(path) as z:
        assert list(z.keys()) == ["velocity_phys_nonexpanded"]
        assert z["velocity_phys_nonexpanded"].shape == flow.phys_shape
    back = flow.init_state(path)
    d = torch.linalg.vector_norm(back - u) / torch.linalg.vector_norm(u)
    assert float(d) < 1e-13


@pytest.mark.parametrize("name", ["kolmogorov_n16", "kolmogorov_tilt30", "waleffe_tilt90",
                                  "couette_n8_p4", "couette_p6"])
def test_snapshots_exchange_with_the_reference(tmp_path, name):
    """Both directions against the reference's own code (golden fixtures made
    by tests/golden/make_golden.py): this package reads the snapshot file
    the reference read into the same state the reference's init_state
    produced, and writes from that state the array the reference's reader
    takes (the file's contents to rounding)."""
    import torch

    from conftest import load_golden, package_params, rel_l2

    case, g = load_golden(name)
    p = package_params(case)
    p.init.start_from_laminar = False
    if case["system"] == "plane-couette":
        from dnsjax_b200.flows.plane_couette import PlaneCouetteFlow

        flow, key = PlaneCouetteFlow(p), "velocity_phys_nonexpanded"
    else:
        from dnsjax_b200.flows.monochromatic import TriplyPeriodicFlow

        flow, key = TriplyPeriodicFlow(p, ly=case.get("ly")), "velocity_phys"
    path = tmp_path / "ref_snapshot.npz"
    np.savez(path, **{key: g["snapshot_phys"]})
    got = flow.init_state(path).cpu().numpy()
    assert rel_l2(got, g["snapshot_loaded"]) < 1e-13
    out = tmp_path / "ours.npz"
    flow.save_snapshot(out, torch.as_tensor(g["snapshot_loaded"], device="cuda"))
    with np.load(out) as z:
        assert list(z.keys()) == [key]
        assert rel_l2(z[key], g["snapshot_phys"]) < 1e-13
