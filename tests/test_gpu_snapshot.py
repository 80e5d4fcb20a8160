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
