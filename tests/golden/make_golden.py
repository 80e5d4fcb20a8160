"""Generate golden fixtures by running the reference solver's own source.

The reference (gokhanyalniz/dnsjax) is pure Python/JAX; JAX is not
installed here, so each case imports the reference's ``src/dnsjax``
through ``tests/golden/jaxshim`` -- a NumPy-backed stand-in for the jax API
subset it uses (eager, one CPU device, float64).  Each case runs in a fresh
subprocess because the reference builds its singletons from ``params`` at
import time.  Inputs are this package's seeded initial fields
(``dnsjax_b200.initial``); outputs are the reference's single-call results
(RHS, predictor, corrector, norm, padded physical field, stats) and a short
trajectory through the reference's step/corrector loop
(``__main__.py:125-203``).

Each case also writes a snapshot file in the reference's npz format from
the seeded field and loads it back through the reference's own
``init_state`` (``flows/plane_couette.py:225-248``,
``flows/monochromatic.py:294-314``), recording the snapshot's array and the
state the reference read from it.

Run from the repository root, given the reference checkout (its path as
``--ref`` or in ``DNSJAX_REFERENCE``):

    python tests/golden/make_golden.py --ref <reference checkout> [case ...]
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
from math import pi
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]

CASES = {
    # Kolmogorov, 2*pi box (the 32^3 workload's geometry) at 8^3.
    "kolmogorov_n8": dict(
        system="kolmogorov", nx=8, ny=8, nz=8, lx=2 * pi, lz=2 * pi,
        ly=2 * pi, re=40.0, dt=0.01, tol=1e-10, steps=5, tilt=0.0,
        energy=1e-2, spectrum="cfg0", seed=0),
    # Kolmogorov, 2*pi box at 16^3, 10 steps.
    "kolmogorov_n16": dict(
        system="kolmogorov", nx=16, ny=16, nz=16, lx=2 * pi, lz=2 * pi,
        ly=2 * pi, re=40.0, dt=0.01, tol=1e-10, steps=10, tilt=0.0,
        energy=1e-2, spectrum="cfg0", seed=1),
    # Non-cubic, tilted forcing, default Ly = 4, stronger perturbation.
    "kolmogorov_tilt30": dict(
        system="kolmogorov", nx=8, ny=12, nz=16, lx=4.0, lz=3.0, ly=None,
        re=100.0, dt=0.01, tol=1e-10, steps=3, tilt=30.0, energy=0.1,
        spectrum="cfg0", seed=2),
    "waleffe_tilt90": dict(
        system="waleffe", nx=8, ny=8, nz=8, lx=4.0, lz=4.0, ly=None,
        re=60.0, dt=0.02, tol=1e-10, steps=3, tilt=90.0, energy=0.05,
        spectrum="cfg0", seed=3),
    "decaying_n12": dict(
        system="decaying-box", nx=12, ny=12, nz=12, lx=4.0, lz=4.0,
        ly=None, re=200.0, dt=0.01, tol=1e-10, steps=3, tilt=0.0,
        energy=0.2, spectrum="k53", seed=4),
    # Plane Couette, the 64x65x64 workload's parameters at 8x17x8.
    "couette_n8_p4": dict(
        system="plane-couette", nx=8, ny=17, nz=8, lx=2 * pi, lz=pi,
        re=400.0, dt=0.02, tol=1e-10, steps=5, p=4, energy=1e-3,
        kscale=8.0, seed=10),
    # Plane Couette, the 128x129x128 workload's parameters at 8x33x12.
    "couette_p6": dict(
        system="plane-couette", nx=8, ny=33, nz=12, lx=2 * pi, lz=pi,
        re=1000.0, dt=0.01, tol=1e-10, steps=3, p=6, energy=5e-2,
        kscale=32.0, seed=11),
    "couette_n16_p4": dict(
        system="plane-couette", nx=16, ny=17, nz=16, lx=2 * pi, lz=pi,
        re=400.0, dt=0.02, tol=1e-10, steps=3, p=4, energy=1e-2,
        kscale=8.0, seed=12),
}


def initial_state(case: dict) -> np.ndarray:
    sys.path.insert(0, str(ROOT))
    from dnsjax_b200 import initial

    if case["system"] == "plane-couette":
        return initial.couette_field(
            case["nx"], case["ny"], case["nz"], case["lx"], case["lz"],
            case["p"], case["seed"], case["kscale"], case["energy"])
    spec = (initial.kolmogorov_spectrum_cfg0 if case["spectrum"] == "cfg0"
            else initial.kolmogorov_spectrum_k53)
    ly = case["ly"] if case["ly"] is not None else 4.0
    return initial.periodic_field(
        case["nx"], case["ny"], case["nz"], case["lx"], ly, case["lz"],
        case["seed"], spec, case["energy"])


CHILD = r'''
import json, sys
import numpy as np
case = json.loads(sys.argv[1]); inp = sys.argv[2]; outp = sys.argv[3]
from dnsjax.parameters import (Parameters, derived_params, padded_res,
                               params, update_parameters)
params.dist.platform = "cpu"
params.phys.system = case["system"]
params.phys.re = case["re"]
params.res.nx, params.res.ny, params.res.nz = case["nx"], case["ny"], case["nz"]
params.res.double_precision = True
params.geo.lx, params.geo.lz = case["lx"], case["lz"]
params.geo.tilt_degree = case.get("tilt", 0.0)
params.step.dt = case["dt"]
params.step.implicitness = 0.5
params.step.corrector_tolerance = case["tol"]
params.step.max_corrector_iterations = 10
if "p" in case:
    params.res.fd_order = case["p"]
update_parameters(Parameters())
if case.get("ly") is not None:
    derived_params.ly = case["ly"]
padded_res.set_padded_resolution(params)
if case["system"] == "plane-couette":
    from dnsjax.flows import plane_couette as fm
    from dnsjax.geometries.cartesian import fourier
else:
    from dnsjax.flows import monochromatic as fm
    from dnsjax.geometries.triply_periodic import fourier
flow = fm.flow
import jax.numpy as jnp
u0 = jnp.asarray(np.load(inp))
out = {"u0": np.asarray(u0)}
out["phys0"] = np.asarray(fm.spec_to_phys(u0))
rhs0 = fm._get_rhs(u0, fourier, flow)
out["rhs0"] = np.asarray(rhs0)
pred = fm._predict(u0, rhs0, fourier, flow)
out["pred0"] = np.asarray(pred)
rhs1 = fm._get_rhs(pred, fourier, flow)
out["rhs1"] = np.asarray(rhs1)
corr_state, corr = fm._correct(u0, pred, rhs0, rhs1, fourier, flow)
out["corr_state0"] = np.asarray(corr_state)
out["corr0"] = np.asarray(corr)
out["norm0"] = np.asarray(fm._norm(corr, fourier, flow))
def stats(u):
    # The reference's get_stats raises for decaying-box: get_input reads
    # flow.unit_force, which only forced systems define
    # (monochromatic.py:237-267, 476-485).
    try:
        st = fm.get_stats(u)
    except AttributeError:
        return None
    return st
st = stats(u0)
if st is not None:
    out["stats0_keys"] = np.array(list(st.keys()))
    out["stats0"] = np.array([float(v) for v in st.values()])
cv, _ = fm.correct_velocity(u0)
out["cv0"] = np.asarray(cv)
# Step loop (__main__.py:125-203) for a fixed number of steps.
state = u0
tol = params.step.corrector_tolerance
last_error = 0.0
cs, errs = [], []
for it in range(case["steps"]):
    if not last_error < tol:
        break
    state_prev = state
    state, rhs, error = fm.predict_and_correct(state_prev)
    c = 0
    while error > tol and c < params.step.max_corrector_iterations:
        state, rhs, error = fm.iterate_correction(state_prev, state, rhs)
        c += 1
    state, _ = fm.correct_velocity(state)
    last_error = float(error)
    cs.append(c)
    errs.append(last_error)
# Snapshot exchange: the reference's snapshot format written from u0 and read
# back by the reference's own init_state.
params.init.start_from_laminar = False
if case["system"] == "plane-couette":
    snap = {"velocity_phys_nonexpanded": out["phys0"]}
else:
    snap = {"velocity_phys": out["phys0"] + np.asarray(flow.base_flow)}
np.savez("snapshot.npz", **snap)
out["snapshot_phys"] = next(iter(snap.values()))
out["snapshot_loaded"] = np.asarray(fm.init_state("snapshot.npz"))
params.init.start_from_laminar = True
out["uN"] = np.asarray(state)
out["iters"] = np.array(cs)
out["errors"] = np.array(errs)
st = stats(state)
if st is not None:
    out["statsN"] = np.array([float(v) for v in st.values()])
if case["system"] == "plane-couette":
    for k in ("Lk_ab", "Hk_ab"):
        out[k] = np.asarray(getattr(flow, k[:2] + "_op").ab)
    out["Lk_piv"] = np.asarray(flow.Lk_op.ipiv)
    out["Hk_piv"] = np.asarray(flow.Hk_op.ipiv)
    for k in ("p1", "p2", "v1", "v2", "q1", "q2", "M_inv", "D1", "D2"):
        out[k] = np.asarray(getattr(flow, k))
else:
    out["ldt_1"] = np.asarray(flow.ldt_1)
    out["ildt_2"] = np.asarray(flow.ildt_2)
np.savez_compressed(outp, **out)
'''


def run_case(name: str, case: dict, ref: Path) -> None:
    u0 = initial_state(case)
    env = dict(os.environ)
    env["PYTHONPATH"] = os.pathsep.join(
        [str(HERE / "jaxshim"), str(ref / "src")])
    with tempfile.TemporaryDirectory() as td:
        inp = Path(td) / "u0.npy"
        np.save(inp, u0)
        outp = HERE / f"{name}.npz"
        subprocess.run(
            [sys.executable, "-W", "ignore", "-c", CHILD, json.dumps(case),
             str(inp), str(outp)],
            check=True, env=env, cwd=td, stdout=subprocess.DEVNULL)
    meta = dict(case)
    with np.load(outp) as z:
        data = dict(z)
    data["case_json"] = np.array(json.dumps(meta))
    np.savez_compressed(outp, **data)
    print(f"{name}: {outp.stat().st_size / 1024:.0f} KB, iters={data['iters']}")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("DNSJAX_REFERENCE"),
                    help="reference checkout (default: $DNSJAX_REFERENCE)")
    ap.add_argument("cases", nargs="*")
    a = ap.parse_args()
    if not a.ref:
        ap.error("give the reference checkout with --ref or DNSJAX_REFERENCE")
    for name in a.cases or CASES:
        run_case(name, CASES[name], Path(a.ref))


if __name__ == "__main__":
    main()
