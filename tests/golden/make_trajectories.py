"""Oracle trajectories of the plane-Couette benchmark workloads (fixtures).

Runs the oracle's restatement of the reference's step / corrector loop
(``src/dnsjax/__main__.py:125-203``, ``oracle/stepper.py``) on the host, in
FP64, from the same seeded initial fields the benchmark and the GPU tests
use, and records what the ``-m gpu`` trajectory tests compare against:

* every step's corrector iterations, final correction norm and perturbation
  energy E' (Simpson in y, ``plane_couette.py:591-613``);
* the state at checkpoint steps: the whole field at the last step of the
  64x65x64 workload, and the low-wavenumber block (``kx`` index < 16,
  ``|kz|`` index < 8, every y point) elsewhere -- the 128x129x128 field is
  50 MB per state, too large to commit.

The influence-matrix operators come from the oracle's restatement of the
reference's ``precompute_imm`` (``geometries/cartesian.py:575-801``), not
from the GPU.  The corrector cap is 60 instead of the reference's default
10: with 10, the reference's loop ends both runs after the first step.

    python tests/golden/make_trajectories.py [--threads N] [case ...]

Cases: ``couette64`` (nx = nz = 64, ny = 65, p = 4, Re 400, dt 0.02,
energy 1e-3, 100 steps) and ``couette128`` (128x129x128, p = 6, Re 1000,
dt 0.01, energy 5e-2, 30 steps).
"""

from __future__ import annotations

import argparse
import json
import sys
import time
from math import pi
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
OUT = HERE / "trajectories"

# kx index < KX_BLOCK and |kz| index < KZ_BLOCK: the checkpoint block.
KX_BLOCK, KZ_BLOCK = 16, 8

CASES = {
    "couette64": dict(nx=64, ny=65, nz=64, p=4, re=400.0, dt=0.02, lx=2 * pi,
                      lz=pi, tol=1e-10, max_iter=60, energy=1e-3, kscale=8.0,
                      seed=1, steps=100, checkpoints=(10, 50, 100), full=(100,)),
    "couette128": dict(nx=128, ny=129, nz=128, p=6, re=1000.0, dt=0.01,
                       lx=2 * pi, lz=pi, tol=1e-10, max_iter=60, energy=5e-2,
                       kscale=32.0, seed=4, steps=30, checkpoints=(10, 30),
                       full=()),
}


def block_index(nz: int) -> np.ndarray:
    """Stored kz rows of the checkpoint block: harmonics 0..KZ_BLOCK-1 and
    -(KZ_BLOCK-1)..-1 of the Nyquist-free kz axis of length nz - 1."""
    nkz = nz - 1
    return np.concatenate([np.arange(KZ_BLOCK), np.arange(nkz - KZ_BLOCK + 1, nkz)])


def block(state: np.ndarray, nz: int) -> np.ndarray:
    return np.ascontiguousarray(state[:, block_index(nz), :KX_BLOCK, :])


def make(name: str) -> Path:
    sys.path.insert(0, str(ROOT))
    from dnsjax_b200 import initial
    from oracle.config import Config
    from oracle.couette import CouetteSetup
    from oracle.stepper import make_stepper

    c = CASES[name]
    cfg = Config(system="plane-couette", nx=c["nx"], ny=c["ny"], nz=c["nz"],
                 lx=c["lx"], lz=c["lz"], re=c["re"], dt=c["dt"],
                 corrector_tolerance=c["tol"], max_corrector_iterations=c["max_iter"],
                 fd_order=c["p"])
    t0 = time.time()
    S = CouetteSetup(cfg)
    print(f"{name}: operators in {time.time() - t0:.1f} s", flush=True)
    u = initial.couette_field(c["nx"], c["ny"], c["nz"], c["lx"], c["lz"], c["p"],
                              c["seed"], c["kscale"], c["energy"])
    pac, itc = make_stepper(S.get_rhs, S.predict, S.correct, S.norm)
    iters, errors, energy = [], [], []
    out = {"e0": np.float64(S.norm2(u) / 2)}
    for n in range(1, c["steps"] + 1):
        t1 = time.time()
        state_prev = u
        u, rhs, err = pac(state_prev)
        k = 0
        while err > cfg.corrector_tolerance and k < cfg.max_corrector_iterations:
            u, rhs, err = itc(state_prev, u, rhs)
            k += 1
        u = S.correct_velocity(u, cfg.correct_divergence)
        iters.append(k)
        errors.append(err)
        energy.append(S.norm2(u) / 2)
        print(f"{name}: step {n} iterations {k} error {err:.3e} "
              f"E' {energy[-1]:.12e} ({time.time() - t1:.1f} s)", flush=True)
        if not err < cfg.corrector_tolerance:
            raise RuntimeError(f"{name}: step {n} did not converge")
        if n in c["checkpoints"]:
            out[f"block_{n}"] = block(u, c["nz"])
        if n in c["full"]:
            out[f"state_{n}"] = u
    case = {k: v for k, v in c.items() if k not in ("checkpoints", "full")}
    case.update(checkpoints=list(c["checkpoints"]), full=list(c["full"]),
                kx_block=KX_BLOCK, kz_block=KZ_BLOCK)
    out.update(case_json=json.dumps(case), iterations=np.array(iters, np.int32),
               errors=np.array(errors), energy=np.array(energy))
    OUT.mkdir(exist_ok=True)
    path = OUT / f"{name}.npz"
    np.savez_compressed(path, **out)
    print(f"{name}: wrote {path} ({path.stat().st_size / 1e6:.1f} MB)", flush=True)
    return path


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("cases", nargs="*", default=sorted(CASES))
    ap.add_argument("--threads", type=int, default=8)
    a = ap.parse_args()
    sys.path.insert(0, str(ROOT))
    from oracle import parallel

    parallel.set_threads(a.threads)
    for name in a.cases:
        make(name)


if __name__ == "__main__":
    main()
