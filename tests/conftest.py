"""Shared test fixtures.  ``gpu``-marked tests need a CUDA device."""

from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))

GOLDEN_CASES = sorted(p.stem for p in GOLDEN.glob("*.npz"))
PERIODIC_CASES = [c for c in GOLDEN_CASES if not c.startswith("couette")]
COUETTE_CASES = [c for c in GOLDEN_CASES if c.startswith("couette")]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_golden(name: str) -> tuple[dict, dict]:
    with np.load(GOLDEN / f"{name}.npz") as z:
        data = dict(z)
    case = json.loads(str(data.pop("case_json")))
    return case, data


def oracle_config(case: dict):
    from oracle.config import Config

    kw = dict(system=case["system"], nx=case["nx"], ny=case["ny"],
              nz=case["nz"], lx=case["lx"], lz=case["lz"], re=case["re"],
              dt=case["dt"], corrector_tolerance=case["tol"],
              tilt_degree=case.get("tilt", 0.0))
    if case.get("ly") is not None:
        kw["ly"] = case["ly"]
    if "p" in case:
        kw["fd_order"] = case["p"]
    return Config(**kw)


def package_params(case: dict, max_iter: int = 10):
    """dnsjax_b200 Parameters for a golden case."""
    from dnsjax_b200.parameters import Parameters

    res = dict(nx=case["nx"], ny=case["ny"], nz=case["nz"])
    if "p" in case:
        res["fd_order"] = case["p"]
    return Parameters(
        phys=dict(system=case["system"], re=case["re"]),
        geo=dict(lx=case["lx"], lz=case["lz"], tilt_degree=case.get("tilt", 0.0)),
        res=res,
        step=dict(dt=case["dt"], implicitness=0.5,
                  corrector_tolerance=case["tol"],
                  max_corrector_iterations=max_iter),
    )


def rel_l2(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))
