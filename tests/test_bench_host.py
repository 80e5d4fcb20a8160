"""Host logic of bench.py, on the CPU: the algorithmic bytes behind every
roofline figure (pinned to the per-workload values of the measurement
plan), the segmenting of long timed runs, strict-JSON output, and the
threads of the oracle's cpu_baseline leg."""

import json

import pytest


def test_algorithmic_bytes():
    import bench

    W = bench.WORKLOADS
    mb = lambda x: round(x / 1e6, 2)  # noqa: E731
    c128 = bench.op_bytes(W["couette128"])
    assert (mb(c128["rhs"]), mb(c128["imm"])) == (557.18, 612.59)
    c64 = bench.op_bytes(W["couette64"])
    assert (mb(c64["rhs"]), mb(c64["imm"])) == (70.09, 64.01)
    k32 = bench.op_bytes(W["kolmogorov32"])
    assert (mb(k32["rhs"]), mb(k32["correct"])) == (18.95, 2.95)
    assert mb(bench.op_bytes(W["kolmogorov128"])["rhs"]) == 1228.02
    # mixed form: the state read and the RHS write stay complex128, the pass
    # buffers are complex64
    k128 = W["kolmogorov128"]
    S = (k128["ny"] - 1) * (k128["nz"] - 1) * k128["nx"] // 2
    f32 = bench.op_bytes(k128, fp32=True)["rhs"]
    assert f32 == 16 * 6 * S + (bench.op_bytes(k128)["rhs"] - 16 * 6 * S) // 2


@pytest.mark.parametrize("k,want", [(0, []), (1, [1]), (30, [30]), (31, [30, 1]),
                                    (70, [30, 30, 10])])
def test_segments(k, want):
    import bench

    assert bench.segments(k) == want
    assert all(s <= bench.SEGMENT for s in want)


def test_strict_json(capsys):
    import bench

    bench.emit({"value": float("nan"), "e2e": {"value": float("inf"), "n": 3},
                "list": [1.0, float("-inf")]})
    line = capsys.readouterr().out.strip()
    d = json.loads(line)
    assert d == {"value": None, "e2e": {"value": None, "n": 3}, "list": [1.0, None]}


def test_cpu_sample_uses_the_host_threads():
    """The cpu_baseline leg on the oracle: one full time step timed whole,
    threads reported as cores, the pool back at one thread afterwards."""
    import bench
    from oracle import parallel

    w = bench.WORKLOADS["kolmogorov32"]
    r = bench.cpu_sample(w, bench.initial_state(w, w["seed"]))
    assert r["kind"] == "port" and r["value"] > 0
    assert r["cores"] == bench.host_threads() and 1 <= r["cores"] <= 32
    assert f"{r['cores']} host threads" in r["sample"]
    assert "1 full time step" in r["sample"]
    assert parallel.threads() == 1


def test_oracle_steps_follow_the_reference_loop():
    """The reference arm's steps: the oracle's corrector loop stops at the
    tolerance, like oracle.stepper.run (the restatement of __main__.py)."""
    import numpy as np

    import bench
    from oracle.stepper import run

    w = dict(bench.WORKLOADS["kolmogorov32"], nx=8, ny=8, nz=8)
    S = bench.oracle_setup(w)
    u0 = bench.initial_state(w, 3)
    u, iters = bench.oracle_steps(S, u0, 3)
    ref = run(S, u0, 3)
    assert iters == ref.corrector_iterations
    assert np.array_equal(u, ref.state)


def test_both_arms_share_the_workload_config():
    import bench

    for name, w in bench.WORKLOADS.items():
        tol = w.get("tol", 1e-10)
        a = bench.workload_config(name, w, tol)
        assert a == bench.workload_config(name, w, tol) and a["workload"] == name
        assert "tol" in a and "l2" in a
    c = bench.workload_config("couette128", bench.WORKLOADS["couette128"], 1e-10)
    assert c["max_corrector_iterations"] == 60 and "deviation" in c


def test_x_pass_flops():
    """The x pass's flop rate from the tuner's timing (Couette 128x129x128:
    129 x 192 rows of 5 length-192 complex FFTs plus the product)."""
    import math

    import bench

    w = bench.WORKLOADS["couette128"]
    tuning = {"variants": [0, 0, 0, 0], "ms": [[0.09, 0.1, 0.1], [0.1063, 0.25, 0.3],
                                               [0.03, 0.05, 0.05], [0.24, 0.32, 1.7]],
              "stages": ["z inverse", "x", "z forward", "IMM"]}
    r = bench.x_pass_flops(w, tuning)
    flops = 129 * 192 * (25 * 192 * math.log2(192) + 40 * 192)
    assert r["flops_per_call"] == flops and r["dtype"] == "f64"
    assert abs(r["tflops"] - flops / 0.1063e-3 / 1e12) < 1e-9
    assert 10.0 < r["tflops"] < 11.0
    assert bench.x_pass_flops(w, None) is None
    assert bench.x_pass_flops(w, {"stages": ["x"], "ms": [[]], "variants": [0]}) is None


def test_step_roofline():
    """Whole-step bytes (2 + c) x (RHS + corrector call), plus the divergence
    correction for the periodic flows."""
    import bench

    w = bench.WORKLOADS["couette128"]
    ob = bench.op_bytes(w)
    r = bench.step_roofline(w, 11.0, 100.0, 6534.5)
    assert r["bytes_per_step"] == 13 * (ob["rhs"] + ob["imm"])
    assert abs(r["achieved_gbs"] - r["bytes_per_step"] * 100.0 / 1e9) < 1e-9
    assert abs(r["frac"] - r["achieved_gbs"] / 6534.5) < 1e-12
    k = bench.WORKLOADS["kolmogorov32"]
    okb = bench.op_bytes(k)
    rk = bench.step_roofline(k, 3.0, 1.0, 1.0)
    assert rk["bytes_per_step"] == 5 * (okb["rhs"] + okb["correct"]) + 16 * 6 * 31 * 31 * 16
    assert bench.step_roofline({"system": "plane-couette"}, 1.0, 1.0, 1.0) is None
