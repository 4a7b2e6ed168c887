"""The serving benchmark's bookkeeping, on the CPU: error definitions and the
routing of requests to operating points (no GPU, no library calls)."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench as B  # noqa: E402


def test_serving_error_definitions():
    ref = np.array([2.0, -0.5, 1e-3], np.float64)
    est = np.array([2.002, -0.5005, 0.0], np.float32)
    # gravity: relative to |ref|
    g = B.serving_error("gravity", est[:2], ref[:2])
    assert np.allclose(g, [1e-3, 1e-3], rtol=1e-4)
    # winding number: relative to max(|ref|, 1) -- its unit is the jump across the surface
    w = B.serving_error("wn", est, ref)
    assert np.allclose(w, [1e-3, 5e-4, 1e-3], rtol=1e-4)
    # smooth distance: the error of D = -log(S) / alpha; a non-positive S is infinite
    s_ref = np.exp(-B.SERVING_ALPHA * np.array([0.3, 0.5]))
    s_est = np.array([s_ref[0] * np.exp(-B.SERVING_ALPHA * 3e-4), -1.0], np.float32)
    e = B.serving_error("smooth", s_est, s_ref)
    assert abs(e[0] - 1e-3) < 2e-5 and np.isinf(e[1])


def test_operating_points_route_requests():
    for kern, m in B.MATCHED.items():
        r = {"kernel": kern}
        assert B.op_of(r, "plain") == m["plain"]
        assert B.op_of(r, "served") == m["served"]
        sto = B.op_of(r, "served_stochastic")
        if m["stochastic"] is None:
            assert sto == m["served"]
        else:
            assert sto == ("stochastic", m["stochastic"])
        # the plain path is the per-call Barnes-Hut drop-in, or exact where no theta suffices
        assert m["plain"][0] in ("barnes_hut", "brute_force")
        assert B.tree_key(m["served"]) == ("sbh" if m["served"][0] == "stochastic" else "bh")


def test_serving_config_is_the_same_for_both_arms():
    a = B.serving_config(1500, 12799492)
    b = B.serving_config(1500, 12799492)
    assert a == b and a["operating_points"]["smooth"]["plain"] == ["brute_force", None]


def test_pair_pipe_bound_counts():
    # 16 MUFU operations and 128 FP32 lane operations per clock per SM: the
    # all-pairs kernels are MUFU-bound, the smooth distance at 1.75 MUFU
    # operations per pair (a sqrt; the exponential on the MUFU for three
    # sources in four), the 2D winding number (one reciprocal) FP32-bound.
    rates = {"rsqrt_per_s": 16.0, "ffma_per_s": 128.0}
    for kernel, mufu in (("plummer", 1.0), ("gravity", 2.0), ("smooth", 1.75)):
        bound, m, fp32 = B.pair_pipe_bound(rates, kernel, 3)
        assert m == mufu and bound == 16.0 / mufu and 128.0 / fp32 > bound
    bound, m, fp32 = B.pair_pipe_bound(rates, "wn", 2)
    assert m == 1.0 and fp32 == 10 and bound == 12.8
    assert B.pair_pipe_bound(rates, "smooth", 3)[2] == 10.0
