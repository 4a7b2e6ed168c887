"""The FP32-pipe exponential of the smooth-distance brute force (pairs.cuh,
exp2_fma), emulated step by step in NumPy FP32 arithmetic with the constants
read from the source: range reduction by rounding, the degree-5 polynomial by
FMA Horner steps (one rounding each), 2^j added to the exponent field as an
integer.  The kernel evaluates 2^u for u = t + 64 (t = -alpha log2(e) r) and
removes the 2^64 from the sums.  CPU only."""
import os
import re

import numpy as np

SRC = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "stochastic-barnes-hut_b200",
                   "csrc", "pairs.cuh")


def constants():
    text = open(SRC).read()
    c = {}
    for name in ("kExp2C1", "kExp2C2", "kExp2C3", "kExp2C4", "kExp2C5", "kExp2Round",
                 "kExp2Unscale"):
        m = re.search(r"constexpr float %s = ([0-9a-fx.p+-]+)f;" % name, text)
        assert m, name
        v = m.group(1)
        c[name] = np.float32(float.fromhex(v) if "x" in v else float(v))
    return c


def fma32(a, b, c):
    # a*b of two FP32 numbers is exact in FP64; one rounding to FP32 after the add
    return (a.astype(np.float64) * b.astype(np.float64) + np.float64(c)).astype(np.float32)


def exp2_fma(u):
    k = constants()
    tc = np.maximum(u.astype(np.float32), np.float32(-125.0))
    tr = (tc + k["kExp2Round"]).astype(np.float32)
    nj = fma32(tr, np.full_like(tr, -1.0), k["kExp2Round"])
    f = (tc + nj).astype(np.float32)
    p = fma32(np.full_like(f, k["kExp2C5"]), f, k["kExp2C4"])
    for name in ("kExp2C3", "kExp2C2", "kExp2C1"):
        p = fma32(p, f, k[name])
    p = fma32(p, f, np.float32(1.0))
    return (p.view(np.uint32) + (tr.view(np.uint32) << np.uint32(23))).view(np.float32)


def test_relative_error_over_the_kernel_range():
    # u = t + 64 for t in [-189, 0]: every value the smooth distance produces
    # that survives the final 2^-64
    u = np.concatenate([np.linspace(-125.0, 64.0, 2_000_001), 64.0 - np.logspace(-12, 0, 5000)])
    u = u.astype(np.float32)
    got = exp2_fma(u).astype(np.float64)
    ref = np.exp2(u.astype(np.float64))
    assert (np.abs(got - ref) / ref).max() < 1.6e-7


def test_exact_points_and_clamp():
    got = exp2_fma(np.array([64.0, 63.0, 0.0, -60.0, -125.0], np.float32))
    assert np.array_equal(got, np.array([2.0 ** 64, 2.0 ** 63, 1.0, 2.0 ** -60, 2.0 ** -125],
                                        np.float32))
    # below -125 the value stays 2^-125, i.e. 2^-189 once unscaled: zero in FP32
    far = exp2_fma(np.array([-126.0, -300.0, -1e30], np.float32))
    assert np.all(far == np.float32(2.0 ** -125))
    assert np.float32(far[0]) * constants()["kExp2Unscale"] == 0.0


def test_scaled_form_keeps_subnormal_terms():
    # t in the FP32 subnormal range (2^-149 .. 2^-126) is an FP32 normal in the
    # scaled form, so a sum of such terms keeps its relative precision
    t = np.linspace(-149.0, -126.0, 10001).astype(np.float32)
    scaled = exp2_fma(t + np.float32(64.0))
    assert np.all(scaled >= np.float32(2.0 ** -85))
    ref = np.exp2(t.astype(np.float64))
    assert (np.abs(scaled.astype(np.float64) * 2.0 ** -64 - ref) / ref).max() < 1.6e-7
