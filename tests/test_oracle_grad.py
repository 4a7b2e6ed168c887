"""The gradient oracles (orc_*_grad in oracle/sbh_oracle.c) checked on the CPU.

The reference has no gradient path to pin against, so the oracles are pinned by
mathematics:
* the FP64 brute-force gradient against FP64 central differences (h = 1e-4) of
  the FP64 brute-force value, for gravity, Plummer and the smooth distance
  D = -log(sum exp(-alpha r)) / alpha, in 2D and 3D;
* Barnes-Hut with beta = inf opens every leaf, so its value and gradient must
  equal brute force;
* the stochastic gradient oracle walks orc_sbh's paths: same contribution
  counts, and for gravity the same value up to FP32 rounding of orc_sbh;
* the smooth distance's value against the plain oracle's exp sums (-log/alpha).
"""
import numpy as np
import pytest

import oracle as O
import sbh_workloads as W

GRAD_KERNELS = (O.GRAVITY, O.PLUMMER, O.SMOOTH_DIST)


def _points(dim, n, seed):
    if dim == 3:
        return W.gaussian_mixture(n, seed=seed)
    return W.gaussian_mixture(n, seed=seed, dim=2)


def _fd(points, masses, kernel, q, alpha, eps, h=1e-4):
    """Central differences of the FP64 brute-force value, with the float32
    perturbed coordinates' actual spacing as the step."""
    q = np.asarray(q, np.float32)
    dim = q.shape[1]
    out = np.zeros(q.shape, np.float64)
    for d in range(dim):
        qp, qm = q.copy(), q.copy()
        qp[:, d] = (q[:, d].astype(np.float64) + h).astype(np.float32)
        qm[:, d] = (q[:, d].astype(np.float64) - h).astype(np.float32)
        vp, _ = O.brute_force_grad_f64(points, masses, kernel, qp, alpha, eps)
        vm, _ = O.brute_force_grad_f64(points, masses, kernel, qm, alpha, eps)
        step = qp[:, d].astype(np.float64) - qm[:, d].astype(np.float64)
        out[:, d] = (vp - vm) / step
    return out


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("kernel", GRAD_KERNELS)
def test_brute_force_gradient_matches_central_differences(dim, kernel):
    pts, nrm, m = _points(dim, 2000, seed=31 + dim)
    rng = np.random.default_rng(32)
    q = rng.uniform(-1.0, 1.0, (40, dim)).astype(np.float32)
    alpha, eps = 20.0, 1e-3
    val, grad = O.brute_force_grad_f64(pts, m, kernel, q, alpha, eps)
    fd = _fd(pts, m, kernel, q, alpha, eps)
    scale = np.linalg.norm(grad, axis=1)
    err = np.linalg.norm(grad - fd, axis=1) / scale
    assert np.median(err) < 1e-6, np.median(err)
    # Near a source the O(h^2) truncation of the h = 1e-4 differences reaches
    # 1e-3 (Plummer's eps = 1e-3 is its length scale); Richardson extrapolation
    # with h/2 removes that term and must agree everywhere.
    rich = (4.0 * _fd(pts, m, kernel, q, alpha, eps, h=5e-5) - fd) / 3.0
    err_r = np.linalg.norm(grad - rich, axis=1) / scale
    assert np.all(err_r < 1e-5), err_r.max()
    assert np.all(np.isfinite(val))


@pytest.mark.parametrize("dim", [2, 3])
def test_smooth_distance_value_is_log_of_plain_sum(dim):
    pts, nrm, m = _points(dim, 3000, seed=40 + dim)
    q = np.random.default_rng(41).uniform(-1.0, 1.0, (30, dim)).astype(np.float32)
    alpha = 30.0
    d, _ = O.brute_force_grad_f64(pts, m, O.SMOOTH_DIST, q, alpha)
    s = O.brute_force_f64(pts, nrm, m, O.SMOOTH_DIST, q, alpha=alpha)
    assert np.allclose(d, -np.log(s) / alpha, rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("dim,dsl", [(2, 1), (3, 1), (3, 2)])
@pytest.mark.parametrize("kernel", GRAD_KERNELS)
def test_barnes_hut_gradient_opens_everything_at_infinite_beta(dim, dsl, kernel):
    pts, nrm, m = _points(dim, 1500, seed=50 + dim)
    lo, hi = W.padded_box(pts)
    t = O.OracleTree(pts, nrm, m, lo, hi, alpha=25.0, dim_split_log=dsl)
    q = np.random.default_rng(51).uniform(-1.0, 1.0, (25, dim)).astype(np.float32)
    val, grad, cnt = t.bh_grad(kernel, q, np.inf, alpha=25.0)
    bval, bgrad = O.brute_force_grad_f64(pts, m, kernel, q, 25.0)
    assert np.array_equal(cnt, np.full(len(q), len(pts)))
    assert np.allclose(val, bval, rtol=1e-12, atol=1e-12)
    assert np.allclose(grad, bgrad, rtol=1e-10, atol=1e-10 * np.abs(bgrad).max())


@pytest.mark.parametrize("dim,dsl", [(2, 2), (3, 2)])
@pytest.mark.parametrize("kernel", GRAD_KERNELS)
def test_barnes_hut_gradient_node_set_matches_plain_walk(dim, dsl, kernel):
    pts, nrm, m = _points(dim, 4000, seed=60 + dim)
    lo, hi = W.padded_box(pts)
    t = O.OracleTree(pts, nrm, m, lo, hi, alpha=25.0, dim_split_log=dsl)
    q = np.random.default_rng(61).uniform(-1.0, 1.0, (200, dim)).astype(np.float32)
    val, grad, cnt = t.bh_grad(kernel, q, 2.0, alpha=25.0)
    pv, pc, _ = t.bh(kernel, q, 2.0)
    assert np.array_equal(cnt, pc)
    if kernel == O.SMOOTH_DIST:
        assert np.allclose(val, -np.log(pv.astype(np.float64)) / 25.0, rtol=1e-5)
    else:
        assert np.allclose(val, pv, rtol=1e-5)


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("kernel", GRAD_KERNELS)
def test_sampler_gradient_walks_the_plain_sampler_paths(dim, kernel):
    pts, nrm, m = _points(dim, 4000, seed=70 + dim)
    lo, hi = W.padded_box(pts)
    t = O.OracleTree(pts, nrm, m, lo, hi, alpha=25.0, dim_split_log=2)
    q = np.random.default_rng(71).uniform(-1.0, 1.0, (200, dim)).astype(np.float32)
    val, grad, cnt = t.sbh_grad(kernel, q, 3, seed=9, alpha=25.0)
    pv, pc = t.sbh(kernel, q, 3, rng=O.RNG_PHILOX, seed=9)
    assert np.array_equal(cnt, pc)
    if kernel == O.SMOOTH_DIST:
        ok = pv > 0
        assert np.allclose(val[ok], -np.log(pv[ok].astype(np.float64)) / 25.0, rtol=1e-4)
    else:
        assert np.allclose(val, pv, rtol=1e-4)
    assert np.all(np.isfinite(grad[np.isfinite(val)]))


@pytest.mark.parametrize("kernel", GRAD_KERNELS)
def test_sampler_gradient_on_the_reference_mt19937_stream(kernel):
    """With the reference CPU sampler's std::mt19937 stream (seeded per query),
    the gradient oracle walks the same paths as orc_sbh on that stream: same
    contribution counts, and values agree to the FP32-vs-FP64 rounding."""
    pts, nrm, m = _points(3, 4000, seed=74)
    lo, hi = W.padded_box(pts)
    t = O.OracleTree(pts, nrm, m, lo, hi, alpha=25.0, dim_split_log=2)
    q = np.random.default_rng(75).uniform(-1.0, 1.0, (200, 3)).astype(np.float32)
    seeds = np.arange(200, dtype=np.uint32) * 7919 + 3
    val, grad, cnt = t.sbh_grad(kernel, q, 2, alpha=25.0, rng=O.RNG_MT19937, mt_seeds=seeds)
    pv, pc = t.sbh(kernel, q, 2, rng=O.RNG_MT19937, mt_seeds=seeds)
    assert np.array_equal(cnt, pc)
    if kernel == O.SMOOTH_DIST:
        ok = pv > 0
        assert np.allclose(val[ok], -np.log(pv[ok].astype(np.float64)) / 25.0, rtol=1e-4)
    else:
        assert np.allclose(val, pv, rtol=1e-4)
    # a different stream takes different paths
    _, _, cnt2 = t.sbh_grad(kernel, q, 2, alpha=25.0, rng=O.RNG_MT19937, mt_seeds=seeds + 1)
    assert not np.array_equal(cnt, cnt2)


def test_sampler_gravity_gradient_is_unbiased():
    """Mean of the stochastic gravity gradient over 512 seeds equals the exact
    gradient within 4 standard errors, per query and component."""
    pts, nrm, m = W.gaussian_mixture(3000, seed=80)
    lo, hi = W.padded_box(pts)
    t = O.OracleTree(pts, nrm, m, lo, hi, dim_split_log=2)
    q = np.random.default_rng(81).uniform(-1.0, 1.0, (6, 3)).astype(np.float32)
    gs = np.stack([t.sbh_grad(O.GRAVITY, q, 1, seed=s)[1] for s in range(512)])
    _, exact = O.brute_force_grad_f64(pts, m, O.GRAVITY, q)
    mean = gs.mean(axis=0)
    se = gs.std(axis=0, ddof=1) / np.sqrt(len(gs))
    assert np.all(np.abs(mean - exact) <= 4 * se + 1e-9 * np.abs(exact))
