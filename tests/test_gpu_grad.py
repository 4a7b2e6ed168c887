"""Values and query gradients on the GPU (sbh_eval_grad*, sbh_torch) against the
gradient oracles.

* brute force: value and gradient against the FP64 oracle;
* Barnes-Hut: gravity/Plummer values bit-identical to sbh_eval's, the same
  contribution counts, gradients and smooth distances against orc_bh_grad (FP64
  sums over the reference's node set);
* stochastic: the same paths as sbh_eval for the same seed (gravity/Plummer
  values bit-identical, same counts), gradients against orc_sbh_grad, and the
  gravity gradient unbiased over seeds against the brute-force gradient;
* the autograd wrapper: forward equals the C call, backward is grad_out * grad,
  and brute-force gradients through autograd match FP64 central differences.
"""
import numpy as np
import pytest

import oracle as O
import sbh_capi as C
import sbh_workloads as W
from helpers import bits_equal

pytestmark = pytest.mark.gpu

KERNELS = (C.GRAVITY, C.PLUMMER, C.SMOOTH_DIST)
ALPHA = 25.0


def _setup(dim, dsl, n=6000, seed=11):
    pts, nrm, m = (W.gaussian_mixture(n, seed=seed) if dim == 3 else
                   W.gaussian_mixture(n, seed=seed, dim=2))
    lo, hi = W.padded_box(pts)
    host = C.HostTree(pts, nrm, m, lo, hi, alpha=ALPHA, dim_split_log=dsl)
    orc = O.OracleTree(pts, nrm, m, lo, hi, alpha=ALPHA, dim_split_log=dsl)
    q = np.random.default_rng(seed + 1).uniform(-1.0, 1.0, (700, dim)).astype(np.float32)
    return pts, m, C.GpuTree(host), orc, q


def _close_values(kernel, got, want, rtol):
    got = got.astype(np.float64)
    if kernel == C.SMOOTH_DIST:
        # D = -log(S)/alpha can cross 0: absolute floor of 1e-6 (distance units).
        return np.all(np.abs(got - want) <= rtol * np.abs(want) + 1e-6)
    return np.all(np.abs(got - want) <= rtol * np.abs(want))


def _close_grads(got, want, rtol):
    err = np.linalg.norm(got.astype(np.float64) - want, axis=1)
    return np.all(err <= rtol * np.linalg.norm(want, axis=1) + 1e-30), (
        err / np.maximum(np.linalg.norm(want, axis=1), 1e-30)).max()


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("kernel", KERNELS)
def test_brute_force_gradient_matches_fp64(dim, kernel):
    pts, m, gpu, orc, q = _setup(dim, 1)
    v, g, _ = gpu.eval_grad(q, C.params(method=C.BRUTE_FORCE, kernel=kernel))
    ov, og = O.brute_force_grad_f64(pts, m, kernel, q, ALPHA)
    assert _close_values(kernel, v, ov, 1e-5)
    ok, worst = _close_grads(g, og, 1e-4)
    assert ok, worst


@pytest.mark.parametrize("dim,dsl", [(2, 1), (2, 2), (3, 1), (3, 2)])
@pytest.mark.parametrize("kernel", KERNELS)
def test_barnes_hut_gradient(dim, dsl, kernel):
    pts, m, gpu, orc, q = _setup(dim, dsl)
    p = C.params(method=C.BARNES_HUT, kernel=kernel, beta=2.0)
    v, g, _, cnt = gpu.eval_grad(q, p, contribs=True)
    pv, _, pcnt = gpu.eval(q, p, contribs=True)
    ov, og, ocnt = orc.bh_grad(kernel, q, 2.0, alpha=ALPHA)
    assert np.array_equal(cnt, pcnt) and np.array_equal(cnt, ocnt)
    if kernel != C.SMOOTH_DIST:
        assert bits_equal(v, pv)
    assert _close_values(kernel, v, ov, 1e-5)
    ok, worst = _close_grads(g, og, 1e-4)
    assert ok, worst


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("kernel", KERNELS)
def test_stochastic_gradient_walks_the_same_paths(dim, kernel):
    pts, m, gpu, orc, q = _setup(dim, 2)
    p = C.params(method=C.STOCHASTIC, kernel=kernel, samples_per_subdomain=2, seed=77)
    v, g, _, cnt = gpu.eval_grad(q, p, contribs=True)
    pv, _, pcnt = gpu.eval(q, p, contribs=True)
    ov, og, ocnt = orc.sbh_grad(kernel, q, 2, seed=77, alpha=ALPHA)
    assert np.array_equal(cnt, pcnt) and np.array_equal(cnt, ocnt)
    if kernel != C.SMOOTH_DIST:
        assert bits_equal(v, pv)
        assert _close_values(kernel, v, ov, 1e-4)
        ok, worst = _close_grads(g, og, 1e-3)
        assert ok, worst
    else:
        # The control-variate sums can cancel; where they do, FP32 and FP64
        # sums of the same terms differ.  Compare where the plain FP32 estimate
        # of S agrees with the FP64 one to 1e-4 (no cancellation).
        s_orc = np.exp(-ALPHA * ov)
        keep = np.isfinite(ov) & (np.abs(pv - s_orc) <= 1e-4 * s_orc)
        assert keep.mean() > 0.8
        assert _close_values(kernel, v[keep], ov[keep], 1e-4)
        ok, worst = _close_grads(g[keep], og[keep], 1e-3)
        assert ok, worst


def test_stochastic_gravity_gradient_is_unbiased():
    pts, m, gpu, orc, q = _setup(3, 2, n=4000)
    q = q[:16]
    gs = np.stack([gpu.eval_grad(q, C.params(method=C.STOCHASTIC, kernel=C.GRAVITY,
                                             samples_per_subdomain=1, seed=s))[1]
                   for s in range(1024)]).astype(np.float64)
    _, exact = O.brute_force_grad_f64(pts, m, C.GRAVITY, q)
    se = gs.std(axis=0, ddof=1) / np.sqrt(len(gs))
    assert np.all(np.abs(gs.mean(axis=0) - exact) <= 4 * se + 1e-6 * np.abs(exact))


def test_gradient_rejects_winding_number_and_checks_buffers():
    pts, m, gpu, orc, q = _setup(3, 1, n=500)
    with pytest.raises(C.SbhError) as e:
        gpu.eval_grad(q, C.params(method=C.BARNES_HUT, kernel=C.WINDING_NUMBER))
    assert e.value.status == C.ERR_UNSUPPORTED
    v, g, _ = gpu.eval_grad(q[:0], C.params(method=C.BARNES_HUT))
    assert v.shape == (0,)
    # values only (no gradient buffer)
    v2, g2, _ = gpu.eval_grad(q, C.params(method=C.BARNES_HUT, kernel=C.GRAVITY), grads=False)
    v3, _, _ = gpu.eval_grad(q, C.params(method=C.BARNES_HUT, kernel=C.GRAVITY))
    assert g2 is None and bits_equal(v2, v3)


def test_far_queries_do_not_underflow():
    """exp(-alpha r) underflows FP32 beyond alpha r ~ 104; the max-shifted sums
    keep the smooth distance finite and exact there."""
    pts, nrm, m = W.circle_points(3000, seed=3)
    lo, hi = W.padded_box(pts)
    gpu = C.GpuTree(C.HostTree(pts, nrm, m, lo, hi, alpha=100.0, dim_split_log=1))
    q = np.array([[1.5, 1.5], [-1.5, 1.4], [0.0, 0.0], [3.0, 0.0]], np.float32)
    v, g, _ = gpu.eval_grad(q, C.params(method=C.BRUTE_FORCE, kernel=C.SMOOTH_DIST))
    ov, og = O.brute_force_grad_f64(pts, m, C.SMOOTH_DIST, q, 100.0)
    assert np.all(np.isfinite(v)) and np.allclose(v, ov, rtol=1e-5)
    assert np.allclose(g, og, rtol=1e-4, atol=1e-5)
    plain, _ = gpu.eval(q, C.params(method=C.BRUTE_FORCE, kernel=C.SMOOTH_DIST, alpha=100.0))
    assert plain[3] == 0.0  # the plain FP32 sum underflows at r = 2


@pytest.mark.parametrize("method", ["brute_force", "barnes_hut", "stochastic"])
def test_autograd_function(method):
    torch = pytest.importorskip("torch")
    import sbh_torch
    pts, m, gpu, orc, q = _setup(3, 2, n=3000)
    tq = torch.from_numpy(q[:300]).cuda().requires_grad_(True)
    d = sbh_torch.smooth_distance(gpu, tq, method=method, samples_per_subdomain=2, seed=5)
    w = torch.linspace(0.5, 1.5, 300, device="cuda")
    (d * w).sum().backward()
    meth = {"brute_force": C.BRUTE_FORCE, "barnes_hut": C.BARNES_HUT,
            "stochastic": C.STOCHASTIC}[method]
    v, g, _ = gpu.eval_grad(q[:300], C.params(method=meth, kernel=C.SMOOTH_DIST,
                                              samples_per_subdomain=2, seed=5))
    assert bits_equal(d.detach().cpu().numpy(), v)
    assert np.allclose(tq.grad.cpu().numpy(), g * w.cpu().numpy()[:, None], rtol=1e-6, atol=0)
    # no gradient requested: values only
    with torch.no_grad():
        d2 = sbh_torch.smooth_distance(gpu, tq.detach(), method=method, samples_per_subdomain=2,
                                       seed=5)
    assert bits_equal(d2.cpu().numpy(), v)


def test_autograd_brute_force_matches_fp64_central_differences():
    torch = pytest.importorskip("torch")
    import sbh_torch
    pts, m, gpu, orc, q = _setup(2, 1, n=2000)
    q = q[:50]
    tq = torch.from_numpy(q).cuda().requires_grad_(True)
    sbh_torch.gravity_potential(gpu, tq, method="brute_force").sum().backward()
    h = 1e-4
    fd = np.zeros(q.shape)
    for d in range(2):
        qp, qm = q.copy(), q.copy()
        qp[:, d] += np.float32(h)
        qm[:, d] -= np.float32(h)
        vp, _ = O.brute_force_grad_f64(pts, m, C.GRAVITY, qp)
        vm, _ = O.brute_force_grad_f64(pts, m, C.GRAVITY, qm)
        fd[:, d] = (vp - vm) / (qp[:, d].astype(np.float64) - qm[:, d].astype(np.float64))
    g = tq.grad.cpu().numpy().astype(np.float64)
    err = np.linalg.norm(g - fd, axis=1) / np.linalg.norm(fd, axis=1)
    assert np.median(err) < 1e-5 and err.max() < 1e-3
