"""GPU parity: the CUDA path (through the C ABI) against the oracle.

Tolerances, as stated by the task:
  * brute force: within 1e-6 relative of the FP64 oracle (relative to the sum of
    |terms| where the terms change sign; for smooth distance, within 1e-6 in the
    distance -log(S)/alpha);
  * deterministic Barnes-Hut: identical opened node set (contribution counts)
    and values bit-identical to the reference CPU for gravity, winding number
    and Plummer; smooth distance within 1e-5 relative (CUDA's expf and glibc's
    expf may differ in the last place);
  * stochastic Barnes-Hut: the oracle's estimator driven by the same Philox
    stream takes the same paths (identical contribution counts) and its values
    agree within 2e-5 of each query's summed magnitude; unbiased (means over 1024 replicates within 3 standard
    errors of brute force).  Per-query variance against the reference's, and
    parity on the benchmark's own trees: test_gpu_config_scale.py.
"""
import numpy as np
import pytest

import oracle as O
import sbh_capi as C
import sbh_workloads as W
from conftest import golden_cases, load_golden
from helpers import bits_equal, sampler_close

pytestmark = pytest.mark.gpu

EXACT_KERNELS = (C.GRAVITY, C.WINDING_NUMBER, C.PLUMMER)


def gpu_tree_from(points, normals, masses, lo, hi, alpha=1.0, dsl=1, leaf=1):
    host = C.HostTree(points, normals, masses, lo, hi, alpha=alpha, dim_split_log=dsl,
                      leaf_size=leaf)
    return host, C.GpuTree(host)


def golden_gpu(case):
    g = load_golden(case)
    host, gpu = gpu_tree_from(g["points"], g["normals"], g["masses"], g["min_corner"],
                              g["max_corner"], alpha=float(g["alpha"]),
                              dsl=int(g["dim_split_log"]), leaf=int(g["leaf_size"]))
    return g, host, gpu


# ----------------------------------------------------------------- brute force

@pytest.mark.parametrize("dim,kernel", [(3, C.PLUMMER), (3, C.GRAVITY), (3, C.WINDING_NUMBER),
                                        (3, C.SMOOTH_DIST), (2, C.PLUMMER), (2, C.GRAVITY),
                                        (2, C.WINDING_NUMBER), (2, C.SMOOTH_DIST)])
def test_brute_force_matches_fp64(dim, kernel):
    if dim == 3:
        pts, nrm, m = W.torus_surface(20000, seed=11, jitter=1e-3)
    else:
        pts, nrm, m = W.circle_points(20000, seed=12)
    alpha = 50.0
    lo, hi = W.padded_box(pts)
    _, gpu = gpu_tree_from(pts, nrm, m, lo, hi, alpha=alpha)
    q = W.uniform_queries(2000, seed=13, dim=dim, lo=-1.5, hi=1.5)
    got, _ = gpu.eval(q, C.params(method=C.BRUTE_FORCE, kernel=kernel, eps=1e-3))
    ref = O.brute_force_f64(pts, nrm, m, kernel, q, alpha=alpha, eps=1e-3)
    if kernel in (C.PLUMMER, C.GRAVITY):
        err = np.abs(got - ref) / np.abs(ref)
        assert err.max() <= 1e-6, err.max()
    elif kernel == C.WINDING_NUMBER:
        scale = O.brute_force_f64(pts, nrm, m, kernel, q, alpha=alpha, abs_sum=True)
        err = np.abs(got - ref) / scale
        assert err.max() <= 1e-6, err.max()
    else:
        ok = ref > 0
        d_got = -np.log(got[ok].astype(np.float64)) / alpha
        d_ref = -np.log(ref[ok]) / alpha
        assert np.abs(d_got - d_ref).max() <= 1e-6


@pytest.mark.parametrize("batched", [False, True])
def test_brute_force_smooth_distance_far_queries(batched):
    # Every term is an FP32 subnormal (alpha * r between 90 and 103): the
    # exponential's scaled form must keep them, in both the single-call kernel
    # and the batched brute-force task.
    pts, nrm, m = W.sphere_surface(20000, seed=31, radius=0.05)
    lo, hi = W.padded_box(pts)
    _, gpu = gpu_tree_from(pts, nrm, m, lo, hi)
    rng = np.random.default_rng(32)
    d = rng.normal(size=(3000, 3))
    q = (d / np.linalg.norm(d, axis=1, keepdims=True) *
         rng.uniform(0.95, 0.98, (3000, 1))).astype(np.float32)
    alpha = 100.0
    p = C.params(method=C.BRUTE_FORCE, kernel=C.SMOOTH_DIST, alpha=alpha)
    if batched:
        import torch
        dq = torch.from_numpy(np.ascontiguousarray(q.T)).cuda()
        out = torch.empty(len(q), dtype=torch.float32, device="cuda")
        C.eval_batch([(gpu, p, dq.data_ptr(), len(q), out.data_ptr(), 0, 0)])
        torch.cuda.synchronize()
        got = out.cpu().numpy()
    else:
        got, _ = gpu.eval(q, p)
    ref = O.brute_force_f64(pts, nrm, m, C.SMOOTH_DIST, q, alpha=alpha)
    nearest = np.sqrt(((q[:, None, :] - pts[None, ::7, :]) ** 2).sum(-1)).min()
    assert alpha * nearest > 88.0  # exp(-88) < 2^-126: every term is subnormal
    d_got = -np.log(got.astype(np.float64)) / alpha
    d_ref = -np.log(ref) / alpha
    assert np.abs(d_got - d_ref).max() <= 1e-6


def test_brute_force_plain_small_workload():
    # Plummer potential over 65,536 Gaussian-mixture sources (the plain-method workload).
    pts, nrm, m = W.gaussian_mixture(65536, seed=21)
    lo, hi = W.padded_box(pts)
    _, gpu = gpu_tree_from(pts, nrm, m, lo, hi, leaf=8)
    q = W.uniform_queries(4096, seed=22)
    got, ms = gpu.eval(q, C.params(method=C.BRUTE_FORCE, kernel=C.PLUMMER, eps=1e-3))
    ref = O.brute_force_f64(pts, nrm, m, O.PLUMMER, q, eps=1e-3)
    assert (np.abs(got - ref) / ref).max() <= 1e-6
    assert ms > 0


# ------------------------------------------------------------- Barnes-Hut

@pytest.mark.parametrize("case", golden_cases())
def test_barnes_hut_matches_reference_bitwise(case):
    g, _, gpu = golden_gpu(case)
    for kernel in (C.GRAVITY, C.WINDING_NUMBER, C.SMOOTH_DIST, C.PLUMMER):
        for beta in (2.0, 1.25):
            v, _, cnt = gpu.eval(g["queries"], C.params(method=C.BARNES_HUT, kernel=kernel,
                                                        beta=beta, eps=1e-3), contribs=True)
            ref = g[f"bh_k{kernel}_b{beta}"]
            assert np.array_equal(cnt, g[f"bh_counts_k{kernel}_b{beta}"]), (kernel, beta)
            if kernel in EXACT_KERNELS:
                assert bits_equal(v, ref), (kernel, beta, np.abs(v - ref).max())
            else:
                assert np.allclose(v, ref, rtol=1e-5, atol=0), (kernel, beta)


@pytest.mark.parametrize("case", ["oct1_leaf8_gauss", "oct2_leaf8_torus", "oct1_gauss"])
def test_barnes_hut_staged_leaves_bitwise(case):
    """Leaf points copied to shared memory by bulk copies (SBH_FLAG_STAGE_LEAVES)
    give the reference's values and node sets bit for bit."""
    g, _, gpu = golden_gpu(case)
    for kernel in (C.GRAVITY, C.WINDING_NUMBER, C.PLUMMER):
        for beta in (2.0, 1.25):
            v, _, cnt = gpu.eval(g["queries"], C.params(method=C.BARNES_HUT, kernel=kernel,
                                                        beta=beta, eps=1e-3,
                                                        flags=C.FLAG_STAGE_LEAVES),
                                 contribs=True)
            assert np.array_equal(cnt, g[f"bh_counts_k{kernel}_b{beta}"]), (kernel, beta)
            assert bits_equal(v, g[f"bh_k{kernel}_b{beta}"]), (kernel, beta)
    gpu.check()


def test_barnes_hut_staged_leaves_large_leaves():
    """Leaves of more than 32 points (duplicates at the depth cap) are staged 32
    points at a time."""
    rng = np.random.default_rng(5)
    p = np.concatenate([np.tile([[0.1, 0.2, 0.3]], (70, 1)),
                        rng.uniform(-1, 1, (500, 3))]).astype(np.float32)
    nr = rng.normal(size=p.shape).astype(np.float32)
    m = rng.uniform(0.5, 1.5, len(p)).astype(np.float32)
    lo, hi = -np.ones(3, np.float32), np.ones(3, np.float32)
    ot = O.OracleTree(p, nr, m, lo, hi, leaf_size=8)
    _, gpu = gpu_tree_from(p, nr, m, lo, hi, leaf=8)
    q = np.concatenate([np.array([[0.1, 0.2, 0.3], [0.1, 0.2, 0.30001]], np.float32),
                        W.uniform_queries(200, seed=6)])
    for kernel in (C.GRAVITY, C.WINDING_NUMBER):
        rv, rc, _ = ot.bh(kernel, q, 2.0)
        v, _, cnt = gpu.eval(q, C.params(method=C.BARNES_HUT, kernel=kernel, beta=2.0,
                                         flags=C.FLAG_STAGE_LEAVES), contribs=True)
        assert np.array_equal(cnt, rc)
        assert bits_equal(v, rv)
    gpu.check()


@pytest.mark.parametrize("case", ["oct1_gauss", "quad2_gauss", "oct2_torus"])
def test_barnes_hut_order_independent(case):
    g, _, gpu = golden_gpu(case)
    q = np.concatenate([g["queries"]] * 5)
    a, _ = gpu.eval(q, C.params(method=C.BARNES_HUT, kernel=C.GRAVITY, beta=2.0))
    b, _ = gpu.eval(q, C.params(method=C.BARNES_HUT, kernel=C.GRAVITY, beta=2.0,
                                flags=C.FLAG_KEEP_ORDER))
    assert bits_equal(a, b)


@pytest.mark.parametrize("case", ["oct1_gauss", "oct2_torus", "quad1_circle", "oct1_leaf8_gauss"])
def test_barnes_hut_vote_matches_oracle(case):
    g, _, gpu = golden_gpu(case)
    ot = O.OracleTree(g["points"], g["normals"], g["masses"], g["min_corner"], g["max_corner"],
                      alpha=float(g["alpha"]), dim_split_log=int(g["dim_split_log"]),
                      leaf_size=int(g["leaf_size"]))
    q = g["queries"][:90]  # a partial last warp
    for kernel in EXACT_KERNELS:
        v, _, cnt = gpu.eval(q, C.params(method=C.BARNES_HUT_VOTE, kernel=kernel, beta=2.0),
                             contribs=True)
        rv, rc = ot.bh_vote(kernel, q, 2.0, group=32)
        assert np.array_equal(cnt, rc)
        assert bits_equal(v, rv)


def test_barnes_hut_exact_beta_is_brute_force():
    pts, nrm, m = W.gaussian_mixture(3000, seed=31)
    lo, hi = W.padded_box(pts)
    host, gpu = gpu_tree_from(pts, nrm, m, lo, hi)
    q = W.uniform_queries(500, seed=32)
    v, _, cnt = gpu.eval(q, C.params(method=C.BARNES_HUT, kernel=C.PLUMMER, beta=np.inf),
                         contribs=True)
    assert (cnt == 3000).all()
    ref = O.brute_force_f64(pts, nrm, m, O.PLUMMER, q)
    assert (np.abs(v - ref) / ref).max() < 1e-5


# -------------------------------------------------------------- sampler

@pytest.mark.parametrize("case", golden_cases())
def test_sampler_matches_oracle(case):
    g, _, gpu = golden_gpu(case)
    ot = O.OracleTree(g["points"], g["normals"], g["masses"], g["min_corner"], g["max_corner"],
                      alpha=float(g["alpha"]), dim_split_log=int(g["dim_split_log"]),
                      leaf_size=int(g["leaf_size"]))
    q = g["queries"]
    for kernel in (C.GRAVITY, C.WINDING_NUMBER, C.SMOOTH_DIST, C.PLUMMER):
        for samples, seed in ((1, 0), (3, 12345678901)):
            rv, rc, sc = ot.sbh(kernel, q, samples, rng=O.RNG_PHILOX, seed=seed,
                                return_scale=True)
            v, _, cnt = gpu.eval(q, C.params(method=C.STOCHASTIC, kernel=kernel,
                                             samples_per_subdomain=samples, seed=seed),
                                 contribs=True)
            # Same paths (identical contribution counts) and the same terms;
            # only the order of each node's children sum differs.
            assert np.array_equal(cnt, rc), (kernel, samples)
            assert sampler_close(v, rv, sc), (kernel, samples, np.abs(v - rv).max())


def _replicate_stats(gpu, q, kernel, samples, reps):
    nq = len(q)
    qq = np.tile(q, (reps, 1))  # query index differs per replicate: independent streams
    v, _ = gpu.eval(qq, C.params(method=C.STOCHASTIC, kernel=kernel,
                                 samples_per_subdomain=samples, seed=99))
    v = v.reshape(reps, nq).astype(np.float64)
    return v.mean(0), v.var(0, ddof=1)


@pytest.mark.parametrize("workload", ["torus_wn", "gauss_gravity", "circle_wn2d"])
def test_sampler_unbiased(workload):
    if workload == "torus_wn":
        pts, nrm, m = W.torus_surface(4000, seed=41)
        kernel, dsl, dim = C.WINDING_NUMBER, 2, 3
    elif workload == "gauss_gravity":
        pts, nrm, m = W.gaussian_mixture(4000, seed=42)
        kernel, dsl, dim = C.GRAVITY, 2, 3
    else:
        pts, nrm, m = W.circle_points(4000, seed=43)
        kernel, dsl, dim = C.WINDING_NUMBER, 2, 2
    lo, hi = W.padded_box(pts)
    _, gpu = gpu_tree_from(pts, nrm, m, lo, hi, dsl=dsl)
    q = W.uniform_queries(64, seed=44, dim=dim)
    reps = 1024
    mean, var = _replicate_stats(gpu, q, kernel, 1, reps)
    exact = O.brute_force_f64(pts, nrm, m, kernel, q)
    se = np.sqrt(var / reps)
    z = (mean - exact) / np.maximum(se, 1e-300)
    live = se > 1e-12 * np.abs(exact).max()
    z = z[live]
    # Each query within 3 SE, allowing the expected ~0.3% excursions; none beyond 5 SE;
    # and the mean z-score consistent with zero.
    assert (np.abs(z) <= 3).mean() >= 0.95
    assert np.abs(z).max() <= 5
    assert abs(z.mean()) <= 4 / np.sqrt(len(z))


def test_sampler_seed_semantics():
    g, _, gpu = golden_gpu("oct2_torus")
    q = g["queries"]
    p = C.params(method=C.STOCHASTIC, kernel=C.WINDING_NUMBER, samples_per_subdomain=2, seed=7)
    a, _ = gpu.eval(q, p)
    b, _ = gpu.eval(q, p)
    assert bits_equal(a, b)
    c, _ = gpu.eval(q, C.params(method=C.STOCHASTIC, kernel=C.WINDING_NUMBER,
                                samples_per_subdomain=2, seed=8))
    assert not bits_equal(a, c)
    k, _ = gpu.eval(q, C.params(method=C.STOCHASTIC, kernel=C.WINDING_NUMBER,
                                samples_per_subdomain=2, seed=7, flags=C.FLAG_KEEP_ORDER))
    assert bits_equal(a, k)


# ------------------------------------------------------------ edge cases

def test_empty_tree_and_empty_queries():
    z = np.zeros((0, 3), np.float32)
    host, gpu = gpu_tree_from(z, z, np.zeros(0, np.float32), -np.ones(3), np.ones(3))
    q = W.uniform_queries(33, seed=1)
    for method in (C.BRUTE_FORCE, C.BARNES_HUT, C.BARNES_HUT_VOTE, C.STOCHASTIC):
        v, _ = gpu.eval(q, C.params(method=method, kernel=C.GRAVITY))
        assert (v == 0).all()
    v, ms = gpu.eval(np.zeros((0, 3), np.float32), C.params(method=C.BARNES_HUT))
    assert v.shape == (0,)


@pytest.mark.parametrize("nq", [1, 31, 33, 1000])
def test_ragged_query_counts(nq):
    g, _, gpu = golden_gpu("oct1_gauss")
    q = W.uniform_queries(nq, seed=nq)
    ot = O.OracleTree(g["points"], g["normals"], g["masses"], g["min_corner"], g["max_corner"])
    v, _ = gpu.eval(q, C.params(method=C.BARNES_HUT, kernel=C.GRAVITY, beta=2.0))
    rv, _, _ = ot.bh(O.GRAVITY, q, 2.0)
    assert bits_equal(v, rv)
    s, _ = gpu.eval(q, C.params(method=C.STOCHASTIC, kernel=C.GRAVITY, samples_per_subdomain=2))
    rs, _, sc = ot.sbh(O.GRAVITY, q, 2, rng=O.RNG_PHILOX, seed=0, return_scale=True)
    assert sampler_close(s, rs, sc)


def test_duplicate_points_chain_on_gpu():
    p = np.array([[0.3, 0.2, 0.1]] * 9 + [[0.5, -0.5, 0.5], [-0.3, 0.1, 0.9]], np.float32)
    nr, m = np.ones_like(p), np.ones(len(p), np.float32)
    lo, hi = -np.ones(3, np.float32), np.ones(3, np.float32)
    q = np.array([[0, 0, 0], [0.3, 0.2, 0.1], [2, 2, 2]], np.float32)
    ot = O.OracleTree(p, nr, m, lo, hi)
    _, gpu = gpu_tree_from(p, nr, m, lo, hi)
    v, _ = gpu.eval(q, C.params(method=C.BARNES_HUT, kernel=C.GRAVITY, beta=2.0))
    assert bits_equal(v, ot.bh(O.GRAVITY, q, 2.0)[0])
    s, _ = gpu.eval(q, C.params(method=C.STOCHASTIC, kernel=C.GRAVITY, samples_per_subdomain=3))
    rs, _, sc = ot.sbh(O.GRAVITY, q, 3, rng=O.RNG_PHILOX, seed=0, return_scale=True)
    assert sampler_close(s, rs, sc)


def test_invalid_requests_are_rejected():
    g, _, gpu = golden_gpu("oct1_gauss")
    with pytest.raises(C.SbhError) as e:
        gpu.eval(g["queries"], C.params(method=C.STOCHASTIC, samples_per_subdomain=0))
    assert e.value.status == C.ERR_INVALID_ARGUMENT
    with pytest.raises(C.SbhError):
        gpu.eval(g["queries"], C.params(method=9))
    with pytest.raises(C.SbhError):
        gpu.eval(g["queries"], C.params(kernel=7))
    # The tree stays usable after rejected calls.
    v, _ = gpu.eval(g["queries"], C.params(method=C.BARNES_HUT, kernel=C.GRAVITY))
    assert bits_equal(v, g["bh_k0_b2.0"])


def test_loaded_tree_evaluates_identically(tmp_path):
    """A tree saved and loaded (sbh_host_tree_save/load) uploads and evaluates
    exactly as the tree it was saved from."""
    pts, nrm, a = W.torus_surface(20000, seed=29)
    lo, hi = W.padded_box(pts)
    t = C.HostTree(pts, nrm, a, lo, hi, dim_split_log=2)
    t.save(str(tmp_path / "t.sbht"))
    u = C.HostTree.load(str(tmp_path / "t.sbht"))
    g1, g2 = C.GpuTree(t), C.GpuTree(u)
    q = W.uniform_queries(3000, seed=30)
    for p in (C.params(method=C.BARNES_HUT, kernel=C.WINDING_NUMBER, beta=2.0),
              C.params(method=C.STOCHASTIC, kernel=C.WINDING_NUMBER, samples_per_subdomain=2,
                       seed=4)):
        assert bits_equal(g1.eval(q, p)[0], g2.eval(q, p)[0])
