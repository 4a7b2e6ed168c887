"""The reference-facing surface on the GPU: `sbh` / `sbh_gpu` modules and the
C ABI's device-pointer entry point."""
import numpy as np
import pytest

import oracle as O
import sbh
import sbh_capi as C
import sbh_gpu
import sbh_workloads as W
from helpers import bits_equal, sampler_close

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torus():
    pts, nrm, a = W.torus_surface(20000, seed=61)
    lo, hi = W.padded_box(pts)
    return pts, nrm, a, lo, hi


def test_reference_call_sequence(torus):
    # python/example.py:27-28,54-55,97-127: build on the host, upload, evaluate.
    pts, nrm, a, lo, hi = torus
    cpu1 = sbh.Octree1(pts.astype(np.float64), nrm, a, lo, hi)
    cpu2 = sbh.Octree2(pts.astype(np.float64), nrm, a, lo, hi)
    g1 = sbh_gpu.OctreeGPU1(cpu1)
    g2 = sbh_gpu.OctreeGPU2(cpu2)
    q = W.uniform_queries(1000, seed=62).astype(np.float64)
    gt, t_gt = sbh_gpu.eval_brute_force_wn(g1, q)
    bh, t_bh = sbh_gpu.eval_barnes_hut_wn(g1, q, 2)
    sb, t_sb = sbh_gpu.multi_level_prefix_control_variate_wn(g2, q, 1)
    for arr, t in ((gt, t_gt), (bh, t_bh), (sb, t_sb)):
        assert arr.dtype == np.float32 and arr.shape == (1000,)
        assert isinstance(t, float) and t >= 0
    # winding number: ~1 inside the torus tube, ~0 outside
    assert np.median(np.abs(bh - gt)) < 1e-2
    ot = O.OracleTree(pts, nrm, a, lo, hi)
    assert bits_equal(bh, ot.bh(O.WINDING_NUMBER, q, 2.0)[0])


def test_gpu_tree_type_must_match(torus):
    pts, nrm, a, lo, hi = torus
    cpu = sbh.Octree1(pts, nrm, a, lo, hi)
    with pytest.raises(TypeError):
        sbh_gpu.OctreeGPU2(cpu)
    with pytest.raises(TypeError):
        sbh_gpu.OctreeGPU1(object())


def test_cpu_named_functions_run_on_gpu(torus):
    pts, nrm, a, lo, hi = torus
    t = sbh.Octree2(pts, nrm, a, lo, hi)
    q = W.uniform_queries(300, seed=63)
    v = sbh.eval_barnes_hut_gravity(t, q, 2.0)
    assert v.shape == (300,) and v.dtype == np.float32
    s, counts = sbh.multi_level_prefix_control_variate_gravity(t, q, 2)
    assert s.shape == (300,) and counts.dtype == np.int32 and (counts > 0).all()
    ot = O.OracleTree(pts, nrm, a, lo, hi, dim_split_log=2)
    assert bits_equal(v, ot.bh(O.GRAVITY, q, 2.0)[0])
    rs, rc, sc = ot.sbh(O.GRAVITY, q, 2, rng=O.RNG_PHILOX, seed=0, return_scale=True)
    assert sampler_close(s, rs, sc) and np.array_equal(counts, rc)


def test_extended_keywords(torus):
    pts, nrm, a, lo, hi = torus
    g = sbh_gpu.TreeGPU(sbh.Tree(pts, nrm, a, lo, hi, dim_split_log=2, leaf_size=8))
    q = W.uniform_queries(200, seed=64)
    v, ms, cnt = sbh_gpu.multi_level_prefix_control_variate_plummer(g, q, 3, seed=5,
                                                                   return_counts=True)
    assert cnt.shape == (200,)
    v2, _ = sbh_gpu.eval_barnes_hut_smoothdist(g, q, 2.0, alpha=20.0)
    assert np.isfinite(v2).all()
    v3, _ = sbh_gpu.eval_barnes_hut_gravity(g, q, 2.0, vote=True)
    v4, _ = sbh_gpu.eval_barnes_hut_gravity(g, q, 2.0)
    assert np.allclose(v3, v4, rtol=1e-2)  # vote opens a superset of the nodes


def test_device_pointer_entry_point(torus):
    torch = pytest.importorskip("torch")
    pts, nrm, a, lo, hi = torus
    host = C.HostTree(pts, nrm, a, lo, hi, dim_split_log=2)
    gpu = C.GpuTree(host)
    q = W.uniform_queries(5000, seed=65)
    dq = torch.from_numpy(np.ascontiguousarray(q.T)).cuda()
    out = torch.empty(5000, dtype=torch.float32, device="cuda")
    cnt = torch.empty(5000, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for method in (C.BARNES_HUT, C.STOCHASTIC, C.BRUTE_FORCE):
        p = C.params(method=method, kernel=C.WINDING_NUMBER, samples_per_subdomain=2)
        gpu.eval_device(dq.data_ptr(), 5000, out.data_ptr(), p, stream=stream,
                        d_contribs=cnt.data_ptr())
        gpu.check(stream)
        ref, _, rcnt = gpu.eval(q, p, contribs=True)
        assert bits_equal(out.cpu().numpy(), ref)
        assert np.array_equal(cnt.cpu().numpy(), rcnt)


@pytest.mark.parametrize("n", [1, 70000, 200003])
def test_float64_queries_convert_exactly(torus, n):
    """Queries passed as a C-ordered float64 (n, 3) array -- the reference's
    callers' form -- are converted to float32 by the module's threads; the
    results equal those of the same queries given as float32 bit for bit, for
    every method."""
    pts, nrm, a, lo, hi = torus
    g1 = sbh_gpu.OctreeGPU1(sbh.Octree1(pts, nrm, a, lo, hi))
    g2 = sbh_gpu.OctreeGPU2(sbh.Octree2(pts, nrm, a, lo, hi))
    q64 = np.random.default_rng(n).uniform(-1.2, 1.2, (n, 3))
    q32 = np.asfortranarray(q64.astype(np.float32))
    assert q64.flags.c_contiguous
    for f in (lambda q: sbh_gpu.eval_brute_force_gravity(g1, q),
              lambda q: sbh_gpu.eval_barnes_hut_wn(g1, q, 2.0),
              lambda q: sbh_gpu.multi_level_prefix_control_variate_gravity(g2, q, 1)):
        assert bits_equal(f(q64)[0], f(q32)[0])
