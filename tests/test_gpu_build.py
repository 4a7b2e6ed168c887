"""The GPU tree build (sbh_gpu_tree_build) against the host build + upload:
the device images must be identical bit for bit -- points in build order,
every node record, masks and path codes -- and evaluate identically."""
import numpy as np
import pytest

import sbh_capi as C
import sbh_workloads as W
from helpers import bits_equal

pytestmark = pytest.mark.gpu


def _inputs(kind, n, seed):
    if kind == "torus":
        return W.torus_surface(n, seed=seed)
    if kind == "gauss":
        return W.gaussian_mixture(n, seed=seed)
    if kind == "gauss2":
        return W.gaussian_mixture(n, seed=seed, dim=2)
    if kind == "circle":
        return W.circle_points(n, seed=seed)
    if kind == "sphere":
        return W.sphere_surface(n, seed=seed)
    rng = np.random.default_rng(seed)
    dim = 3 if kind == "uniform" else 2
    p = rng.uniform(-1, 1, (n, dim)).astype(np.float32)
    return p, np.ones_like(p), rng.uniform(0.5, 1.5, n).astype(np.float32)


CASES = [("torus", 200000, 1), ("torus", 50000, 2), ("gauss", 100000, 1), ("gauss", 30000, 3),
         ("sphere", 40000, 2), ("uniform", 60000, 2), ("gauss2", 80000, 1), ("circle", 50000, 2),
         ("uniform2", 20000, 3), ("gauss", 1, 1), ("gauss", 0, 2), ("torus", 7, 1)]


@pytest.mark.parametrize("kind,n,dsl", CASES)
def test_gpu_build_equals_host_build(kind, n, dsl):
    pts, nrm, m = _inputs(kind, max(n, 1), seed=n + dsl)
    pts, nrm, m = pts[:n], nrm[:n], m[:n]
    lo, hi = W.padded_box(pts) if n else (np.full(pts.shape[1], -1, np.float32),
                                          np.full(pts.shape[1], 1, np.float32))
    ref = C.GpuTree(C.HostTree(pts, nrm, m, lo, hi, alpha=7.0, dim_split_log=dsl))
    got = C.GpuTree.build(pts, nrm, m, lo, hi, alpha=7.0, dim_split_log=dsl)
    assert got.built_on_device
    for f in ("num_points", "num_nodes", "depth", "root_children", "dim_split_log"):
        assert getattr(got.info, f) == getattr(ref.info, f), f
    a, b = ref.export(), got.export()
    for k in a:
        assert bits_equal(a[k], b[k]), k
    if n:
        q = W.uniform_queries(2000, seed=5, dim=pts.shape[1])
        for p in (C.params(method=C.BARNES_HUT, kernel=C.GRAVITY, beta=2.0),
                  C.params(method=C.STOCHASTIC, kernel=C.GRAVITY, samples_per_subdomain=2)):
            assert bits_equal(ref.eval(q, p)[0], got.eval(q, p)[0])


def test_gpu_build_falls_back_where_partition_order_matters():
    pts, nrm, m = W.gaussian_mixture(20000, seed=3)
    lo, hi = W.padded_box(pts)
    # leaf size 8: std::partition's order inside leaves -> host build
    g = C.GpuTree.build(pts, nrm, m, lo, hi, dim_split_log=1, leaf_size=8)
    ref = C.GpuTree(C.HostTree(pts, nrm, m, lo, hi, dim_split_log=1, leaf_size=8))
    assert not g.built_on_device
    a, b = ref.export(), g.export()
    for k in a:
        assert bits_equal(a[k], b[k]), k
    # duplicate points reach the depth cap together -> host build
    p = np.array([[0.3, 0.2, 0.1]] * 5 + [[0.5, -0.5, 0.5]], np.float32)
    g = C.GpuTree.build(p, np.ones_like(p), np.ones(6, np.float32), -np.ones(3, np.float32),
                        np.ones(3, np.float32), max_depth=20)
    assert not g.built_on_device and g.info.depth == 20


def test_server_serves_device_built_trees():
    pts, nrm, a = W.torus_surface(30000, seed=8)
    lo, hi = W.padded_box(pts)
    g = C.GpuTree.build(pts, nrm, a, lo, hi, dim_split_log=2)
    server = C.Server(slots=2, slot_queries=4096)
    tid = server.add_tree(g)
    q = W.uniform_queries(10000, seed=9)
    p = C.params(method=C.STOCHASTIC, kernel=C.WINDING_NUMBER, samples_per_subdomain=2, seed=1)
    r = server.submit(tid, q, p)
    assert bits_equal(r.wait(), g.eval(q, p)[0])
    server.close()
