"""The product's host tree build (csrc/host_tree.cpp) against the reference.

Bit-exact comparison of every node field and of the point permutation with the
golden vectors the reference produced, through both the C ABI and the `sbh`
pybind11 module; plus the edge cases of the build.  No GPU needed.
"""
import numpy as np
import pytest

import sbh
import sbh_capi as C
import sbh_workloads as W
from conftest import golden_cases, load_golden
from helpers import bits_equal, tree_mismatches

NAMED = {(2, 1): sbh.Quadtree1, (2, 2): sbh.Quadtree2, (2, 3): sbh.Quadtree3,
         (3, 1): sbh.Octree1, (3, 2): sbh.Octree2, (3, 3): sbh.Octree3}


@pytest.mark.parametrize("case", golden_cases())
def test_capi_tree_matches_reference(case):
    g = load_golden(case)
    t = C.HostTree(g["points"], g["normals"], g["masses"], g["min_corner"], g["max_corner"],
                   alpha=float(g["alpha"]), dim_split_log=int(g["dim_split_log"]),
                   leaf_size=int(g["leaf_size"]))
    assert t.info().num_nodes == len(g["start"])
    assert tree_mismatches(t.export_nodes(), t.export_points(), g) == []


@pytest.mark.parametrize("case", golden_cases())
def test_pybind_tree_matches_reference(case):
    g = load_golden(case)
    args = (g["points"].astype(np.float64), g["normals"], g["masses"], g["min_corner"],
            g["max_corner"])
    if int(g["leaf_size"]) == 1:
        cls = NAMED[(int(g["dim"]), int(g["dim_split_log"]))]
        t = cls(*args, alpha=float(g["alpha"]))
    else:
        t = sbh.Tree(*args, alpha=float(g["alpha"]), dim_split_log=int(g["dim_split_log"]),
                     leaf_size=int(g["leaf_size"]))
    assert tree_mismatches(t.export_nodes(), t.export_points(), g) == []


def test_named_classes_are_the_plugin_types():
    pts, nrm, m = W.gaussian_mixture(300, seed=1)
    lo, hi = W.padded_box(pts)
    t = sbh.Octree2(pts, nrm, m, lo, hi)
    assert (t.dim, t.dim_split_log, t.leaf_size, t.max_depth) == (3, 2, 1, 100)
    assert isinstance(t, sbh.Tree)
    assert sbh.fp == 32


def test_empty_tree():
    z = np.zeros((0, 3), np.float32)
    t = C.HostTree(z, z, np.zeros(0, np.float32), -np.ones(3), np.ones(3))
    i = t.info()
    assert (i.num_points, i.num_nodes, i.root_children) == (0, 1, 0)


def test_single_point_and_pair():
    p = np.array([[0.1, 0.2, 0.3]], np.float32)
    t = C.HostTree(p, p, np.ones(1), -np.ones(3), np.ones(3))
    assert t.info().num_nodes == 1
    p2 = np.array([[0.1, 0.2, 0.3], [-0.5, 0.5, 0.5]], np.float32)
    t2 = C.HostTree(p2, p2, np.ones(2), -np.ones(3), np.ones(3))
    nodes = t2.export_nodes()
    assert t2.info().num_nodes == 3 and nodes["num_children"][0] == 2


def test_duplicate_points_reach_depth_cap():
    p = np.array([[0.3, 0.2, 0.1]] * 9 + [[0.5, -0.5, 0.5], [-0.3, 0.1, 0.9]], np.float32)
    t = C.HostTree(p, np.ones_like(p), np.ones(len(p)), -np.ones(3), np.ones(3))
    i = t.info()
    assert i.num_nodes == 103 and i.depth == 100


def test_points_outside_the_box_are_clamped_into_cells():
    pts = np.array([[2.0, 0.0, 0.0], [-3.0, 0.5, 0.1], [0.1, 0.1, 0.1]], np.float32)
    t = C.HostTree(pts, pts, np.ones(3), -np.ones(3), np.ones(3))
    assert t.info().num_nodes >= 3


@pytest.mark.parametrize("bad", [dict(dim_split_log=0), dict(dim_split_log=4), dict(leaf_size=0),
                                 dict(max_depth=-1)])
def test_invalid_arguments_raise(bad):
    pts = np.zeros((4, 3), np.float32)
    with pytest.raises(C.SbhError) as e:
        C.HostTree(pts, pts, np.ones(4), -np.ones(3), np.ones(3), **bad)
    assert e.value.status == C.ERR_INVALID_ARGUMENT


def test_wrong_dimension_raises():
    with pytest.raises(C.SbhError):
        C.HostTree(np.zeros((4, 4), np.float32), np.zeros((4, 4), np.float32), np.ones(4),
                   -np.ones(4), np.ones(4))
    with pytest.raises(ValueError):
        sbh.Octree1(np.zeros((4, 2)), np.zeros((4, 2)), np.ones(4), -np.ones(3), np.ones(3))


def test_large_torus_build_is_deterministic():
    pts, nrm, a = W.torus_surface(200_000, seed=5)
    lo, hi = W.padded_box(pts)
    t1 = C.HostTree(pts, nrm, a, lo, hi, dim_split_log=2)
    t2 = C.HostTree(pts, nrm, a, lo, hi, dim_split_log=2)
    e1, e2 = t1.export_nodes(), t2.export_nodes()
    for k in e1:
        assert np.array_equal(e1[k], e2[k]), k


# ------------------------------------------------------------ serialisation

def test_save_load_roundtrip_is_bit_identical(tmp_path):
    pts, nrm, m = W.torus_surface(5000, seed=17)
    lo, hi = W.padded_box(pts)
    for dsl, leaf in ((1, 1), (2, 1), (1, 8)):
        t = C.HostTree(pts, nrm, m, lo, hi, alpha=3.5, dim_split_log=dsl, leaf_size=leaf)
        path = str(tmp_path / f"tree_{dsl}_{leaf}.sbht")
        t.save(path)
        u = C.HostTree.load(path)
        a, b = t.export_nodes(), u.export_nodes()
        for k in a:
            assert bits_equal(a[k], b[k]), k
        pa, pb = t.export_points(), u.export_points()
        for k in pa:
            assert bits_equal(pa[k], pb[k]), k
        ia, ib = t.info(), u.info()
        assert (ia.num_nodes, ia.depth, ia.root_children, ia.alpha) == \
            (ib.num_nodes, ib.depth, ib.root_children, ib.alpha)


def test_load_rejects_damaged_files(tmp_path):
    pts, nrm, m = W.gaussian_mixture(2000, seed=18)
    lo, hi = W.padded_box(pts)
    t = C.HostTree(pts, nrm, m, lo, hi, dim_split_log=2)
    path = tmp_path / "t.sbht"
    t.save(str(path))
    raw = bytearray(path.read_bytes())
    bad = tmp_path / "bad.sbht"
    for damage in ("flip", "truncate", "magic"):
        b = bytearray(raw)
        if damage == "flip":
            b[len(b) // 2] ^= 0x40
        elif damage == "truncate":
            b = b[: len(b) - 100]
        else:
            b[0:4] = b"XXXX"
        bad.write_bytes(bytes(b))
        with pytest.raises(C.SbhError) as e:
            C.HostTree.load(str(bad))
        assert e.value.status == C.ERR_INVALID_ARGUMENT
    with pytest.raises(C.SbhError):
        C.HostTree.load(str(tmp_path / "missing.sbht"))
