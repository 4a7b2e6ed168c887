"""Shared helpers for the tests (bit-level comparisons, tree comparisons)."""
import numpy as np


def bits_equal(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    if a.shape != b.shape:
        return False
    if a.dtype.kind == "f":
        return np.array_equal(a.view(np.uint32 if a.dtype == np.float32 else np.uint64),
                              b.astype(a.dtype).view(np.uint32 if a.dtype == np.float32 else np.uint64))
    return np.array_equal(a, b)


def sampler_close(v, rv, scale, rtol=2e-5):
    """The GPU sampler against the oracle's estimator on the same Philox paths.
    Both take the same terms; the GPU adds each node's children as a balanced
    tree, the oracle left to right, so they differ by rounding: at most a few
    ulp of `scale`, the magnitude of everything the estimate sums (orc_sbh's
    scales).  NaN where the oracle has NaN."""
    v = np.asarray(v, np.float64)
    rv = np.asarray(rv, np.float64)
    nan = np.isnan(rv)
    if not np.array_equal(np.isnan(v), nan):
        return False
    return bool(np.all(np.abs(v[~nan] - rv[~nan]) <= rtol * np.asarray(scale)[~nan] + 1e-30))


def tree_mismatches(nodes, points, g):
    """Fields of a product tree export that differ (bitwise) from a golden record."""
    bad = []
    pairs = [("start", nodes["start"], g["start"]), ("end", nodes["end"], g["end"]),
             ("parent", nodes["parent"], g["parent"]), ("depth", nodes["depth"], g["depth"]),
             ("num_children", nodes["num_children"], g["num_children"]),
             ("is_leaf", nodes["is_leaf"].astype(bool), g["is_leaf"].astype(bool)),
             ("mask", nodes["mask"], g["mask"]), ("bmin", nodes["bmin"], g["bmin"]),
             ("bmax", nodes["bmax"], g["bmax"]), ("diameter", nodes["diameter"], g["diameter"]),
             ("agg", nodes["agg"], g["agg"]), ("points", points["points"], g["perm_points"]),
             ("normals", points["normals"], g["perm_normals"]),
             ("masses", points["masses"], g["perm_masses"])]
    for name, a, b in pairs:
        if not bits_equal(a, b):
            bad.append(name)
    internal = ~g["is_leaf"].astype(bool)
    if not np.array_equal(nodes["first_child"][internal], g["first_child"][internal]):
        bad.append("first_child")
    return bad
