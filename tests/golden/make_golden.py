"""Generates tests/golden/*.npz from the reference's own code.

The reference ships no tests, fixtures or known-answer vectors, so the golden
vectors here are outputs of the reference itself: its headers and CPU plugin
compiled unmodified in oracle/_ref (see oracle/ref_harness.cpp).  Each fixture
holds the inputs, the reference tree (every node field and the permuted
points) and the reference's per-query results:

* deterministic Barnes-Hut (include/barnes_hut.h:23-78): values, contribution
  counts and accepted-set hashes for every kernel at two opening thresholds;
* stochastic Barnes-Hut (include/tree_sampler.h:21-113) with std::mt19937
  seeded per query: values and contribution counts.

Run from the repository root after `make -C oracle`:
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "stochastic-barnes-hut_b200"))

import oracle as O  # noqa: E402
import sbh_workloads as W  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# name, dim, dim_split_log, leaf_size, generator, n points, alpha
CASES = [
    ("oct1_gauss", 3, 1, 1, "gauss", 1500, 1.0),
    ("oct2_torus", 3, 2, 1, "torus", 1500, 1.0),
    ("oct3_gauss", 3, 3, 1, "gauss", 1200, 1.0),
    ("oct1_leaf8_gauss", 3, 1, 8, "gauss", 2000, 1.0),
    ("quad1_circle", 2, 1, 1, "circle", 1500, 50.0),
    ("quad2_gauss", 2, 2, 1, "gauss", 1500, 1.0),
    ("quad3_circle", 2, 3, 1, "circle", 1200, 50.0),
    ("oct2_leaf8_torus", 3, 2, 8, "torus", 2000, 100.0),
]
NQ = 96
BETAS = (2.0, 1.25)
KERNELS = (O.GRAVITY, O.WINDING_NUMBER, O.SMOOTH_DIST, O.PLUMMER)


def inputs(gen, dim, n, seed):
    if gen == "gauss":
        return W.gaussian_mixture(n, seed, dim=dim)
    if gen == "torus":
        return W.torus_surface(n, seed, jitter=1e-3)
    return W.circle_points(n, seed, jitter=1e-3)


def first_child_and_mask(child):
    nn, bf = child.shape
    mw = max(1, bf // 64)
    first = np.zeros(nn, np.int64)
    mask = np.zeros((nn, mw), np.uint64)
    for v in range(nn):
        bits = np.nonzero(child[v] >= 0)[0]
        if len(bits):
            first[v] = child[v, bits[0]]
            for b in bits:
                mask[v, b >> 6] |= np.uint64(1) << np.uint64(b & 63)
    return first, mask


def main():
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libsbh_ref.so is not built (needs the reference checkout)")
    for i, (name, dim, dsl, leaf, gen, n, alpha) in enumerate(CASES):
        pts, nrm, mass = inputs(gen, dim, n, seed=1000 + i)
        lo, hi = W.padded_box(pts)
        t = O.RefTree(pts, nrm, mass, lo, hi, alpha=alpha, dim_split_log=dsl, leaf_size=leaf)
        d = t.dump()
        first, mask = first_child_and_mask(d.child)
        q = W.uniform_queries(NQ, seed=2000 + i, dim=dim, lo=-1.2, hi=1.2)
        rec = dict(dim=dim, dim_split_log=dsl, leaf_size=leaf, alpha=np.float32(alpha),
                   points=pts, normals=nrm, masses=mass, min_corner=lo, max_corner=hi, queries=q,
                   start=d.start, end=d.end, parent=d.parent, depth=d.depth,
                   num_children=d.num_children, is_leaf=d.is_leaf, first_child=first, mask=mask,
                   bmin=d.bmin, bmax=d.bmax, diameter=d.diameter, agg=d.agg, perm_points=d.pos,
                   perm_normals=d.nrm, perm_masses=d.mass)
        for k in KERNELS:
            for b in BETAS:
                v, c, h = t.bh(k, q, b, eps=1e-3)
                rec[f"bh_k{k}_b{b}"] = v
                rec[f"bh_counts_k{k}_b{b}"] = c
                rec[f"bh_hash_k{k}_b{b}"] = h
        seeds = np.arange(NQ, dtype=np.uint32) * 7919 + 17
        rec["sbh_seeds"] = seeds
        for k in KERNELS:
            v, c = t.sbh(k, q, 2, seeds, eps=1e-3)
            rec[f"sbh_k{k}"] = v
            rec[f"sbh_counts_k{k}"] = c
        path = os.path.join(OUT, f"{name}.npz")
        np.savez_compressed(path, **rec)
        print(f"{path}: {t.num_nodes} nodes, {os.path.getsize(path) // 1024} KiB")


if __name__ == "__main__":
    main()
