"""The oracle (oracle/sbh_oracle.c) pinned against the reference.

* against the committed golden vectors the reference produced
  (tests/golden/make_golden.py), bit for bit, everywhere;
* against the reference's own code compiled in oracle/_ref, on fresh random
  inputs, where that build exists;
* the RNG restatements against published known-answer vectors (Philox4x32-10)
  and against libstdc++ itself (std::mt19937 + uniform_real_distribution).
"""
import numpy as np
import pytest

import oracle as O
from conftest import golden_cases, load_golden
from helpers import bits_equal

KERNELS = (O.GRAVITY, O.WINDING_NUMBER, O.SMOOTH_DIST, O.PLUMMER)


def _oracle_tree(g):
    return O.OracleTree(g["points"], g["normals"], g["masses"], g["min_corner"], g["max_corner"],
                        alpha=float(g["alpha"]), dim_split_log=int(g["dim_split_log"]),
                        leaf_size=int(g["leaf_size"]))


@pytest.mark.parametrize("case", golden_cases())
def test_oracle_tree_matches_golden(case):
    g = load_golden(case)
    t = _oracle_tree(g)
    d = t.dump()
    assert t.num_nodes == len(g["start"])
    for f in ("start", "end", "parent", "depth", "num_children", "bmin", "bmax", "diameter", "agg"):
        assert bits_equal(getattr(d, f), g[f]), f
    assert np.array_equal(d.is_leaf, g["is_leaf"].astype(bool))
    assert bits_equal(d.pos, g["perm_points"]) and bits_equal(d.nrm, g["perm_normals"])
    assert bits_equal(d.mass, g["perm_masses"])


@pytest.mark.parametrize("case", golden_cases())
def test_oracle_barnes_hut_matches_golden(case):
    g = load_golden(case)
    t = _oracle_tree(g)
    for k in KERNELS:
        for b in (2.0, 1.25):
            v, c, h = t.bh(k, g["queries"], b)
            assert bits_equal(v, g[f"bh_k{k}_b{b}"]), (k, b)
            assert np.array_equal(c, g[f"bh_counts_k{k}_b{b}"]), (k, b)
            assert np.array_equal(h, g[f"bh_hash_k{k}_b{b}"]), (k, b)


@pytest.mark.parametrize("case", golden_cases())
def test_oracle_sampler_matches_golden(case):
    g = load_golden(case)
    t = _oracle_tree(g)
    for k in KERNELS:
        v, c = t.sbh(k, g["queries"], 2, rng=O.RNG_MT19937, mt_seeds=g["sbh_seeds"])
        assert bits_equal(v, g[f"sbh_k{k}"]), k
        assert np.array_equal(c, g[f"sbh_counts_k{k}"]), k


def test_philox_known_answers():
    # Known-answer vectors published with the Random123 library for philox4x32-10.
    assert list(O.philox4x32_10([0, 0, 0, 0], [0, 0])) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C,
                                                          0x9B00DBD8]
    assert list(O.philox4x32_10([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2)) == [
        0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert list(O.philox4x32_10([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344],
                                [0xA4093822, 0x299F31D0])) == [0xD16CFE09, 0x94FDCCEB,
                                                               0x5001E420, 0x24126EA1]


def test_mt19937_known_answer():
    # The C++ standard fixes the 10000th output of a default-seeded mt19937.
    raw, _ = O.mt19937_stream(5489, 10000)
    assert raw[-1] == 4123659995


needs_ref = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built here")


@needs_ref
def test_mt19937_matches_libstdcxx():
    for seed in (0, 1, 12345, 2**32 - 1):
        a = O.mt19937_stream(seed, 3000)
        b = O.mt19937_stream(seed, 3000, ref=True)
        assert np.array_equal(a[0], b[0]) and bits_equal(a[1], b[1])


@needs_ref
@pytest.mark.parametrize("dim,dsl,leaf", [(3, 1, 1), (3, 2, 1), (3, 3, 8), (2, 1, 8), (2, 2, 1),
                                          (2, 3, 1)])
def test_oracle_matches_live_reference(dim, dsl, leaf):
    import sbh_workloads as W
    pts, nrm, m = W.gaussian_mixture(2500, seed=dim * 100 + dsl * 10 + leaf, dim=dim)
    lo, hi = W.padded_box(pts)
    r = O.RefTree(pts, nrm, m, lo, hi, alpha=30.0, dim_split_log=dsl, leaf_size=leaf)
    c = O.OracleTree(pts, nrm, m, lo, hi, alpha=30.0, dim_split_log=dsl, leaf_size=leaf)
    a, b = r.dump(), c.dump()
    for f in a.__dataclass_fields__:
        assert bits_equal(getattr(a, f), getattr(b, f)), f
    q = W.uniform_queries(200, seed=7, dim=dim, lo=-1.3, hi=1.3)
    for k in KERNELS:
        for beta in (2.0, 1 / 0.3, 1.25, np.inf):
            rv, rc, rh = r.bh(k, q, beta)
            cv, cc, ch = c.bh(k, q, beta)
            assert bits_equal(rv, cv) and np.array_equal(rc, cc) and np.array_equal(rh, ch)
    seeds = np.arange(200, dtype=np.uint32) * 31 + 5
    for k in KERNELS:
        rv, rc = r.sbh(k, q, 3, seeds)
        cv, cc = c.sbh(k, q, 3, rng=O.RNG_MT19937, mt_seeds=seeds)
        assert bits_equal(rv, cv) and np.array_equal(rc, cc)


@needs_ref
def test_oracle_duplicate_points_chain():
    # Nine identical points force a single-child chain down to the depth cap (100).
    p = np.array([[0.3, 0.2, 0.1]] * 9 + [[0.5, -0.5, 0.5], [-0.3, 0.1, 0.9]], np.float32)
    nr = np.ones_like(p)
    m = np.ones(len(p), np.float32)
    lo, hi = -np.ones(3, np.float32), np.ones(3, np.float32)
    q = np.array([[0, 0, 0], [0.3, 0.2, 0.1], [2, 2, 2]], np.float32)
    for dsl in (1, 2, 3):
        r = O.RefTree(p, nr, m, lo, hi, dim_split_log=dsl)
        c = O.OracleTree(p, nr, m, lo, hi, dim_split_log=dsl)
        assert r.num_nodes == c.num_nodes == 103
        rv, rc, _ = r.bh(0, q, 2.0)
        cv, cc, _ = c.bh(0, q, 2.0)
        assert bits_equal(rv, cv) and np.array_equal(rc, cc)


def test_brute_force_f64_analytic():
    # One source: the FP64 brute force is the kernel formula itself.
    p = np.array([[0.25, 0.5, 0.25]], np.float32)
    n = np.array([[0.0, 0.0, 1.0]], np.float32)
    m = np.array([2.0], np.float32)
    q = np.array([[0.25, 0.5, 1.25]], np.float32)
    r = 1.0
    assert O.brute_force_f64(p, n, m, O.PLUMMER, q, eps=1e-3)[0] == pytest.approx(
        2.0 / np.sqrt(r + float(np.float32(1e-3)) ** 2), rel=1e-12)
    assert O.brute_force_f64(p, n, m, O.GRAVITY, q)[0] == pytest.approx(
        -2.0 / (1.0 + float(np.float32(0.1))), rel=1e-7)
    assert O.brute_force_f64(p, n, m, O.SMOOTH_DIST, q, alpha=3.0)[0] == pytest.approx(np.exp(-3.0),
                                                                                   rel=1e-7)


def test_gpu_fp64_brute_force_library_loads():
    """The FP64 GPU brute force (the benchmark's accuracy reference) is built
    and exports its entry point; running it needs a GPU."""
    lib = O.gpu_lib()
    assert hasattr(lib, "orc_gpu_brute_force_f64")


def test_indexed_barnes_hut_walk_equals_the_stackless_walk(golden):
    """orc_bh_indexed (sibling steps by index) is the reference's stackless walk
    (nextChild by midpoint quantization) bit for bit -- values, counts and
    accepted-node hashes -- on every golden tree, where the quantization is
    exact."""
    for name, g in golden.items():
        ot = O.OracleTree(g["points"], g["normals"], g["masses"], g["min_corner"],
                          g["max_corner"], alpha=float(g["alpha"]),
                          dim_split_log=int(g["dim_split_log"]), leaf_size=int(g["leaf_size"]))
        for kernel in (O.GRAVITY, O.WINDING_NUMBER, O.PLUMMER):
            for beta in (2.0, 1.25):
                a, ac, ah = ot.bh(kernel, g["queries"], beta)
                b, bc, bh = ot.bh_indexed(kernel, g["queries"], beta)
                assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), name
                assert np.array_equal(ac, bc) and np.array_equal(ah, bh), name
