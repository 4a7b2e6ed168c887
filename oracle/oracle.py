"""ctypes bindings for the oracle: TEST INFRASTRUCTURE ONLY.

Two libraries, both built by ``oracle/Makefile``:

* ``libsbh_oracle.so`` -- this project's C restatement of the reference path
  (``oracle/sbh_oracle.c``); always available once built.
* ``_ref/libsbh_ref.so`` -- the reference's own headers and CPU plugin
  (``src/sbh.cpp``) compiled unmodified against the shims in this folder; built
  where the reference checkout exists and carried to other machines prebuilt.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this module.  The product never does.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libsbh_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libsbh_ref.so")

GRAVITY, WINDING_NUMBER, SMOOTH_DIST, PLUMMER = 0, 1, 2, 3
RNG_MT19937, RNG_PHILOX = 0, 1

_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_F = ctypes.c_float


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_P)


def _f32(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if shape is not None:
        a = a.reshape(shape)
    return a


_lib_cache: dict[str, ctypes.CDLL] = {}


def _load(path: str, kind: str) -> ctypes.CDLL:
    if path in _lib_cache:
        return _lib_cache[path]
    if not os.path.exists(path):
        raise FileNotFoundError(f"{kind} library not built: {path} (run `make -C oracle`)")
    lib = ctypes.CDLL(path)
    _lib_cache[path] = lib
    return lib


def oracle_lib() -> ctypes.CDLL:
    lib = _load(ORACLE_SO, "oracle")
    if not getattr(lib, "_typed", False):
        lib.orc_tree_build.restype = _P
        lib.orc_tree_build.argtypes = [ctypes.c_int] * 4 + [_P, _P, _P, _I64, _P, _P, _F]
        lib.orc_tree_free.argtypes = [_P]
        lib.orc_tree_num_nodes.restype = _I64
        lib.orc_tree_num_nodes.argtypes = [_P]
        lib.orc_tree_branch.argtypes = [_P]
        lib.orc_tree_dump_nodes.argtypes = [_P] * 12
        lib.orc_tree_dump_points.argtypes = [_P] * 5
        lib.orc_bh.argtypes = [_P, ctypes.c_int, _P, _I64, _F, _F, _P, _P, _P]
        lib.orc_bh_vote.argtypes = [_P, ctypes.c_int, _P, _I64, _F, _F, ctypes.c_int, _P, _P]
        lib.orc_sbh.argtypes = [_P, ctypes.c_int, _P, _I64, ctypes.c_int, ctypes.c_int,
                                ctypes.c_uint64, _P, _F, _P, _P, _P]
        lib.orc_brute_force_f64.argtypes = [_P, _P, _P, _I64, ctypes.c_int, ctypes.c_int, _F, _F,
                                            _P, _I64, _P]
        lib.orc_brute_force_abs_f64.argtypes = lib.orc_brute_force_f64.argtypes
        lib.orc_bh_grad.argtypes = [_P, ctypes.c_int, _P, _I64, _F, _F, _F, _P, _P, _P]
        lib.orc_sbh_grad.argtypes = [_P, ctypes.c_int, _P, _I64, ctypes.c_int, ctypes.c_uint64,
                                     _F, _F, _P, _P, _P]
        lib.orc_bh_indexed.argtypes = lib.orc_bh.argtypes
        lib.orc_sbh_deepest.argtypes = [_P, ctypes.c_int, _P, _I64, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_uint64, _P, _F, _P]
        lib.orc_sbh_grad_rng.argtypes = [_P, ctypes.c_int, _P, _I64, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_uint64, _P, _F, _F, _P, _P, _P]
        lib.orc_brute_force_grad_f64.argtypes = [_P, _P, _I64, ctypes.c_int, ctypes.c_int, _F, _F,
                                                 _P, _I64, _P, _P]
        lib.orc_philox4x32_10.argtypes = [_P, _P, _P]
        lib.orc_mt19937_stream.argtypes = [ctypes.c_uint32, _I64, _P, _P]
        lib._typed = True
    return lib


_gpu_lib = None


def gpu_lib() -> ctypes.CDLL:
    """libsbh_bf64.so: the FP64 GPU brute force."""
    global _gpu_lib
    if _gpu_lib is None:
        path = os.path.join(HERE, "libsbh_bf64.so")
        if not os.path.exists(path):
            raise ImportError(f"{path} is not built; run `make -C {HERE}`")
        lib = ctypes.CDLL(path)
        lib.orc_gpu_brute_force_f64.restype = ctypes.c_int
        lib.orc_gpu_brute_force_f64.argtypes = [_P, _P, _P, _I64, ctypes.c_int, ctypes.c_int, _F,
                                                _F, _P, _I64, ctypes.c_int, _P]
        _gpu_lib = lib
    return _gpu_lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib() -> ctypes.CDLL:
    lib = _load(REF_SO, "reference")
    if not getattr(lib, "_typed", False):
        lib.ref_tree_create.restype = _P
        lib.ref_tree_create.argtypes = [ctypes.c_int] * 3 + [_P, _P, _P, _I64, _P, _P, _F]
        lib.ref_tree_destroy.argtypes = [_P]
        lib.ref_tree_num_nodes.restype = _I64
        lib.ref_tree_num_nodes.argtypes = [_P]
        lib.ref_tree_num_points.restype = _I64
        lib.ref_tree_num_points.argtypes = [_P]
        lib.ref_tree_branch.argtypes = [_P]
        lib.ref_tree_root_children.argtypes = [_P]
        lib.ref_tree_dump_nodes.argtypes = [_P] * 12
        lib.ref_tree_dump_points.argtypes = [_P] * 5
        lib.ref_bh.argtypes = [_P, ctypes.c_int, _P, _I64, _F, _F, _P, _P, _P]
        lib.ref_sbh.argtypes = [_P, ctypes.c_int, _P, _I64, ctypes.c_int, _P, _F, _P, _P]
        lib.ref_plugin_bh.restype = ctypes.c_double
        lib.ref_plugin_bh.argtypes = [_P, ctypes.c_int, _P, _I64, _F, _P]
        lib.ref_plugin_sbh.restype = ctypes.c_double
        lib.ref_plugin_sbh.argtypes = [_P, ctypes.c_int, _P, _I64, ctypes.c_int, _P, _P]
        lib.ref_hardware_concurrency.restype = ctypes.c_int
        lib.ref_mt19937_stream.argtypes = [ctypes.c_uint32, _I64, _P, _P]
        lib._typed = True
    return lib


@dataclass
class TreeDump:
    start: np.ndarray
    end: np.ndarray
    parent: np.ndarray
    depth: np.ndarray
    num_children: np.ndarray
    is_leaf: np.ndarray
    child: np.ndarray
    bmin: np.ndarray
    bmax: np.ndarray
    diameter: np.ndarray
    agg: np.ndarray
    pos: np.ndarray
    nrm: np.ndarray
    mass: np.ndarray
    alpha: np.ndarray


class _TreeBase:
    dim: int
    _h: int

    def _dump(self, lib, prefix, nn, bf, npts) -> TreeDump:
        d = self.dim
        start = np.zeros(nn, np.int64)
        end = np.zeros(nn, np.int64)
        parent = np.zeros(nn, np.int64)
        depth = np.zeros(nn, np.int32)
        nch = np.zeros(nn, np.int32)
        leaf = np.zeros(nn, np.uint8)
        child = np.zeros((nn, bf), np.int64)
        bmin = np.zeros((nn, d), np.float32)
        bmax = np.zeros((nn, d), np.float32)
        diam = np.zeros(nn, np.float32)
        agg = np.zeros((nn, 2 * d + 2), np.float32)
        getattr(lib, prefix + "_dump_nodes")(
            self._h, *[_ptr(a) for a in (start, end, parent, depth, nch, leaf, child, bmin, bmax,
                                         diam, agg)])
        pos = np.zeros((npts, d), np.float32)
        nrm = np.zeros((npts, d), np.float32)
        mass = np.zeros(npts, np.float32)
        alpha = np.zeros(npts, np.float32)
        getattr(lib, prefix + "_dump_points")(self._h, _ptr(pos), _ptr(nrm), _ptr(mass),
                                              _ptr(alpha))
        return TreeDump(start, end, parent, depth, nch, leaf.astype(bool), child, bmin, bmax, diam,
                        agg, pos, nrm, mass, alpha)


class OracleTree(_TreeBase):
    """C restatement of Tree2D/Tree3D (include/tree3d.h:330-412)."""

    def __init__(self, points, normals, masses, min_corner, max_corner, alpha=1.0,
                 dim_split_log=1, leaf_size=1, max_depth=100):
        self.lib = oracle_lib()
        pts = _f32(points)
        self.dim = pts.shape[1]
        n = pts.shape[0]
        nrm = _f32(normals, (n, self.dim))
        m = _f32(masses, (n,))
        lo = _f32(min_corner, (self.dim,))
        hi = _f32(max_corner, (self.dim,))
        self.n = n
        self._h = self.lib.orc_tree_build(self.dim, dim_split_log, leaf_size, max_depth,
                                          _ptr(pts), _ptr(nrm), _ptr(m), n, _ptr(lo), _ptr(hi),
                                          float(np.float32(alpha)))
        if not self._h:
            raise ValueError("oracle tree build rejected its arguments")
        self.num_nodes = self.lib.orc_tree_num_nodes(self._h)
        self.branch = self.lib.orc_tree_branch(self._h)

    def __del__(self):
        if getattr(self, "_h", None):
            self.lib.orc_tree_free(self._h)
            self._h = None

    def dump(self) -> TreeDump:
        return self._dump(self.lib, "orc_tree", self.num_nodes, self.branch, self.n)

    def bh(self, kernel, queries, beta, eps=1e-3):
        q = _f32(queries, (-1, self.dim))
        nq = q.shape[0]
        out = np.zeros(nq, np.float32)
        cnt = np.zeros(nq, np.int32)
        hs = np.zeros(nq, np.uint64)
        self.lib.orc_bh(self._h, kernel, _ptr(q), nq, float(np.float32(beta)), eps, _ptr(out),
                        _ptr(cnt), _ptr(hs))
        return out, cnt, hs

    def bh_indexed(self, kernel, queries, beta, eps=1e-3):
        """bh() with sibling steps by index instead of nextChild's midpoint
        quantization (see orc_bh_indexed)."""
        q = _f32(queries, (-1, self.dim))
        nq = q.shape[0]
        out = np.zeros(nq, np.float32)
        cnt = np.zeros(nq, np.int32)
        hs = np.zeros(nq, np.uint64)
        self.lib.orc_bh_indexed(self._h, kernel, _ptr(q), nq, float(np.float32(beta)), eps,
                                _ptr(out), _ptr(cnt), _ptr(hs))
        return out, cnt, hs

    def bh_vote(self, kernel, queries, beta, eps=1e-3, group=32):
        q = _f32(queries, (-1, self.dim))
        nq = q.shape[0]
        out = np.zeros(nq, np.float32)
        cnt = np.zeros(nq, np.int32)
        self.lib.orc_bh_vote(self._h, kernel, _ptr(q), nq, float(np.float32(beta)), eps, group,
                             _ptr(out), _ptr(cnt))
        return out, cnt

    def sbh(self, kernel, queries, samples, rng=RNG_PHILOX, seed=0, mt_seeds=None, eps=1e-3,
            return_scale=False):
        """(values, counts[, scales]): scales are the per-query magnitudes of all
        summed terms (see orc_sbh), for tolerances between summation orders."""
        q = _f32(queries, (-1, self.dim))
        nq = q.shape[0]
        out = np.zeros(nq, np.float32)
        cnt = np.zeros(nq, np.int32)
        sc = np.zeros(nq, np.float64) if return_scale else None
        ms = None if mt_seeds is None else np.ascontiguousarray(mt_seeds, np.uint32)
        self.lib.orc_sbh(self._h, kernel, _ptr(q), nq, samples, rng, seed, _ptr(ms), eps,
                         _ptr(out), _ptr(cnt), _ptr(sc))
        return (out, cnt, sc) if return_scale else (out, cnt)


    def sbh_deepest(self, kernel, queries, samples, rng=RNG_PHILOX, seed=0, mt_seeds=None,
                    eps=1e-3):
        """Per query, the depth of the deepest node the sampler's paths reach
        (the paths of sbh() with the same stream)."""
        q = _f32(queries, (-1, self.dim))
        nq = q.shape[0]
        deep = np.zeros(nq, np.int32)
        ms = None if mt_seeds is None else np.ascontiguousarray(mt_seeds, np.uint32)
        self.lib.orc_sbh_deepest(self._h, kernel, _ptr(q), nq, samples, rng, seed, _ptr(ms), eps,
                                 _ptr(deep))
        return deep

    def bh_grad(self, kernel, queries, beta, alpha=1.0, eps=1e-3):
        """Barnes-Hut value and gradient in FP64 over the reference's node set:
        (val[nq], grad[nq, dim], counts)."""
        q = _f32(queries, (-1, self.dim))
        nq = q.shape[0]
        val = np.zeros(nq, np.float64)
        grad = np.zeros((nq, self.dim), np.float64)
        cnt = np.zeros(nq, np.int32)
        self.lib.orc_bh_grad(self._h, kernel, _ptr(q), nq, float(np.float32(beta)), eps,
                             float(np.float32(alpha)), _ptr(val), _ptr(grad), _ptr(cnt))
        return val, grad, cnt

    def sbh_grad(self, kernel, queries, samples, seed=0, alpha=1.0, eps=1e-3, rng=RNG_PHILOX,
                 mt_seeds=None):
        """Stochastic estimator value and gradient on the paths of sbh() with the
        same random stream (Philox keyed by seed, or the reference's mt19937
        seeded per query from mt_seeds): (val[nq], grad[nq, dim], counts)."""
        q = _f32(queries, (-1, self.dim))
        nq = q.shape[0]
        val = np.zeros(nq, np.float64)
        grad = np.zeros((nq, self.dim), np.float64)
        cnt = np.zeros(nq, np.int32)
        ms = None if mt_seeds is None else np.ascontiguousarray(mt_seeds, np.uint32)
        self.lib.orc_sbh_grad_rng(self._h, kernel, _ptr(q), nq, samples, rng, seed, _ptr(ms), eps,
                                  float(np.float32(alpha)), _ptr(val), _ptr(grad), _ptr(cnt))
        return val, grad, cnt


class RefTree(_TreeBase):
    """The reference's own PyQuadtree/PyOctree (include/py_tree.h) built in oracle/_ref."""

    def __init__(self, points, normals, masses, min_corner, max_corner, alpha=1.0,
                 dim_split_log=1, leaf_size=1):
        self.lib = ref_lib()
        pts = _f32(points)
        self.dim = pts.shape[1]
        n = pts.shape[0]
        nrm = _f32(normals, (n, self.dim))
        m = _f32(masses, (n,))
        lo = _f32(min_corner, (self.dim,))
        hi = _f32(max_corner, (self.dim,))
        self.n = n
        self._h = self.lib.ref_tree_create(self.dim, dim_split_log, leaf_size, _ptr(pts),
                                           _ptr(nrm), _ptr(m), n, _ptr(lo), _ptr(hi),
                                           float(np.float32(alpha)))
        if not self._h:
            raise ValueError("unsupported reference tree type")
        self.num_nodes = self.lib.ref_tree_num_nodes(self._h)
        self.branch = self.lib.ref_tree_branch(self._h)
        self.root_children = self.lib.ref_tree_root_children(self._h)

    def __del__(self):
        if getattr(self, "_h", None):
            self.lib.ref_tree_destroy(self._h)
            self._h = None

    def dump(self) -> TreeDump:
        return self._dump(self.lib, "ref_tree", self.num_nodes, self.branch, self.n)

    def bh(self, kernel, queries, beta, eps=1e-3):
        q = _f32(queries, (-1, self.dim))
        nq = q.shape[0]
        out = np.zeros(nq, np.float32)
        cnt = np.zeros(nq, np.int32)
        hs = np.zeros(nq, np.uint64)
        self.lib.ref_bh(self._h, kernel, _ptr(q), nq, float(np.float32(beta)), eps, _ptr(out),
                        _ptr(cnt), _ptr(hs))
        return out, cnt, hs

    def sbh(self, kernel, queries, samples, mt_seeds, eps=1e-3):
        q = _f32(queries, (-1, self.dim))
        nq = q.shape[0]
        out = np.zeros(nq, np.float32)
        cnt = np.zeros(nq, np.int32)
        ms = np.ascontiguousarray(mt_seeds, np.uint32)
        self.lib.ref_sbh(self._h, kernel, _ptr(q), nq, samples, _ptr(ms), eps, _ptr(out),
                         _ptr(cnt))
        return out, cnt

    def plugin_bh(self, kernel, queries, beta):
        """src/sbh.cpp evalBarnesHut (its own std::thread pool); returns (values, seconds)."""
        q = _f32(queries, (-1, self.dim))
        out = np.zeros(q.shape[0], np.float32)
        secs = self.lib.ref_plugin_bh(self._h, kernel, _ptr(q), q.shape[0],
                                      float(np.float32(beta)), _ptr(out))
        return out, secs

    def plugin_sbh(self, kernel, queries, samples):
        """src/sbh.cpp multiLevelPrefixControlVariateSampler; returns (values, counts, seconds)."""
        q = _f32(queries, (-1, self.dim))
        out = np.zeros(q.shape[0], np.float32)
        cnt = np.zeros(q.shape[0], np.int32)
        secs = self.lib.ref_plugin_sbh(self._h, kernel, _ptr(q), q.shape[0], samples, _ptr(out),
                                       _ptr(cnt))
        return out, cnt, secs


def ref_hardware_concurrency() -> int:
    return ref_lib().ref_hardware_concurrency()


def brute_force_f64(points, normals, masses, kernel, queries, alpha=1.0, eps=1e-3, abs_sum=False):
    lib = oracle_lib()
    pts = _f32(points)
    dim = pts.shape[1]
    n = pts.shape[0]
    nrm = _f32(normals, (n, dim))
    m = _f32(masses, (n,))
    q = _f32(queries, (-1, dim))
    out = np.zeros(q.shape[0], np.float64)
    fn = lib.orc_brute_force_abs_f64 if abs_sum else lib.orc_brute_force_f64
    fn(_ptr(pts), _ptr(nrm), _ptr(m), n, dim, kernel, float(np.float32(alpha)),
       float(np.float32(eps)), _ptr(q), q.shape[0], _ptr(out))
    return out


def gpu_brute_force_f64(points, normals, masses, kernel, queries, alpha=1.0, eps=1e-3,
                        abs_sum=False):
    """brute_force_f64 on the GPU (libsbh_bf64.so): every term in FP64 from the
    float inputs, summed over every source, for checks at benchmark scale."""
    lib = gpu_lib()
    pts = _f32(points)
    dim = pts.shape[1]
    n = pts.shape[0]
    nrm = _f32(normals, (n, dim))
    m = _f32(masses, (n,))
    q = _f32(queries, (-1, dim))
    out = np.zeros(q.shape[0], np.float64)
    rc = lib.orc_gpu_brute_force_f64(_ptr(pts), _ptr(nrm), _ptr(m), n, dim, kernel,
                                     float(np.float32(alpha)), float(np.float32(eps)), _ptr(q),
                                     q.shape[0], int(abs_sum), _ptr(out))
    if rc != 0:
        raise RuntimeError(f"orc_gpu_brute_force_f64 failed with CUDA error {rc}")
    return out


def brute_force_grad_f64(points, masses, kernel, queries, alpha=1.0, eps=1e-3):
    """FP64 value and query gradient over every source: (val[nq], grad[nq, dim]).
    Smooth distance: D = -log(sum exp(-alpha r)) / alpha and dD/dq."""
    lib = oracle_lib()
    pts = _f32(points)
    dim = pts.shape[1]
    n = pts.shape[0]
    m = _f32(masses, (n,))
    q = _f32(queries, (-1, dim))
    val = np.zeros(q.shape[0], np.float64)
    grad = np.zeros((q.shape[0], dim), np.float64)
    lib.orc_brute_force_grad_f64(_ptr(pts), _ptr(m), n, dim, kernel, float(np.float32(alpha)),
                                 float(np.float32(eps)), _ptr(q), q.shape[0], _ptr(val),
                                 _ptr(grad))
    return val, grad


def philox4x32_10(ctr, key):
    lib = oracle_lib()
    c = np.ascontiguousarray(ctr, np.uint32)
    k = np.ascontiguousarray(key, np.uint32)
    out = np.zeros(4, np.uint32)
    lib.orc_philox4x32_10(_ptr(c), _ptr(k), _ptr(out))
    return out


def mt19937_stream(seed, n, ref=False):
    lib = ref_lib() if ref else oracle_lib()
    raw = np.zeros(n, np.uint32)
    uni = np.zeros(n, np.float32)
    (lib.ref_mt19937_stream if ref else lib.orc_mt19937_stream)(seed, n, _ptr(raw), _ptr(uni))
    return raw, uni
