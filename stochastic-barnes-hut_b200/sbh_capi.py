"""ctypes binding of the C ABI in include/sbh_b200.h (libsbh_b200.so).

This is the language-neutral boundary of the library: host trees, device
trees and the evaluation calls, with plain pointers and sizes.  The pybind11
modules `sbh` / `sbh_gpu` cover the reference's Python surface; this module is
for callers that hold raw buffers (device pointers from PyTorch, CuPy, another
runtime) and is what the parity tests call.

Importing this module loads the library and raises if it is missing: there is
no fallback implementation.
"""
from __future__ import annotations

import ctypes
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsbh_b200.so")

OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_CUDA = 2
ERR_OUT_OF_MEMORY = 3
ERR_NO_DEVICE = 4
ERR_DEVICE_LIMIT = 5
ERR_UNSUPPORTED = 6

GRAVITY, WINDING_NUMBER, SMOOTH_DIST, PLUMMER = 0, 1, 2, 3
BRUTE_FORCE, BARNES_HUT, BARNES_HUT_VOTE, STOCHASTIC = 0, 1, 2, 3
FLAG_KEEP_ORDER = 0x1
FLAG_STAGE_LEAVES = 0x2

# Every function the header declares, with its ctypes signature.
_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_SIGNATURES = {
    "sbh_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "sbh_last_error": (ctypes.c_char_p, []),
    "sbh_abi_version": (ctypes.c_int, []),
    "sbh_params_init": (None, [_P]),
    "sbh_host_tree_create": (ctypes.c_int, [ctypes.c_int] * 4 + [_P, _P, _P, _I64, _P, _P,
                                                                 ctypes.c_float, _P]),
    "sbh_host_tree_destroy": (None, [_P]),
    "sbh_host_tree_info": (ctypes.c_int, [_P, _P]),
    "sbh_host_tree_export_nodes": (ctypes.c_int, [_P] * 13),
    "sbh_host_tree_export_points": (ctypes.c_int, [_P] * 4),
    "sbh_gpu_tree_create": (ctypes.c_int, [_P, ctypes.c_int, _P]),
    "sbh_gpu_tree_destroy": (None, [_P]),
    "sbh_gpu_tree_info": (ctypes.c_int, [_P, _P]),
    "sbh_eval": (ctypes.c_int, [_P, _P, _P, _I64, _P, _P, _P, _P]),
    "sbh_eval_device": (ctypes.c_int, [_P, _P, _P, _I64, _P, _P, _P]),
    "sbh_gpu_tree_check": (ctypes.c_int, [_P, _P]),
    "sbh_eval_device_static_scratch": (ctypes.c_int, [_P, _P, _P, _I64, _P, _P, _P]),
    "sbh_eval_batch": (ctypes.c_int, [_P, ctypes.c_int, _P]),
    "sbh_server_config_init": (None, [_P]),
    "sbh_server_create": (ctypes.c_int, [_P, _P]),
    "sbh_server_add_tree": (ctypes.c_int, [_P, _P, _P]),
    "sbh_server_submit": (ctypes.c_int, [_P, ctypes.c_int32, _P, _P, _I64, _P, _P, _P]),
    "sbh_server_wait": (ctypes.c_int, [_P, ctypes.c_uint64, ctypes.c_double, _P]),
    "sbh_server_stats_get": (ctypes.c_int, [_P, _P]),
    "sbh_server_destroy": (None, [_P]),
    "sbh_eval_grad": (ctypes.c_int, [_P, _P, _P, _I64, _P, _P, _P, _P, _P]),
    "sbh_eval_grad_device": (ctypes.c_int, [_P, _P, _P, _I64, _P, _P, _P, _P]),
    "sbh_measure_pipe_rates": (ctypes.c_int, [ctypes.c_int, _P, _P, _P, _P, _P]),
    "sbh_gpu_tree_build": (ctypes.c_int, [ctypes.c_int] * 4 + [_P, _P, _P, _I64, _P, _P,
                                                               ctypes.c_float, ctypes.c_int, _P,
                                                               _P]),
    "sbh_gpu_tree_export": (ctypes.c_int, [_P] * 10),
    "sbh_server_add_gpu_tree": (ctypes.c_int, [_P, _P, _P]),
    "sbh_host_tree_save": (ctypes.c_int, [_P, ctypes.c_char_p]),
    "sbh_host_tree_load": (ctypes.c_int, [ctypes.c_char_p, _P]),
    "sbh_batch_tuning_init": (None, [_P]),
    "sbh_batch_set_tuning": (ctypes.c_int, [ctypes.c_int, _P]),
    "sbh_batch_get_tuning": (ctypes.c_int, [ctypes.c_int, _P]),
    "sbh_batch_autotune": (ctypes.c_int, [_P, ctypes.c_int, _P, ctypes.c_int, _P, _P, _P]),
}

# Largest query count sbh_eval_device_static_scratch accepts per call.
STATIC_SCRATCH_MAX_QUERIES = 262144


class Params(ctypes.Structure):
    _fields_ = [("method", ctypes.c_int32), ("kernel", ctypes.c_int32), ("beta", ctypes.c_float),
                ("samples_per_subdomain", ctypes.c_int32), ("seed", ctypes.c_uint64),
                ("alpha", ctypes.c_float), ("eps", ctypes.c_float), ("flags", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32)]


class TreeInfo(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int32), ("dim_split_log", ctypes.c_int32),
                ("leaf_size", ctypes.c_int32), ("max_depth", ctypes.c_int32),
                ("num_points", ctypes.c_int64), ("num_nodes", ctypes.c_int64),
                ("depth", ctypes.c_int32), ("root_children", ctypes.c_int32),
                ("alpha", ctypes.c_float), ("reserved", ctypes.c_int32),
                ("device_bytes", ctypes.c_uint64)]


class BatchItem(ctypes.Structure):
    _fields_ = [("tree", _P), ("params", Params), ("d_queries", _P), ("nq", ctypes.c_int64),
                ("d_results", _P), ("d_contribs", _P), ("d_self_mass", _P)]


class BatchTuning(ctypes.Structure):
    _fields_ = [("sampler_unit_queries", ctypes.c_int32), ("bucket_queries", ctypes.c_int32),
                ("blocks_per_sm", ctypes.c_int32), ("bh_unit_queries", ctypes.c_int32),
                ("direct_queries", ctypes.c_int32)]

    def as_dict(self) -> dict:
        return {"sampler_unit_queries": self.sampler_unit_queries,
                "bucket_queries": self.bucket_queries, "blocks_per_sm": self.blocks_per_sm,
                "bh_unit_queries": self.bh_unit_queries, "direct_queries": self.direct_queries}


class ServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("slots", ctypes.c_int32),
                ("slot_queries", ctypes.c_int64), ("max_requests_per_batch", ctypes.c_int32),
                ("reserved", ctypes.c_int32), ("tuning", BatchTuning)]


class RequestInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("batches", ctypes.c_int32), ("nq", ctypes.c_int64),
                ("queue_ms", ctypes.c_double), ("latency_ms", ctypes.c_double)]


class ServerStats(ctypes.Structure):
    _fields_ = [("requests", ctypes.c_int64), ("queries", ctypes.c_int64),
                ("batches", ctypes.c_int64), ("busy_ms", ctypes.c_double)]


class SbhError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{message} (status {status})")
        self.status = status


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built; run `make -C {HERE}`")
        l = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            f = getattr(l, name)
            f.restype = res
            f.argtypes = args
        _lib = l
    return _lib


def _check(status: int):
    if status != OK:
        l = lib()
        msg = (l.sbh_last_error() or b"").decode() or l.sbh_status_string(status).decode()
        raise SbhError(status, msg)


def _ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def params(method=BRUTE_FORCE, kernel=GRAVITY, beta=2.0, samples_per_subdomain=1, seed=0,
           alpha=None, eps=1e-3, flags=0) -> Params:
    p = Params()
    lib().sbh_params_init(ctypes.byref(p))
    p.method, p.kernel, p.beta = method, kernel, beta
    p.samples_per_subdomain, p.seed = samples_per_subdomain, seed
    p.alpha = math.nan if alpha is None else alpha
    p.eps, p.flags = eps, flags
    return p


class HostTree:
    """sbh_host_tree_*: the reference tree built on the host."""

    def __init__(self, points, normals, masses, min_corner, max_corner, alpha=1.0,
                 dim_split_log=1, leaf_size=1, max_depth=100):
        pts = np.ascontiguousarray(points, np.float32)
        if pts.ndim != 2:
            raise ValueError("points must be (n, dim)")
        n, dim = pts.shape
        nrm = np.ascontiguousarray(normals, np.float32).reshape(n, dim)
        m = np.ascontiguousarray(masses, np.float32).reshape(n)
        lo = np.ascontiguousarray(min_corner, np.float32).reshape(dim)
        hi = np.ascontiguousarray(max_corner, np.float32).reshape(dim)
        h = ctypes.c_void_p()
        _check(lib().sbh_host_tree_create(dim, dim_split_log, leaf_size, max_depth, _ptr(pts),
                                          _ptr(nrm), _ptr(m), n, _ptr(lo), _ptr(hi),
                                          ctypes.c_float(alpha), ctypes.byref(h)))
        self.handle = h

    def info(self) -> TreeInfo:
        i = TreeInfo()
        _check(lib().sbh_host_tree_info(self.handle, ctypes.byref(i)))
        return i

    def save(self, path: str):
        """sbh_host_tree_save: the whole tree to a file."""
        _check(lib().sbh_host_tree_save(self.handle, os.fsencode(path)))

    @classmethod
    def load(cls, path: str) -> "HostTree":
        """sbh_host_tree_load: a tree saved by save(), verified."""
        h = ctypes.c_void_p()
        _check(lib().sbh_host_tree_load(os.fsencode(path), ctypes.byref(h)))
        t = cls.__new__(cls)
        t.handle = h
        return t

    def export_nodes(self) -> dict:
        i = self.info()
        nn, d = i.num_nodes, i.dim
        mw = max(1, (1 << (d * i.dim_split_log)) >> 6)
        out = dict(start=np.zeros(nn, np.int64), end=np.zeros(nn, np.int64),
                   parent=np.zeros(nn, np.int64), depth=np.zeros(nn, np.int32),
                   num_children=np.zeros(nn, np.int32), is_leaf=np.zeros(nn, np.uint8),
                   first_child=np.zeros(nn, np.int64), mask=np.zeros((nn, mw), np.uint64),
                   bmin=np.zeros((nn, d), np.float32), bmax=np.zeros((nn, d), np.float32),
                   diameter=np.zeros(nn, np.float32), agg=np.zeros((nn, 2 * d + 2), np.float32))
        keys = ["start", "end", "parent", "depth", "num_children", "is_leaf", "first_child",
                "mask", "bmin", "bmax", "diameter", "agg"]
        _check(lib().sbh_host_tree_export_nodes(self.handle, *[_ptr(out[k]) for k in keys]))
        return out

    def export_points(self) -> dict:
        i = self.info()
        out = dict(points=np.zeros((i.num_points, i.dim), np.float32),
                   normals=np.zeros((i.num_points, i.dim), np.float32),
                   masses=np.zeros(i.num_points, np.float32))
        _check(lib().sbh_host_tree_export_points(self.handle, _ptr(out["points"]),
                                                 _ptr(out["normals"]), _ptr(out["masses"])))
        return out

    def close(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.sbh_host_tree_destroy(self.handle)
        self.handle = None

    def __del__(self):
        self.close()


class GpuTree:
    """sbh_gpu_tree_*: a tree resident in device memory."""

    def __init__(self, host: HostTree, device: int = 0):
        h = ctypes.c_void_p()
        _check(lib().sbh_gpu_tree_create(host.handle, device, ctypes.byref(h)))
        self._adopt(h, device)
        self.built_on_device = False

    def _adopt(self, h, device):
        self.handle = h
        i = TreeInfo()
        _check(lib().sbh_gpu_tree_info(h, ctypes.byref(i)))
        self.info = i
        self.dim = i.dim
        self.device = device

    @classmethod
    def build(cls, points, normals, masses, min_corner, max_corner, alpha=1.0, dim_split_log=1,
              leaf_size=1, max_depth=100, device: int = 0) -> "GpuTree":
        """sbh_gpu_tree_build: the same tree as GpuTree(HostTree(...)), built on
        the device (leaf size 1) or on the host (otherwise); `built_on_device`
        tells which."""
        pts = np.ascontiguousarray(points, np.float32)
        n, dim = pts.shape
        nrm = np.ascontiguousarray(normals, np.float32).reshape(n, dim)
        m = np.ascontiguousarray(masses, np.float32).reshape(n)
        lo = np.ascontiguousarray(min_corner, np.float32).reshape(dim)
        hi = np.ascontiguousarray(max_corner, np.float32).reshape(dim)
        h = ctypes.c_void_p()
        on = ctypes.c_int32(0)
        _check(lib().sbh_gpu_tree_build(dim, dim_split_log, leaf_size, max_depth, _ptr(pts),
                                        _ptr(nrm), _ptr(m), n, _ptr(lo), _ptr(hi),
                                        ctypes.c_float(alpha), device, ctypes.byref(h),
                                        ctypes.byref(on)))
        t = cls.__new__(cls)
        t._adopt(h, device)
        t.built_on_device = bool(on.value)
        return t

    def export(self) -> dict:
        """sbh_gpu_tree_export: the device image as numpy arrays."""
        n, nn = self.info.num_points, self.info.num_nodes
        mw = max(1, (1 << (self.dim * self.info.dim_split_log)) >> 6)
        out = dict(pt_pm=np.zeros((n, 4), np.float32), pt_nrm=np.zeros((n, 4), np.float32),
                   nd_cm=np.zeros((nn, 4), np.float32), nd_agg=np.zeros((nn, 4), np.float32),
                   nd_topo=np.zeros((nn, 4), np.int32), nd_bmin=np.zeros((nn, 4), np.float32),
                   nd_bmax=np.zeros((nn, 4), np.float32), nd_mask=np.zeros((nn, mw), np.uint64),
                   pt_code=np.zeros(n, np.uint64))
        keys = ["pt_pm", "pt_nrm", "nd_cm", "nd_agg", "nd_topo", "nd_bmin", "nd_bmax", "nd_mask",
                "pt_code"]
        _check(lib().sbh_gpu_tree_export(self.handle, *[_ptr(out[k]) for k in keys]))
        return out

    def eval(self, queries, p: Params, stream: int = 0, contribs: bool = False):
        """Blocking evaluation of host queries (n, dim): returns (values, kernel_ms[, counts])."""
        q = np.asfortranarray(queries, np.float32)
        if q.ndim != 2 or q.shape[1] != self.dim:
            raise ValueError(f"queries must be (n, {self.dim})")
        nq = q.shape[0]
        out = np.zeros(nq, np.float32)
        cnt = np.zeros(nq, np.int32) if contribs else None
        ms = ctypes.c_float(0)
        _check(lib().sbh_eval(self.handle, ctypes.byref(p), _ptr(q), nq, _ptr(out), _ptr(cnt),
                              ctypes.byref(ms), ctypes.c_void_p(stream)))
        return (out, ms.value, cnt) if contribs else (out, ms.value)

    def eval_host_ptr(self, q_ptr: int, nq: int, out_ptr: int, p: Params, stream: int = 0,
                      contribs_ptr: int = 0) -> float:
        """Blocking evaluation with raw host pointers (SoA [dim][nq] queries)."""
        ms = ctypes.c_float(0)
        _check(lib().sbh_eval(self.handle, ctypes.byref(p), ctypes.c_void_p(q_ptr), nq,
                              ctypes.c_void_p(out_ptr), ctypes.c_void_p(contribs_ptr or None),
                              ctypes.byref(ms), ctypes.c_void_p(stream)))
        return ms.value

    def eval_device(self, d_queries: int, nq: int, d_results: int, p: Params, stream: int = 0,
                    d_contribs: int = 0):
        """Asynchronous evaluation on device pointers (SoA [dim][nq] float32 queries)."""
        _check(lib().sbh_eval_device(self.handle, ctypes.byref(p), ctypes.c_void_p(d_queries), nq,
                                     ctypes.c_void_p(d_results),
                                     ctypes.c_void_p(d_contribs or None), ctypes.c_void_p(stream)))

    def eval_device_static_scratch(self, d_queries: int, nq: int, d_results: int, p: Params,
                                   stream: int = 0, d_contribs: int = 0):
        """As eval_device, without any device allocation: scratch comes from a fixed
        array in the library (at most STATIC_SCRATCH_MAX_QUERIES queries per call;
        calls that overlap on the GPU race on that array)."""
        _check(lib().sbh_eval_device_static_scratch(
            self.handle, ctypes.byref(p), ctypes.c_void_p(d_queries), nq,
            ctypes.c_void_p(d_results), ctypes.c_void_p(d_contribs or None),
            ctypes.c_void_p(stream)))

    def eval_grad(self, queries, p: Params, stream: int = 0, contribs: bool = False,
                  grads: bool = True):
        """Blocking sbh_eval_grad of host queries (n, dim): returns (values, grads
        (n, dim) or None, kernel_ms[, counts])."""
        q = np.asfortranarray(queries, np.float32)
        if q.ndim != 2 or q.shape[1] != self.dim:
            raise ValueError(f"queries must be (n, {self.dim})")
        nq = q.shape[0]
        out = np.zeros(nq, np.float32)
        g = np.zeros((nq, self.dim), np.float32, order="F") if grads else None
        cnt = np.zeros(nq, np.int32) if contribs else None
        ms = ctypes.c_float(0)
        _check(lib().sbh_eval_grad(self.handle, ctypes.byref(p), _ptr(q), nq, _ptr(out), _ptr(g),
                                   _ptr(cnt), ctypes.byref(ms), ctypes.c_void_p(stream)))
        return (out, g, ms.value, cnt) if contribs else (out, g, ms.value)

    def eval_grad_device(self, d_queries: int, nq: int, d_values: int, d_grads: int, p: Params,
                         stream: int = 0, d_contribs: int = 0):
        """Asynchronous sbh_eval_grad_device on device pointers (SoA queries and
        gradients [dim][nq] float32; d_grads may be 0)."""
        _check(lib().sbh_eval_grad_device(self.handle, ctypes.byref(p), ctypes.c_void_p(d_queries),
                                          nq, ctypes.c_void_p(d_values),
                                          ctypes.c_void_p(d_grads or None),
                                          ctypes.c_void_p(d_contribs or None),
                                          ctypes.c_void_p(stream)))

    def check(self, stream: int = 0):
        _check(lib().sbh_gpu_tree_check(self.handle, ctypes.c_void_p(stream)))

    def close(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.sbh_gpu_tree_destroy(self.handle)
        self.handle = None

    def __del__(self):
        self.close()


def _batch_items(entries):
    arr = (BatchItem * len(entries))()
    for i, (tree, p, dq, nq, dout, dcnt, dself) in enumerate(entries):
        arr[i].tree = tree.handle
        arr[i].params = p
        arr[i].d_queries = dq
        arr[i].nq = nq
        arr[i].d_results = dout
        arr[i].d_contribs = dcnt or None
        arr[i].d_self_mass = dself or None
    return arr


def eval_batch(entries, stream: int = 0):
    """sbh_eval_batch: entries are (gpu_tree, params, d_queries, nq, d_results,
    d_contribs or 0, d_self_mass or 0) with device pointers; one pipeline for all."""
    _check(lib().sbh_eval_batch(_batch_items(entries), len(entries), ctypes.c_void_p(stream)))


def batch_tuning(sampler_unit_queries=None, bucket_queries=None, blocks_per_sm=None,
                 bh_unit_queries=None, direct_queries=None) -> BatchTuning:
    """A tuning with the library defaults, overridden where given."""
    t = BatchTuning()
    lib().sbh_batch_tuning_init(ctypes.byref(t))
    if sampler_unit_queries is not None:
        t.sampler_unit_queries = sampler_unit_queries
    if bucket_queries is not None:
        t.bucket_queries = bucket_queries
    if blocks_per_sm is not None:
        t.blocks_per_sm = blocks_per_sm
    if bh_unit_queries is not None:
        t.bh_unit_queries = bh_unit_queries
    if direct_queries is not None:
        t.direct_queries = direct_queries
    return t


def set_batch_tuning(t: BatchTuning, device: int = 0):
    _check(lib().sbh_batch_set_tuning(device, ctypes.byref(t)))


def get_batch_tuning(device: int = 0) -> BatchTuning:
    t = BatchTuning()
    _check(lib().sbh_batch_get_tuning(device, ctypes.byref(t)))
    return t


def batch_autotune(entries, stream: int = 0, repeats: int = 3):
    """sbh_batch_autotune: returns (best tuning, best ms, starting tuning's ms);
    the best is installed for later sbh_eval_batch calls on the device."""
    best = BatchTuning()
    best_ms, start_ms = ctypes.c_float(0), ctypes.c_float(0)
    _check(lib().sbh_batch_autotune(_batch_items(entries), len(entries), ctypes.c_void_p(stream),
                                    repeats, ctypes.byref(best), ctypes.byref(best_ms),
                                    ctypes.byref(start_ms)))
    return best, best_ms.value, start_ms.value


def measure_pipe_rates(device: int = 0) -> dict:
    """sbh_measure_pipe_rates: measured MUFU rsqrt / FFMA / FFMA2-lane rates."""
    v = [ctypes.c_double(0) for _ in range(5)]
    _check(lib().sbh_measure_pipe_rates(device, *[ctypes.byref(x) for x in v]))
    return {"rsqrt_per_s": v[0].value, "ffma_per_s": v[1].value,
            "ffma2_lanes_per_s": v[2].value, "rsqrt_per_clk_sm": v[3].value,
            "sm_clock_mhz": v[4].value}


class Request:
    """A request submitted to a Server; `results` fills in when wait() returns."""

    def __init__(self, server, rid, queries, results, contribs):
        self.server, self.id = server, rid
        self._queries = queries  # kept alive until the request finishes
        self.results, self.contribs = results, contribs
        self.info = None

    def wait(self, timeout_ms: float = -1.0):
        if self.info is None:
            info = RequestInfo()
            _check(lib().sbh_server_wait(self.server.handle, self.id, timeout_ms,
                                         ctypes.byref(info)))
            self.info = {"status": info.status, "batches": info.batches, "nq": info.nq,
                         "queue_ms": info.queue_ms, "latency_ms": info.latency_ms}
            self._queries = None
            if info.status != OK:
                raise SbhError(info.status, "request failed")
        return self.results


class Server:
    """sbh_server_*: resident trees and continuous batching on one device."""

    def __init__(self, device=0, slots=3, slot_queries=1 << 20, max_requests_per_batch=4096,
                 tuning: BatchTuning | None = None):
        cfg = ServerConfig()
        lib().sbh_server_config_init(ctypes.byref(cfg))
        cfg.device, cfg.slots, cfg.slot_queries = device, slots, slot_queries
        cfg.max_requests_per_batch = max_requests_per_batch
        if tuning is not None:
            cfg.tuning = tuning
        h = ctypes.c_void_p()
        _check(lib().sbh_server_create(ctypes.byref(cfg), ctypes.byref(h)))
        self.handle = h
        self.dims = []

    def add_tree(self, tree) -> int:
        """A HostTree (uploaded) or a GpuTree of the server's device (copied)."""
        tid = ctypes.c_int32()
        if isinstance(tree, GpuTree):
            _check(lib().sbh_server_add_gpu_tree(self.handle, tree.handle, ctypes.byref(tid)))
            self.dims.append(tree.dim)
        else:
            _check(lib().sbh_server_add_tree(self.handle, tree.handle, ctypes.byref(tid)))
            self.dims.append(tree.info().dim)
        return tid.value

    def submit(self, tree_id: int, queries, p: Params, contribs: bool = False) -> Request:
        if not 0 <= tree_id < len(self.dims):
            raise SbhError(ERR_INVALID_ARGUMENT, "unknown tree id")
        dim = self.dims[tree_id]
        q = np.asfortranarray(queries, np.float32)
        if q.ndim != 2 or q.shape[1] != dim:
            raise ValueError(f"queries must be (n, {dim})")
        nq = q.shape[0]
        out = np.empty(nq, np.float32)
        cnt = np.empty(nq, np.int32) if contribs else None
        rid = ctypes.c_uint64()
        _check(lib().sbh_server_submit(self.handle, tree_id, ctypes.byref(p), _ptr(q), nq,
                                       _ptr(out), _ptr(cnt), ctypes.byref(rid)))
        return Request(self, rid.value, q, out, cnt)

    def stats(self) -> dict:
        st = ServerStats()
        _check(lib().sbh_server_stats_get(self.handle, ctypes.byref(st)))
        return {"requests": st.requests, "queries": st.queries, "batches": st.batches,
                "busy_ms": st.busy_ms}

    def close(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.sbh_server_destroy(self.handle)
        self.handle = None

    def __del__(self):
        self.close()
