"""sbh_eval_device_static_scratch: evaluation that allocates no device memory.

Some callers cannot allocate device memory while they run -- a serving loop
that reserves its HBM budget at start-up, or code whose memory belongs to a
framework's caching allocator.  For them the C ABI has an entry point whose
per-call scratch (the query ordering of the Barnes-Hut and stochastic methods)
lives in a fixed array inside the library.  These tests call it through the C
ABI twice in a row and compare each result with the allocating entry point
(sbh_eval_device) on the same inputs; the second call is smaller than the first,
so stale contents of the shared array from the first call would show.  Brute
force and calls that keep the given query order use none of the array and take
any query count.  This
file is collected last and needs nothing from the other test files.
"""
import numpy as np
import pytest

import sbh_capi as C
import sbh_workloads as W
from helpers import bits_equal

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    torch = pytest.importorskip("torch")
    pts, nrm, a = W.torus_surface(50_000, seed=81)
    lo, hi = W.padded_box(pts)
    host = C.HostTree(pts, nrm, a, lo, hi, dim_split_log=2)
    gpu = C.GpuTree(host)
    return torch, host, gpu


def _device_queries(torch, nq, seed):
    q = W.uniform_queries(nq, seed=seed)
    return torch.from_numpy(np.ascontiguousarray(q.T)).cuda()


@pytest.mark.parametrize("method,flags", [(C.STOCHASTIC, 0), (C.BARNES_HUT, 0),
                                          (C.STOCHASTIC, C.FLAG_KEEP_ORDER),
                                          (C.BRUTE_FORCE, 0)])
def test_static_scratch_matches_allocating_entry_point(setup, method, flags):
    torch, _, gpu = setup
    stream = torch.cuda.current_stream().cuda_stream
    p = C.params(method=method, kernel=C.WINDING_NUMBER, beta=2.0, samples_per_subdomain=2,
                 seed=11, flags=flags)
    sizes = [(C.STATIC_SCRATCH_MAX_QUERIES, 82), (100_003, 83)]
    inputs = [(_device_queries(torch, nq, seed), nq) for nq, seed in sizes]
    # Expected values from the allocating entry point.
    expected = []
    for dq, nq in inputs:
        out = torch.empty(nq, dtype=torch.float32, device="cuda")
        cnt = torch.empty(nq, dtype=torch.int32, device="cuda")
        gpu.eval_device(dq.data_ptr(), nq, out.data_ptr(), p, stream=stream,
                        d_contribs=cnt.data_ptr())
        expected.append((out, cnt))
    gpu.check(stream)
    # Two calls in a row of the allocation-free entry point.
    got = []
    for dq, nq in inputs:
        out = torch.empty(nq, dtype=torch.float32, device="cuda")
        cnt = torch.empty(nq, dtype=torch.int32, device="cuda")
        gpu.eval_device_static_scratch(dq.data_ptr(), nq, out.data_ptr(), p, stream=stream,
                                       d_contribs=cnt.data_ptr())
        got.append((out, cnt))
    gpu.check(stream)
    for (eo, ec), (go, gc) in zip(expected, got):
        assert bits_equal(go.cpu().numpy(), eo.cpu().numpy())
        assert np.array_equal(gc.cpu().numpy(), ec.cpu().numpy())


def test_static_scratch_rejects_oversized_batches(setup):
    torch, _, gpu = setup
    nq = C.STATIC_SCRATCH_MAX_QUERIES + 1
    dq = _device_queries(torch, nq, 84)
    out = torch.empty(nq, dtype=torch.float32, device="cuda")
    with pytest.raises(C.SbhError) as e:
        gpu.eval_device_static_scratch(dq.data_ptr(), nq, out.data_ptr(),
                                       C.params(method=C.STOCHASTIC, kernel=C.GRAVITY))
    assert e.value.status == C.ERR_INVALID_ARGUMENT
    assert str(C.STATIC_SCRATCH_MAX_QUERIES) in str(e.value)


def test_static_scratch_limit_applies_to_ordering_calls_only(setup):
    """Brute force and calls that keep the given query order use none of the
    fixed array, so they take more queries than it can order."""
    torch, _, gpu = setup
    stream = torch.cuda.current_stream().cuda_stream
    nq = C.STATIC_SCRATCH_MAX_QUERIES + 1000
    dq = _device_queries(torch, nq, 85)
    p = C.params(method=C.STOCHASTIC, kernel=C.GRAVITY, samples_per_subdomain=1, seed=2,
                 flags=C.FLAG_KEEP_ORDER)
    a = torch.empty(nq, dtype=torch.float32, device="cuda")
    b = torch.empty(nq, dtype=torch.float32, device="cuda")
    gpu.eval_device(dq.data_ptr(), nq, a.data_ptr(), p, stream=stream)
    gpu.eval_device_static_scratch(dq.data_ptr(), nq, b.data_ptr(), p, stream=stream)
    gpu.check(stream)
    assert bits_equal(b.cpu().numpy(), a.cpu().numpy())
