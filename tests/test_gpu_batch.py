"""Batched evaluation and the serving loop on the GPU.

Every request's result must be the same in a batch or in the server's mix as
when evaluated alone: bit for bit for Barnes-Hut and the sampler (per-query
exact traversal; random streams keyed by (seed, query index in the request)),
within the brute-force tolerance for brute force (the batch runs a different
summation schedule)."""
import threading

import numpy as np
import pytest

import sbh_capi as C
import sbh_workloads as W
from helpers import bits_equal

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    torch = pytest.importorskip("torch")
    trees = {}
    pts, nrm, a = W.torus_surface(30000, seed=91)
    lo, hi = W.padded_box(pts)
    trees["torus2"] = C.HostTree(pts, nrm, a, lo, hi, dim_split_log=2)
    pts, nrm, m = W.gaussian_mixture(20000, seed=92)
    lo, hi = W.padded_box(pts)
    trees["gauss1"] = C.HostTree(pts, nrm, m, lo, hi, dim_split_log=1)
    trees["gauss1_pts"] = (pts, m)
    pts, nrm, m = W.circle_points(20000, seed=93)
    lo, hi = W.padded_box(pts)
    trees["circle2"] = C.HostTree(pts, nrm, m, lo, hi, dim_split_log=2, alpha=30.0)
    gpus = {k: C.GpuTree(v) for k, v in trees.items() if isinstance(v, C.HostTree)}
    return torch, trees, gpus


def _dev(torch, q):
    return torch.from_numpy(np.ascontiguousarray(np.asarray(q, np.float32).T)).cuda()


REQUESTS = [
    # tree, method, kernel, nq, extra params
    ("torus2", C.STOCHASTIC, C.WINDING_NUMBER, 1000, dict(samples_per_subdomain=2, seed=5)),
    ("torus2", C.BARNES_HUT, C.WINDING_NUMBER, 33, dict(beta=2.0)),
    ("gauss1", C.BARNES_HUT, C.GRAVITY, 5000, dict(beta=1.25)),
    ("gauss1", C.STOCHASTIC, C.PLUMMER, 1, dict(samples_per_subdomain=3, seed=9)),
    ("circle2", C.STOCHASTIC, C.SMOOTH_DIST, 700, dict(samples_per_subdomain=1, seed=1)),
    ("circle2", C.BARNES_HUT_VOTE, C.GRAVITY, 300, dict(beta=2.0)),
    ("gauss1", C.BRUTE_FORCE, C.GRAVITY, 100, dict()),
    ("torus2", C.BRUTE_FORCE, C.WINDING_NUMBER, 130, dict()),
    ("circle2", C.BRUTE_FORCE, C.SMOOTH_DIST, 65, dict()),
    ("gauss1", C.BRUTE_FORCE, C.PLUMMER, 1, dict()),
    ("torus2", C.STOCHASTIC, C.GRAVITY, 2000, dict(samples_per_subdomain=1, seed=2,
                                                   flags=C.FLAG_KEEP_ORDER)),
    ("gauss1", C.BARNES_HUT, C.PLUMMER, 0, dict(beta=2.0)),
]


def _check_same(method, kernel, got, want):
    if method == C.BRUTE_FORCE and kernel == C.WINDING_NUMBER:
        # sign-changing sums that cancel to ~1e-3 of their O(1) terms: compared
        # in the winding number's natural unit (the jump across the surface)
        assert np.allclose(got, want, rtol=2e-6, atol=2e-6)
    elif method == C.BRUTE_FORCE:
        assert np.allclose(got, want, rtol=2e-6, atol=0)
    elif kernel == C.SMOOTH_DIST:
        assert np.allclose(got, want, rtol=1e-5, atol=1e-30)
    else:
        assert bits_equal(got, want)


def test_batch_matches_single_calls(env):
    torch, trees, gpus = env
    rng = np.random.default_rng(94)
    entries, checks = [], []
    for name, method, kernel, nq, extra in REQUESTS:
        dim = gpus[name].dim
        q = rng.uniform(-1.2, 1.2, (nq, dim)).astype(np.float32)
        p = C.params(method=method, kernel=kernel, **extra)
        dq = _dev(torch, q) if nq else torch.empty((dim, 1), device="cuda")
        out = torch.empty(max(nq, 1), dtype=torch.float32, device="cuda")
        cnt = torch.empty(max(nq, 1), dtype=torch.int32, device="cuda")
        entries.append((gpus[name], p, dq.data_ptr(), nq, out.data_ptr(), cnt.data_ptr(), 0))
        checks.append((name, method, kernel, q, p, dq, out, cnt))
    stream = torch.cuda.current_stream().cuda_stream
    C.eval_batch(entries, stream=stream)
    # A second batch on the same engine (reuses the captured graph).
    C.eval_batch(entries[::-1], stream=stream)
    torch.cuda.synchronize()
    for name, method, kernel, q, p, dq, out, cnt in checks:
        if len(q) == 0:
            continue
        want, _, wcnt = gpus[name].eval(q, p, contribs=True)
        _check_same(method, kernel, out.cpu().numpy()[:len(q)], want)
        if method != C.BRUTE_FORCE:
            assert np.array_equal(cnt.cpu().numpy()[:len(q)], wcnt)


def test_batch_results_do_not_depend_on_request_order(env):
    # The engine reorders requests (by class, then by the cost of their work
    # units); every unit is still summed by one warp on its own, so each
    # request's results are the same bit for bit whatever order it was given in,
    # brute force included.
    torch, trees, gpus = env
    rng = np.random.default_rng(95)
    reqs = []
    for name, method, kernel, nq, extra in REQUESTS:
        if nq == 0:
            continue
        q = rng.uniform(-1.2, 1.2, (nq, gpus[name].dim)).astype(np.float32)
        reqs.append((gpus[name], C.params(method=method, kernel=kernel, **extra), _dev(torch, q),
                     nq))
    stream = torch.cuda.current_stream().cuda_stream
    results = []
    for order in (list(range(len(reqs))), list(reversed(range(len(reqs)))),
                  list(rng.permutation(len(reqs)))):
        outs = [torch.empty(r[3], dtype=torch.float32, device="cuda") for r in reqs]
        entries = [(reqs[i][0], reqs[i][1], reqs[i][2].data_ptr(), reqs[i][3],
                    outs[i].data_ptr(), 0, 0) for i in order]
        C.eval_batch(entries, stream=stream)
        torch.cuda.synchronize()
        results.append([o.cpu().numpy() for o in outs])
    for other in results[1:]:
        for a, b in zip(results[0], other):
            assert bits_equal(a, b)


def test_batch_excludes_self_terms(env):
    torch, trees, gpus = env
    pts, m = trees["gauss1_pts"]
    q = pts[:3000]
    p = C.params(method=C.BARNES_HUT, kernel=C.GRAVITY, beta=2.0)
    dq = _dev(torch, q)
    dm = torch.from_numpy(m[:3000]).cuda()
    out = torch.empty(3000, dtype=torch.float32, device="cuda")
    C.eval_batch([(gpus["gauss1"], p, dq.data_ptr(), 3000, out.data_ptr(), 0, dm.data_ptr())],
                 stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    full, _ = gpus["gauss1"].eval(q, p)
    self_term = np.float32(-1.0) * m[:3000] / np.float32(0.1)  # -m / (0 + 0.1), IEEE float32
    assert bits_equal(out.cpu().numpy(), (full - self_term).astype(np.float32))


def test_server_same_alone_and_in_the_mix(env):
    torch, trees, gpus = env
    # Small slots force requests to be split across batches.
    server = C.Server(slots=3, slot_queries=4096, max_requests_per_batch=64)
    ids = {name: server.add_tree(trees[name]) for name in ("torus2", "gauss1", "circle2")}
    rng = np.random.default_rng(95)
    jobs = []
    for i in range(60):
        name, method, kernel, _, extra = REQUESTS[i % 8]
        nq = int(rng.integers(1, 9000))
        dim = gpus[name].dim
        q = rng.uniform(-1.2, 1.2, (nq, dim)).astype(np.float32)
        jobs.append((name, C.params(method=method, kernel=kernel, **extra), q))
    results = [None] * len(jobs)

    def worker(k):
        reqs = [(j, server.submit(ids[jobs[j][0]], jobs[j][2], jobs[j][1], contribs=True))
                for j in range(k, len(jobs), 4)]
        for j, r in reqs:
            r.wait()
            results[j] = r

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    split = 0
    for (name, p, q), r in zip(jobs, results):
        want, _, wcnt = gpus[name].eval(q, p, contribs=True)
        _check_same(p.method, p.kernel, r.results, want)
        if p.method != C.BRUTE_FORCE:
            assert np.array_equal(r.contribs, wcnt)
        assert r.info["status"] == C.OK and r.info["latency_ms"] >= r.info["queue_ms"] >= 0
        split += r.info["batches"] > 1
    assert split > 0
    st = server.stats()
    assert st["requests"] == len(jobs) and st["batches"] >= split
    server.close()


def test_server_rejects_bad_requests(env):
    torch, trees, gpus = env
    server = C.Server(slots=1, slot_queries=1024)
    tid = server.add_tree(trees["gauss1"])
    with pytest.raises(C.SbhError):
        server.submit(tid + 5, np.zeros((4, 3), np.float32), C.params(method=C.BARNES_HUT))
    with pytest.raises(C.SbhError):
        server.submit(tid, np.zeros((4, 3), np.float32),
                      C.params(method=C.STOCHASTIC, samples_per_subdomain=0))
    r = server.submit(tid, np.zeros((0, 3), np.float32), C.params(method=C.BARNES_HUT))
    assert r.wait().shape == (0,)
    server.close()


def _batch(env, rng_seed=96):
    torch, trees, gpus = env
    rng = np.random.default_rng(rng_seed)
    entries, keep = [], []
    for name, method, kernel, nq, extra in REQUESTS:
        dim = gpus[name].dim
        q = rng.uniform(-1.2, 1.2, (nq, dim)).astype(np.float32)
        p = C.params(method=method, kernel=kernel, **extra)
        dq = _dev(torch, q) if nq else torch.empty((dim, 1), device="cuda")
        out = torch.zeros(max(nq, 1), dtype=torch.float32, device="cuda")
        entries.append((gpus[name], p, dq.data_ptr(), nq, out.data_ptr(), 0, 0))
        keep.append((dq, out, nq))
    return entries, keep


def test_batch_results_do_not_depend_on_tuning(env):
    torch = env[0]
    entries, keep = _batch(env)
    stream = torch.cuda.current_stream().cuda_stream
    default = C.get_batch_tuning()
    outs = []
    try:
        for t in (C.batch_tuning(), C.batch_tuning(sampler_unit_queries=1, bucket_queries=32),
                  C.batch_tuning(sampler_unit_queries=8, bucket_queries=2, blocks_per_sm=1,
                                 bh_unit_queries=8),
                  C.batch_tuning(bh_unit_queries=3), C.batch_tuning(direct_queries=1),
                  C.batch_tuning(direct_queries=0)):
            C.set_batch_tuning(t)
            for _, out, _ in keep:
                out.zero_()
            C.eval_batch(entries, stream=stream)
            torch.cuda.synchronize()
            outs.append([out.cpu().numpy()[:nq].copy() for _, out, nq in keep])
    finally:
        C.set_batch_tuning(default)
    for other in outs[1:]:
        for a, b in zip(outs[0], other):
            assert bits_equal(a, b)
    with pytest.raises(C.SbhError):
        C.set_batch_tuning(C.batch_tuning(sampler_unit_queries=0))
    with pytest.raises(C.SbhError):
        C.set_batch_tuning(C.batch_tuning(bucket_queries=1))
    with pytest.raises(C.SbhError):
        C.set_batch_tuning(C.batch_tuning(bh_unit_queries=33))
    with pytest.raises(C.SbhError):
        C.set_batch_tuning(C.batch_tuning(direct_queries=-1))


def test_direct_stochastic_requests_equal_batched(env):
    """Stochastic requests at or above the tuning's direct_queries leave the
    batch graph for their own sampler launches on side streams: values, counts
    and the self-term subtraction must not change."""
    torch, trees, gpus = env
    pts, m = trees["gauss1_pts"]
    stream = torch.cuda.current_stream().cuda_stream
    reqs = []
    for nq, self_mass in ((3000, True), (777, False), (40, True)):
        dq = _dev(torch, pts[:nq])
        dm = torch.from_numpy(np.ascontiguousarray(m[:nq])).cuda()
        out = torch.empty(nq, dtype=torch.float32, device="cuda")
        cnt = torch.empty(nq, dtype=torch.int32, device="cuda")
        reqs.append((nq, dq, dm if self_mass else None, out, cnt))
    p = C.params(method=C.STOCHASTIC, kernel=C.GRAVITY, samples_per_subdomain=3, seed=11)
    bh = C.params(method=C.BARNES_HUT, kernel=C.GRAVITY, beta=2.0)
    bh_out = torch.empty(500, dtype=torch.float32, device="cuda")
    default = C.get_batch_tuning()
    results = []
    try:
        for direct in (0, 1, 500):
            C.set_batch_tuning(C.batch_tuning(direct_queries=direct))
            entries = [(gpus["gauss1"], p, dq.data_ptr(), nq, out.data_ptr(), cnt.data_ptr(),
                        dm.data_ptr() if dm is not None else 0)
                       for nq, dq, dm, out, cnt in reqs]
            entries.append((gpus["gauss1"], bh, reqs[0][1].data_ptr(), 500, bh_out.data_ptr(), 0,
                            0))
            for _, _, _, out, cnt in reqs:
                out.fill_(float("nan"))
                cnt.fill_(-1)
            C.eval_batch(entries, stream=stream)
            torch.cuda.synchronize()
            results.append([(out.cpu().numpy().copy(), cnt.cpu().numpy().copy())
                            for _, _, _, out, cnt in reqs])
    finally:
        C.set_batch_tuning(default)
    for other in results[1:]:
        for (a, ca), (b, cb) in zip(results[0], other):
            assert bits_equal(a, b)
            assert np.array_equal(ca, cb)
    # the request without self terms equals a plain call
    want, _, wcnt = gpus["gauss1"].eval(pts[:777], p, contribs=True)
    assert bits_equal(results[1][1][0], want)
    assert np.array_equal(results[1][1][1], wcnt)


def test_autotune_installs_a_valid_tuning(env):
    torch, trees, gpus = env
    entries, keep = _batch(env, rng_seed=97)
    stream = torch.cuda.current_stream().cuda_stream
    default = C.get_batch_tuning()
    try:
        best, best_ms, start_ms = C.batch_autotune(entries, stream=stream, repeats=2)
        assert 0 < best_ms <= start_ms
        assert 1 <= best.sampler_unit_queries <= 64 and 2 <= best.bucket_queries <= 4096
        assert best.blocks_per_sm >= 0 and 1 <= best.bh_unit_queries <= 32
        assert C.get_batch_tuning().as_dict() == best.as_dict()
        # the buffers hold the batch's results
        torch.cuda.synchronize()
        for (name, method, kernel, nq, extra), (dq, out, _) in zip(REQUESTS, keep):
            if nq == 0:
                continue
            q = dq.cpu().numpy().T.copy()
            want, _ = gpus[name].eval(q, C.params(method=method, kernel=kernel, **extra))
            _check_same(method, kernel, out.cpu().numpy()[:nq], want)
    finally:
        C.set_batch_tuning(default)


def test_server_with_a_tuning(env):
    torch, trees, gpus = env
    t = C.batch_tuning(sampler_unit_queries=4, bucket_queries=16, blocks_per_sm=2)
    server = C.Server(slots=2, slot_queries=8192, tuning=t)
    tid = server.add_tree(trees["torus2"])
    q = np.random.default_rng(98).uniform(-1.2, 1.2, (5000, 3)).astype(np.float32)
    p = C.params(method=C.STOCHASTIC, kernel=C.WINDING_NUMBER, samples_per_subdomain=2, seed=3)
    r = server.submit(tid, q, p)
    want, _ = gpus["torus2"].eval(q, p)
    assert bits_equal(r.wait(), want)
    server.close()
    with pytest.raises(C.SbhError):
        C.Server(slots=1, slot_queries=1024, tuning=C.batch_tuning(bucket_queries=0))


def test_server_direct_stochastic_parts(env):
    """A stochastic request split across slots, every part at or above
    direct_queries (own sampler launches keyed by the part's offset in the
    request), next to a Barnes-Hut request in the slot graphs: both equal
    single calls, values and counts."""
    torch, trees, gpus = env
    t = C.batch_tuning(direct_queries=1024)
    server = C.Server(slots=2, slot_queries=4096, tuning=t)
    tid = server.add_tree(trees["torus2"])
    rng = np.random.default_rng(99)
    q = rng.uniform(-1.2, 1.2, (10000, 3)).astype(np.float32)
    qb = rng.uniform(-1.2, 1.2, (700, 3)).astype(np.float32)
    p = C.params(method=C.STOCHASTIC, kernel=C.WINDING_NUMBER, samples_per_subdomain=2, seed=8)
    pb = C.params(method=C.BARNES_HUT, kernel=C.WINDING_NUMBER, beta=2.0)
    r = server.submit(tid, q, p, contribs=True)
    rb = server.submit(tid, qb, pb)
    got = r.wait()
    cnt = r.contribs
    want, _, wcnt = gpus["torus2"].eval(q, p, contribs=True)
    assert bits_equal(got, want)
    assert np.array_equal(cnt, wcnt)
    wantb, _ = gpus["torus2"].eval(qb, pb)
    assert bits_equal(rb.wait(), wantb)
    server.close()
