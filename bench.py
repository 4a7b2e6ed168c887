"""Benchmark of the stochastic Barnes-Hut summation path on B200.

Default workload (the configuration the headline metric is quoted on): serving.
32 resident trees (16 3D, 16 2D; Gaussian mixtures, torus, sphere and circle
surfaces; 10^4..2*10^6 points) and 1,500 seeded requests (a tree, a kernel --
gravity, winding number or smooth distance with alpha 100 --, 1..10^5 queries in
the tree's box, a sample budget 64/256/1024).  Both paths run at matched
accuracy, median relative error <= 1e-3 against FP64 brute force per kernel
(MATCHED): the plain per-call drop-in at Barnes-Hut's largest sufficient theta
(exact summation where no theta suffices), the served path at the fastest
operating point that meets the target; stochastic BH's own matched figures
(where it meets the target) are reported beside.  The errors are re-measured in
every run.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload serving|sbh_wn|bh_wn|plain_small_bf|plain_small_bh|
                                differentiation|batching|tree_build] [--calibrate]

Serving line: `value` is queries/s of the whole request stream evaluated as one
batch with every request's queries resident in HBM (CUDA events, L2 flushed
between steps); `e2e` the same stream through the server's C ABI (host buffers
in and out, continuous batching, every request submitted at t = 0), with p50 /
p99 latency; `plain_barnes_hut` the reference-style one blocking call per
request; `served_over_plain` their ratio; `latency_at_rates` p50 / p99 under
Poisson arrivals at 0.5x, 1x and 2x the plain path's capacity.

Single-configuration workloads (sbh_wn, bh_wn, plain_small_*): `value` is
queries/s with queries resident in HBM (Morton bucketing + kernel), `e2e` the
blocking C ABI call with pinned host buffers, `e2e_plugin` the reference's own
Python call (`sbh_gpu`) with a float64 NumPy array.  Under torchrun every rank
evaluates its own query batch against its own replica of the tree (replicas
only: the path has no exchange step); `value` is all ranks' queries over the
slowest rank's time.

`--impl reference` times the reference's own CPU implementation (src/sbh.cpp,
compiled unmodified in oracle/_ref) on the same workload and operating points,
on bounded samples, with all host threads; under torchrun only rank 0 runs it.
Accuracy figures come from the oracle's FP64 GPU brute force, outside every
timed region.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "stochastic-barnes-hut_b200")
sys.path.insert(0, PKG)

METRIC = "served vs plain-BH queries/s at 1e-3 med rel err (FP64 ref); p50/p99 ms"
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
L2_FLUSH_BYTES = 512 << 20

# DRAM bytes (read + written) of one launch of each workload's main kernel at
# its default size: dram__bytes_read.sum + dram__bytes_write.sum from a
# single-pass ncu capture of the same bench command (--clock-control none).
# Recaptured after every change to the kernel; the capture command and the
# figures are listed with the kernel's profile.  Null in the bench line when
# the query count or budget is overridden.
DRAM_TRAFFIC = {
    "sbh_wn": 5.8709e9 + 0.2320e9,
    "served_smooth": 194.35e6 + 7.80e6,
    "bh_wn": 307.58e6 + 31.53e6,
    "plain_small_bf": 1.85e6,
    "plain_small_bh": 3.36e6,
}

# What each single-configuration workload measures (the headline metric is the
# serving workload's).
WORKLOAD_METRIC = {
    "sbh_wn": "stochastic BH winding-number queries/s (1,048,576-point torus, 4,194,304 "
              "queries, 256 paths/query)",
    "bh_wn": "deterministic BH winding-number queries/s (1,048,576-point torus, 4,194,304 "
             "queries, theta 0.5)",
    "plain_small_bf": "brute-force Plummer queries/s (65,536 x 65,536)",
    "plain_small_bh": "deterministic BH Plummer queries/s (65,536 x 65,536, theta 0.5, leaf 8)",
}

WORKLOADS = {
    # name: (description, method, kernel, n points, n queries, tree kind, budget/beta)
    "sbh_wn": dict(desc="stochastic BH winding number, torus 1,048,576 pts, 4,194,304 queries, "
                        "Octree2 (branching 64, leaf 1), 256 sampled paths/query",
                   method="stochastic", kernel="wn", n=1 << 20, nq=1 << 22, dsl=2, leaf=1,
                   budget=256, source="torus"),
    "bh_wn": dict(desc="deterministic BH winding number, torus 1,048,576 pts, 4,194,304 queries, "
                       "Octree1 (branching 8, leaf 1), theta 0.5",
                  method="barnes_hut", kernel="wn", n=1 << 20, nq=1 << 22, dsl=1, leaf=1,
                  beta=2.0, source="torus"),
    "plain_small_bf": dict(desc="brute-force Plummer potential (eps 1e-3), 65,536 Gaussian-mixture "
                                "sources x 65,536 queries", method="brute_force",
                           kernel="plummer", n=65536, nq=65536, dsl=1, leaf=8, source="gauss"),
    "plain_small_bh": dict(desc="deterministic BH Plummer potential (eps 1e-3), 65,536 "
                                "Gaussian-mixture sources x 65,536 queries, theta 0.5, leaf 8",
                           method="barnes_hut", kernel="plummer", n=65536, nq=65536, dsl=1,
                           leaf=8, beta=2.0, source="gauss"),
}


def load_peaks():
    try:
        with open(PEAKS_FILE) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def make_inputs(wl, rank=0):
    import sbh_workloads as W
    if wl["source"] == "torus":
        pts, nrm, m = W.torus_surface(wl["n"], seed=2024)
    else:
        pts, nrm, m = W.gaussian_mixture(wl["n"], seed=2024)
    lo, hi = W.padded_box(pts)
    q = W.uniform_queries(wl["nq"], seed=4048 + rank)
    return pts, nrm, m, lo, hi, q


def kernel_id(C, name):
    return {"gravity": C.GRAVITY, "wn": C.WINDING_NUMBER, "smooth": C.SMOOTH_DIST,
            "plummer": C.PLUMMER}[name]


def method_id(C, name):
    return {"brute_force": C.BRUTE_FORCE, "barnes_hut": C.BARNES_HUT,
            "stochastic": C.STOCHASTIC}[name]


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled during the timed
    region: NVML polled every 2 ms from a thread (read-only queries), or
    nvidia-smi at 100 ms where NVML is unavailable."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.sm, self.sm_max, self.reasons = [], [], set()
        self.proc = None
        self.thread = None
        self.stop = threading.Event()

    def _nvml_handle(self):
        """NVML handle of CUDA device `dev`: the NVML device whose PCI domain,
        bus and device numbers equal the CUDA device's (NVML enumerates every
        GPU of the machine, CUDA only the visible ones).  Only NVML handles and
        integers are passed to NVML."""
        import pynvml
        import torch
        pynvml.nvmlInit()
        props = torch.cuda.get_device_properties(self.dev)
        want = (int(props.pci_domain_id), int(props.pci_bus_id), int(props.pci_device_id))
        for i in range(pynvml.nvmlDeviceGetCount()):
            h = pynvml.nvmlDeviceGetHandleByIndex(i)
            pci = pynvml.nvmlDeviceGetPciInfo(h)
            if (int(pci.domain), int(pci.bus), int(pci.device)) == want:
                return pynvml, h
        raise RuntimeError("no NVML device matches the CUDA device")

    def _poll_nvml(self, nv, h):
        masks = [(name, getattr(nv, attr)) for name, attr in self.REASONS]
        while not self.stop.is_set():
            try:
                self.sm.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
                self.sm_max.append(float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.reasons.update(name for name, m in masks if r & m)
            except Exception:
                break
            self.stop.wait(0.002)

    def _read_smi(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) != 9:
                continue
            if parts[1].replace(".", "").isdigit():
                self.sm.append(float(parts[1]))
            if parts[2].replace(".", "").isdigit():
                self.sm_max.append(float(parts[2]))
            self.reasons.update(self.REASONS[i][0] for i in range(4)
                                if parts[5 + i].lower() == "active")

    def __enter__(self):
        try:
            nv, h = self._nvml_handle()
            self.thread = threading.Thread(target=self._poll_nvml, args=(nv, h), daemon=True)
        except Exception:
            try:
                self.proc = subprocess.Popen(
                    ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                     "-lms", "100", "-i", str(self.dev)], stdout=subprocess.PIPE,
                    stderr=subprocess.DEVNULL, text=True)
                self.thread = threading.Thread(target=self._read_smi, daemon=True)
            except Exception:
                self.thread = None
        if self.thread:
            self.thread.start()
        return self

    def __exit__(self, *a):
        self.stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)

    def summary(self):
        if not self.sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(self.sm),
                "sm_max_mhz": max(self.sm_max) if self.sm_max else None,
                "reasons": sorted(self.reasons), "samples": len(self.sm)}


def max_over_ranks(values, dist, device):
    """Element-wise maximum of each rank's timings, returned on every rank (the
    job's time is its slowest rank's).  `dist` is torch.distributed with a
    process group initialised, or None for a single process."""
    if dist is None:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def whole_job_rate(world, units_per_rank, total_ms, steps):
    """Units all ranks processed per second, over the slowest rank's time."""
    return world * units_per_rank / (total_ms / 1e3 / steps)


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def pair_pipe_bound(rates, kernel, dim=3):
    """Pairs per second the all-pairs kernels' arithmetic allows: the slower of
    the MUFU pipe (its measured rsqrt rate; every MUFU operation issues at that
    rate) and the FP32 pipe (measured FFMA rate), for the operations a pair
    costs in pairs.cuh: Plummer one rsqrt; gravity a sqrt and a reciprocal; the
    winding number a reciprocal (and a sqrt in 3D); the smooth distance a sqrt,
    and an exponential on the MUFU for three sources in four, on the FP32 pipe
    (eight operations) for the fourth.  Returns (pairs/s, MUFU ops per pair,
    FP32 lane operations per pair)."""
    sub = 3 if dim == 3 else 2  # the differences; r^2 (or n.d) takes as many more
    mufu, fp32 = {
        "plummer": (1.0, 2 * sub + 1),
        "gravity": (2.0, 2 * sub + 2),
        "wn": (2.0 if dim == 3 else 1.0, 3 * sub + 4),
        "smooth": (1.75, 2 * sub + 2 + 0.25 * 8),
    }[kernel]
    return min(rates["rsqrt_per_s"] / mufu, rates["ffma_per_s"] / fp32), mufu, fp32


def dram_traffic(wl):
    """DRAM bytes per launch of the workload's main kernel (ncu), or None."""
    if wl.get("resized"):
        return None
    return DRAM_TRAFFIC.get(wl.get("name"))


def timed_device(fn, stream, flush, warmup, steps):
    """Event-timed runs of fn() on `stream`, L2 flushed before each; ms per run."""
    import torch
    for _ in range(warmup):
        flush.zero_()
        fn()
    ev = []
    for _ in range(steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        ev.append((e0, e1))
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in ev]


def sampler_load_bytes(info_l2, leaf_points, nq, paths, deeper_terms):
    """Global-memory bytes the stochastic kernel's loads request per launch,
    from its own counts: the first-level records (32 B each: centroid/diameter
    and aggregate) staged once per warp of 32 queries; per sampled path its
    subdomain's topology (16 B), the sample's path code (8 B), the subdomain's
    centroid (16 B), its child mask (8 B) and the topology and centroid of the
    node the first step reaches (32 B); 32 B per deeper kernel term."""
    units = (nq + 31) // 32
    return units * (info_l2 + leaf_points) * 32 + nq * paths * 80 + deeper_terms * 32


def run_ours(args, wl):
    import torch

    import sbh_capi as C
    import sbh_workloads as W

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    s_handle = stream.cuda_stream

    pts, nrm, m, lo, hi, q = make_inputs(wl, rank)
    t0 = time.perf_counter()
    host = C.HostTree(pts, nrm, m, lo, hi, dim_split_log=wl["dsl"], leaf_size=wl["leaf"])
    build_s = time.perf_counter() - t0
    gpu = C.GpuTree(host, device=local)
    info = gpu.info
    nq = q.shape[0]
    samples = W.samples_for_budget(wl.get("budget", 1), info.root_children)
    p = C.params(method=method_id(C, wl["method"]), kernel=kernel_id(C, wl["kernel"]),
                 beta=wl.get("beta", 2.0), samples_per_subdomain=samples, seed=1234,
                 flags=C.FLAG_STAGE_LEAVES if args.stage_leaves else 0)

    d_q = torch.from_numpy(np.ascontiguousarray(q.T)).to(dev)  # SoA [3][nq]
    d_out = torch.empty(nq, dtype=torch.float32, device=dev)
    d_cnt = torch.empty(nq, dtype=torch.int32, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)

    def step_device():
        gpu.eval_device(d_q.data_ptr(), nq, d_out.data_ptr(), p, stream=s_handle)

    # Work counts (untimed): contributions per query (the reference's count).
    gpu.eval_device(d_q.data_ptr(), nq, d_out.data_ptr(), p, stream=s_handle,
                    d_contribs=d_cnt.data_ptr())
    gpu.check(s_handle)
    contribs = d_cnt.to(torch.int64).sum().item()

    # Device-resident timing.
    for _ in range(args.warmup):
        flush.zero_()
        step_device()
    gpu.check(s_handle)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    times = []
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step_device()
            e1.record(stream)
            times.append((e0, e1))
        torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    gpu.check(s_handle)
    step_ms = [a.elapsed_time(b) for a, b in times]
    total_ms = float(sum(step_ms))

    # Dominant kernel alone: the evaluation on pre-bucketed queries (no sort launch).
    order = morton_order(q)
    d_qs = torch.from_numpy(np.ascontiguousarray(q[order].T)).to(dev)
    pk = C.params(method=p.method, kernel=p.kernel, beta=p.beta, samples_per_subdomain=samples,
                  seed=p.seed, flags=p.flags | C.FLAG_KEEP_ORDER)
    kern_ms = timed_device(lambda: gpu.eval_device(d_qs.data_ptr(), nq, d_out.data_ptr(), pk,
                                                   stream=s_handle),
                           stream, flush, max(1, args.warmup), args.steps)

    # End to end through the blocking C ABI call with pinned host buffers.
    h_q = torch.from_numpy(np.ascontiguousarray(q.T)).pin_memory()
    h_out = torch.empty(nq, dtype=torch.float32).pin_memory()
    for _ in range(args.warmup):
        gpu.eval_host_ptr(h_q.data_ptr(), nq, h_out.data_ptr(), p, stream=s_handle)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    e2e = []
    for _ in range(args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        gpu.eval_host_ptr(h_q.data_ptr(), nq, h_out.data_ptr(), p, stream=s_handle)
        e1.record(stream)
        e2e.append((e0, e1))
    torch.cuda.synchronize(dev)
    e2e_ms = float(sum(a.elapsed_time(b) for a, b in e2e))

    # End to end through the reference's own Python call: the `sbh_gpu` module
    # with a NumPy float64 (n, 3) array, as the reference's callers pass it
    # (pageable memory, float64 -> float32 conversion and layout change inside).
    plugin = plugin_e2e(wl, pts, nrm, m, lo, hi, q, samples, args)

    # Accuracy on a query subset against FP64 brute force, and (stochastic) the
    # Pareto comparison with deterministic Barnes-Hut the workload prescribes.
    accuracy = compare = None
    if not args.no_accuracy:
        accuracy, compare = accuracy_report(C, torch, wl, gpu, p, pts, nrm, m, lo, hi, d_q, nq,
                                            s_handle, args)

    if dist:
        total_ms, e2e_ms = max_over_ranks([total_ms, e2e_ms], dist, dev)
        dist.destroy_process_group()
    if rank != 0:
        return None

    kmean_s = statistics.mean(kern_ms) / 1e3
    peak, peak_kind = load_peaks()
    traffic = dram_traffic(wl)
    if wl["method"] == "brute_force":
        # Brute force is bound by its arithmetic pipes (pair_pipe_bound).
        rates = C.measure_pipe_rates(local)
        bound, mufu_per_pair, fp32_per_pair = pair_pipe_bound(rates, wl["kernel"])
        pairs = float(nq) * float(wl["n"])
        roofline = {
            "bound": "sfu", "kernel": "brute_force_kernel",
            "achieved": pairs / kmean_s, "peak": bound,
            "unit": "pairs/s", "frac": pairs / kmean_s / bound,
            "peak_source": "measured MUFU rsqrt rate (sbh_measure_pipe_rates): "
                           f"{rates['rsqrt_per_clk_sm']:.2f}/clk/SM at "
                           f"{rates['sm_clock_mhz']:.0f} MHz; {mufu_per_pair} MUFU op(s) and "
                           f"{fp32_per_pair} FP32 lane op(s) per pair",
            "kernel_ms": statistics.mean(kern_ms), "pairs_per_launch": pairs,
            "pipe_rates": rates, "traffic": traffic,
        }
    else:
        if wl["method"] == "stochastic":
            l2, terms, internal, leafpts = sampler_first_level(host)
            first = nq * (samples * terms + internal + leafpts)
            deeper = max(0, contribs - first)
            alg = sampler_load_bytes(l2, leafpts, nq, samples * info.root_children, deeper)
            definition = ("global-memory bytes the kernel's loads request, from its own counts: "
                          "first-level records 32 B each once per 32 queries, 80 B per sampled "
                          "path's first step, 32 B per deeper kernel term")
            kernel_name = "stochastic_kernel"
        else:
            bpe = 32 if wl["kernel"] == "wn" else 16
            alg = contribs * bpe + nq * 16
            definition = (f"{bpe} B per kernel evaluation (node or point record) + 16 B per "
                          "query (SURVEY 8(d) per-unit figure; the opening tests' 32 B reads are "
                          "not counted)")
            kernel_name = "barnes_hut_kernel"
        roofline = {
            "bound": "issue", "kernel": kernel_name,
            "achieved": alg / kmean_s / 1e9, "peak": peak, "unit": "GB/s",
            "frac": alg / kmean_s / 1e9 / peak,
            "peak_source": (f"{peak_kind} HBM copy bandwidth (MEASURED_PEAKS.json hbm_gbs)"
                            if peak_kind == "measured" else "fallback 6650 GB/s"),
            "kernel_ms": statistics.mean(kern_ms),
            "algorithmic_bytes": alg, "bytes_definition": definition,
            "traffic": traffic,
            "dram_gbs": None if traffic is None else traffic / kmean_s / 1e9,
            "dram_frac": None if traffic is None else traffic / kmean_s / 1e9 / peak,
            "note": "issue- and latency-bound (ncu: the traversal's records come from L1/L2; "
                    "DRAM traffic is a small fraction of HBM bandwidth); achieved/frac are the "
                    "requested load bandwidth against the HBM roof, dram_frac the DRAM share",
        }
    launches_per_step = {"stochastic": 6, "barnes_hut": 6, "brute_force": 1}[wl["method"]]
    clk = clocks.summary()
    out = {
        "metric": WORKLOAD_METRIC[wl["name"]],
        "value": whole_job_rate(world, nq, total_ms, args.steps),
        "unit": "queries/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded generators; the reference publishes no dataset)",
        "config": dict(workload_config(wl, info.num_nodes, info.root_children, samples),
                       **({"leaf_staging": "bulk asynchronous copies (SBH_FLAG_STAGE_LEAVES)"}
                          if args.stage_leaves else {})),
        "work": {"mean_kernel_evals_per_query_reference_count": contribs / nq,
                 "host_build_s": round(build_s, 3)},
        "e2e": {"value": whole_job_rate(world, nq, e2e_ms, args.steps), "unit": "queries/s",
                "h2d_bytes_per_step": nq * 12, "d2h_bytes_per_step": nq * 4,
                "ms_per_step": e2e_ms / args.steps,
                "path": "sbh_eval (C ABI), pinned float32 SoA host buffers"},
        "roofline": roofline,
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clk,
    }
    if plugin is not None:
        out["e2e_plugin"] = plugin
    if accuracy is not None:
        out["accuracy"] = accuracy
        out["compare"] = compare
    if not args.no_cpu_baseline and world == 1:
        out["cpu_baseline"] = cpu_baseline(wl, pts, nrm, m, lo, hi, q, samples,
                                           budget_s=args.cpu_seconds)
    return out


def workload_config(wl, num_nodes, root_children, samples):
    """The configuration keys both arms report (identical for the same workload)."""
    return {
        "workload": wl["desc"],
        "method": wl["method"], "kernel": wl["kernel"], "points": wl["n"],
        "queries_per_gpu": wl["nq"], "tree": f"dim 3, dim_split_log {wl['dsl']}, leaf {wl['leaf']}",
        "tree_nodes": num_nodes, "root_children": root_children,
        "samples_per_subdomain": samples if wl["method"] == "stochastic" else None,
        "paths_per_query": samples * root_children if wl["method"] == "stochastic" else None,
        "beta": wl.get("beta"),
        "l2": "512 MiB buffer written between timed steps; tree+queries exceed L2 as well",
    }


def sampler_first_level(host):
    """The root's first level as the sampler sums it: (records in the range of
    the root's grandchildren, kernel terms they stand for -- a leaf record
    holding several points, or none, stands for its points --, internal root
    children, points of leaf root children)."""
    n = host.export_nodes()
    kids = np.nonzero(n["parent"] == 0)[0]
    kids = kids[kids != 0]
    leaf = n["is_leaf"][kids].astype(bool)
    internal = kids[~leaf]
    grand = np.isin(n["parent"], internal)
    grand[0] = False
    pts = n["end"][grand] - n["start"][grand]
    terms = np.where(n["is_leaf"][grand].astype(bool), pts, 1)
    leafpts = int((n["end"][kids[leaf]] - n["start"][kids[leaf]]).sum())
    return int(grand.sum()), int(terms.sum()), int(len(internal)), leafpts


def plugin_e2e(wl, pts, nrm, m, lo, hi, q, samples, args):
    """Wall-clock of the reference-facing Python call (`sbh_gpu`, blocking)
    with a float64 (n, 3) NumPy array, the form the reference's callers use."""
    import sbh
    import sbh_gpu
    cls = {1: "Octree1", 2: "Octree2", 3: "Octree3"}[wl["dsl"]]
    if wl["leaf"] != 1:
        return None
    h = getattr(sbh, cls)(pts, nrm, m, lo, hi)
    g = getattr(sbh_gpu, cls.replace("Octree", "OctreeGPU"))(h)
    q64 = q.astype(np.float64)
    suffix = {"wn": "wn", "gravity": "gravity", "smooth": "smoothdist"}.get(wl["kernel"])
    if suffix is None:
        return None
    if wl["method"] == "stochastic":
        fn = lambda: getattr(sbh_gpu, "multi_level_prefix_control_variate_" + suffix)(
            g, q64, samples)
        call = f"sbh_gpu.multi_level_prefix_control_variate_{suffix}(tree, q, {samples})"
    elif wl["method"] == "barnes_hut":
        fn = lambda: getattr(sbh_gpu, "eval_barnes_hut_" + suffix)(g, q64, wl.get("beta", 2.0))
        call = f"sbh_gpu.eval_barnes_hut_{suffix}(tree, q, {wl.get('beta', 2.0)})"
    else:
        fn = lambda: getattr(sbh_gpu, "eval_brute_force_" + suffix)(g, q64)
        call = f"sbh_gpu.eval_brute_force_{suffix}(tree, q)"
    for _ in range(max(1, args.warmup // 2)):
        fn()
    steps = max(2, args.steps // 4)
    t0 = time.perf_counter()
    for _ in range(steps):
        fn()
    secs = (time.perf_counter() - t0) / steps
    return {"value": len(q) / secs, "unit": "queries/s", "ms_per_step": secs * 1e3,
            "h2d_bytes_per_step": len(q) * 12, "d2h_bytes_per_step": len(q) * 4,
            "call": call + " with q a C-ordered float64 (n, 3) NumPy array; host wall clock",
            "steps": steps}


ACCURACY_SUBSET = 65536


def rel_errors(kernel, est, ref):
    """Per-query relative error.  The winding number vanishes outside the
    surface, so its error is taken relative to max(|ref|, 1) (its natural unit:
    the jump across the surface); the potentials never vanish."""
    est = est.astype(np.float64)
    if kernel == "wn":
        return np.abs(est - ref) / np.maximum(np.abs(ref), 1.0)
    return np.abs(est - ref) / np.abs(ref)


def fp64_reference(pts, nrm, m, kernel, q, alpha=1.0):
    """FP64 brute force on the GPU, from the oracle (libsbh_bf64.so): the
    accuracy reference, computed outside every timed region."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    kid = {"gravity": O.GRAVITY, "wn": O.WINDING_NUMBER, "smooth": O.SMOOTH_DIST,
           "plummer": O.PLUMMER}[kernel]
    return O.gpu_brute_force_f64(pts, nrm, m, kid, q, alpha=alpha)


def accuracy_report(C, torch, wl, gpu, p, pts, nrm, m, lo, hi, d_q, nq, s_handle, args):
    dev = d_q.device
    n_sub = min(ACCURACY_SUBSET, nq)
    q_sub = d_q[:, :n_sub].t().contiguous().cpu().numpy()
    ref = fp64_reference(pts, nrm, m, wl["kernel"], q_sub)
    d_sub = d_q[:, :n_sub].contiguous()
    est = torch.empty(n_sub, dtype=torch.float32, device=dev)
    gpu.eval_device(d_sub.data_ptr(), n_sub, est.data_ptr(), p, stream=s_handle)
    torch.cuda.synchronize(dev)
    e = rel_errors(wl["kernel"], est.cpu().numpy(), ref)
    accuracy = {"median_rel_err": float(np.median(e)), "p99_rel_err": float(np.percentile(e, 99)),
                "subset_queries": n_sub,
                "reference": "FP64 brute force on the GPU (the oracle's libsbh_bf64.so)",
                "definition": ("|est-ref|/max(|ref|,1)" if wl["kernel"] == "wn"
                               else "|est-ref|/|ref|")}
    compare = {}
    if wl["method"] != "stochastic":
        return accuracy, compare
    # Pareto comparison on the same queries: the sampler at budgets 64-1024 on
    # this tree, deterministic Barnes-Hut at theta 0.3/0.5/0.8 on Octree1 (the
    # reference's recommended tree for it); throughput on all queries
    # (device-resident, sort included), errors on the subset.
    host1 = C.HostTree(pts, nrm, m, lo, hi, dim_split_log=1, leaf_size=1)
    gpu1 = C.GpuTree(host1, device=dev.index or 0)
    out = torch.empty(nq, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    kid = p.kernel
    R = gpu.info.root_children
    runs = [(f"stochastic_budget_{b}", gpu,
             C.params(method=C.STOCHASTIC, kernel=kid, samples_per_subdomain=max(1, b // R),
                      seed=p.seed), {"tree": "dim_split_log 2 (branching 64), leaf 1",
                                     "paths_per_query": max(1, b // R) * R})
            for b in (64, 128, 256, 512, 1024)]
    runs += [(f"barnes_hut_theta_{th}", gpu1, C.params(method=C.BARNES_HUT, kernel=kid,
                                                       beta=1.0 / th),
              {"tree": "dim_split_log 1 (branching 8), leaf 1"}) for th in (0.3, 0.5, 0.8)]
    for name, g, pr, extra in runs:
        ms = statistics.mean(timed_device(
            lambda: g.eval_device(d_q.data_ptr(), nq, out.data_ptr(), pr, stream=s_handle),
            stream, flush, 3, max(3, args.steps // 4)))
        eb = rel_errors(wl["kernel"], out[:n_sub].cpu().numpy(), ref)
        compare[name] = dict(extra, queries_per_s=nq / (ms / 1e3), ms_per_step=ms,
                             median_rel_err=float(np.median(eb)),
                             p99_rel_err=float(np.percentile(eb, 99)))
    gpu1.check(s_handle)
    return accuracy, compare


def morton_order(q):
    lo, hi = q.min(0), q.max(0)
    c = np.clip(((q - lo) / np.maximum(hi - lo, 1e-30) * 64).astype(np.int64), 0, 63)
    key = np.zeros(len(q), np.int64)
    for b in range(6):
        for d in range(3):
            key |= ((c[:, d] >> b) & 1) << (3 * b + d)
    return np.argsort(key, kind="stable")


def cpu_baseline(wl, pts, nrm, m, lo, hi, q, samples, budget_s=20.0):
    """The reference's CPU plugin on a bounded sample of the same workload."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not O.ref_available():
        return {"value": None, "unit": "queries/s", "kind": "reference",
                "sample": "unavailable: oracle/_ref not built"}
    t = O.RefTree(pts, nrm, m, lo, hi, dim_split_log=wl["dsl"], leaf_size=wl["leaf"])
    kid = {"gravity": 0, "wn": 1, "smooth": 2}.get(wl["kernel"])
    cores = O.ref_hardware_concurrency()
    # Probe with a small sample, then size the timed sample to ~budget_s.
    n0 = 512
    secs = run_ref(t, wl, kid, q[:n0], samples)
    n = int(min(len(q), max(n0, n0 * budget_s / max(secs, 1e-3))))
    secs = run_ref(t, wl, kid, q[:n], samples)
    return {"value": n / secs, "unit": "queries/s", "cores": cores, "kind": "reference",
            "sample": f"first {n} of the {len(q)} queries, same tree and parameters, "
                      f"{secs:.1f} s, src/sbh.cpp thread pool ({cores} threads)"}


def run_ref(t, wl, kid, q, samples):
    if wl["method"] == "stochastic":
        _, _, secs = t.plugin_sbh(kid, q, samples)
    elif wl["method"] == "barnes_hut":
        if kid is None:
            t0 = time.perf_counter()
            t.bh(3, q, wl.get("beta", 2.0))
            return time.perf_counter() - t0
        _, secs = t.plugin_bh(kid, q, wl.get("beta", 2.0))
    else:  # brute force: the reference CPU path is Barnes-Hut with beta = inf
        if kid is None:
            t0 = time.perf_counter()
            t.bh(3, q, np.inf)
            return time.perf_counter() - t0
        _, secs = t.plugin_bh(kid, q, np.inf)
    return secs


def run_reference(args, wl):
    """The reference's own CPU plugin (src/sbh.cpp, compiled unmodified in
    oracle/_ref) on the same workload: its std::thread pool over all host
    threads, a bounded query sample per step.  Nothing of this library is
    loaded: the tree, its root-child count (the sampler's budget mapping) and
    the configuration come from the reference build itself."""
    world, rank, _ = dist_setup()
    if rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import sbh_workloads as W
    if not O.ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libsbh_ref.so is not built"}
    pts, nrm, m, lo, hi, q = make_inputs(wl, 0)
    t = O.RefTree(pts, nrm, m, lo, hi, dim_split_log=wl["dsl"], leaf_size=wl["leaf"])
    samples = W.samples_for_budget(wl.get("budget", 1), t.root_children)
    kid = {"gravity": 0, "wn": 1, "smooth": 2}.get(wl["kernel"])
    cores = O.ref_hardware_concurrency()
    per_step = max(64, args.ref_sample)
    secs = run_ref(t, wl, kid, q[:64], samples)
    per_step = int(min(per_step, max(64, 64 * args.ref_step_seconds / max(secs, 1e-3))))
    for i in range(args.warmup):
        run_ref(t, wl, kid, q[:min(per_step, 256)], samples)
    total = 0.0
    for i in range(args.steps):
        lo_i = (i * per_step) % max(1, len(q) - per_step)
        total += run_ref(t, wl, kid, q[lo_i:lo_i + per_step], samples)
    value = args.steps * per_step / total
    sample = (f"{per_step} queries per step of the {len(q)}-query workload, "
              f"src/sbh.cpp thread pool ({cores} threads), tree build excluded")
    return {
        "impl": "reference", "metric": WORKLOAD_METRIC[wl["name"]], "value": value,
        "unit": "queries/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded generators; the reference publishes no dataset)",
        "config": workload_config(wl, t.num_nodes, t.root_children, samples),
        "cpu_baseline": {"value": value, "unit": "queries/s", "cores": cores,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


# ----------------------------------------------------------------- serving

SERVING_KERNELS = ("gravity", "wn", "smooth")
# The server's slots: 3 batch contexts of up to 2^21 queries each.  Measured on
# the stream submitted at t = 0 (two runs each): 3 x 2^20 queries 19.9-20.6 M
# queries/s (p99 578-622 ms), 4 x 2^20 21.8-22.7 M, 2 x 2^22 22.2-24.9 M,
# 3 x 2^21 23.9-24.2 M (p99 529-536 ms).
SERVER_SLOT_QUERIES = 1 << 21
SERVING_KID = {"gravity": 0, "wn": 1, "smooth": 2}  # SBH_KERNEL_* (the reference's KernelFuncID)
SERVING_ALPHA = 100.0
MATCH_TARGET = 1e-3

# Operating points at matched accuracy: median relative error <= 1e-3 against
# FP64 brute force, per kernel, on the serving mix.  An operating point is
# (method, parameter): ("barnes_hut", theta), ("stochastic", factor on every
# request's drawn sample budget 64/256/1024) or ("brute_force", None).
#   plain       the per-call drop-in: Barnes-Hut at the largest theta that meets
#               the target, or exact summation where no theta of the ladder does
#   stochastic  the smallest budget factor at which stochastic BH meets the
#               target (None: not within 16x the drawn budgets)
#   served      the fastest of the points that meet the target, by the batched
#               throughput the calibration measures
# Chosen by `python bench.py --workload serving --calibrate` (FP64 references of
# 50 requests per kernel; the ladders and timings are kept with the profiles);
# every bench run re-measures the errors at these points.
MATCHED = {
    "gravity": {"plain": ("barnes_hut", 0.5), "stochastic": 0.25,
                "served": ("barnes_hut", 0.5)},
    "wn": {"plain": ("barnes_hut", 0.2), "stochastic": None, "served": ("barnes_hut", 0.2)},
    "smooth": {"plain": ("brute_force", None), "stochastic": None,
               "served": ("brute_force", None)},
}
CAL_THETAS = (0.8, 0.6, 0.5, 0.4, 0.3, 0.25, 0.2, 0.15, 0.1, 0.07, 0.05)
CAL_SCALES = (0.25, 0.5, 1.0, 2.0, 4.0, 8.0, 16.0)


def serving_setup(C, seed=77, n_trees=32, n_requests=1500, device_trees=True, device=0):
    """32 resident trees (16 3D, 16 2D; Gaussian mixtures, torus, sphere and
    circle surfaces; 10^4..2*10^6 points log-uniform) and a seeded request list:
    tree, kernel (gravity / winding number / smooth distance alpha 100), query
    count log-uniform in [1, 10^5] uniform in the tree's box, budget 64/256/1024.
    With device_trees the trees are built on the GPU in both layouts (Octree1 /
    Quadtree1 for Barnes-Hut and brute force, Octree2 / Quadtree2 for the
    sampler)."""
    import sbh_workloads as W
    rng = np.random.default_rng(seed)
    trees = []
    for i in range(n_trees):
        dim = 3 if i < n_trees // 2 else 2
        n = int(np.exp(rng.uniform(np.log(1e4), np.log(2e6))))
        if dim == 3:
            kind = ("gauss", "torus", "sphere")[i % 3]
            pts, nrm, m = (W.gaussian_mixture(n, seed + i) if kind == "gauss" else
                           W.torus_surface(n, seed + i) if kind == "torus" else
                           W.sphere_surface(n, seed + i))
        else:
            kind = ("gauss", "circle")[i % 2]
            pts, nrm, m = (W.gaussian_mixture(n, seed + i, dim=2) if kind == "gauss" else
                           W.circle_points(n, seed + i))
        lo, hi = W.padded_box(pts)
        t = dict(dim=dim, kind=kind, n=n, lo=lo, hi=hi, pts=pts, nrm=nrm, m=m)
        if device_trees:
            # built on the device (sbh_gpu_tree_build; the same trees as a host build)
            t["bh"] = C.GpuTree.build(pts, nrm, m, lo, hi, dim_split_log=1, device=device)
            t["sbh"] = C.GpuTree.build(pts, nrm, m, lo, hi, dim_split_log=2, device=device)
            t["root2"] = t["sbh"].info.root_children
        trees.append(t)
    reqs = []
    for r in range(n_requests):
        ti = int(rng.integers(n_trees))
        t = trees[ti]
        kern = SERVING_KERNELS[int(rng.integers(3))]
        nq = int(np.exp(rng.uniform(0.0, np.log(1e5))))
        budget = int(rng.choice([64, 256, 1024]))
        q = rng.uniform(t["lo"], t["hi"], (nq, t["dim"])).astype(np.float32)
        reqs.append(dict(tree=ti, kernel=kern, nq=nq, budget=budget, q=np.asfortranarray(q)))
    return trees, reqs


def request_params(C, W, t, r, op):
    """Parameters of request r at operating point op = (method, parameter)."""
    method, x = op
    kid = SERVING_KID[r["kernel"]]
    alpha = SERVING_ALPHA if r["kernel"] == "smooth" else None
    if method == "stochastic":
        return C.params(method=C.STOCHASTIC, kernel=kid, alpha=alpha, seed=r["nq"],
                        samples_per_subdomain=W.samples_for_budget(
                            int(round(r["budget"] * x)), t["root2"]))
    if method == "barnes_hut":
        return C.params(method=C.BARNES_HUT, kernel=kid, alpha=alpha, beta=1.0 / x)
    return C.params(method=C.BRUTE_FORCE, kernel=kid, alpha=alpha)


def op_of(r, role):
    """The operating point of request r in a role: "plain", "served", or
    "served_stochastic" (stochastic BH where it meets the target, else the
    served point)."""
    m = MATCHED[r["kernel"]]
    if role == "served_stochastic":
        return ("stochastic", m["stochastic"]) if m["stochastic"] is not None else m["served"]
    return m[role]


def tree_key(op):
    return "sbh" if op[0] == "stochastic" else "bh"


def wait_until(t0, at):
    while True:
        d = at - (time.perf_counter() - t0)
        if d <= 0:
            return
        time.sleep(d if d > 2e-3 else 0)


def drive_plain(C, W, trees, reqs, arrivals):
    """The reference's usage: one blocking per-call evaluation per request (host
    buffers, copies inside the call), in arrival order, at each kernel's plain
    operating point."""
    outs = []
    lat = []
    t0 = time.perf_counter()
    for r, at in zip(reqs, arrivals):
        wait_until(t0, at)
        t = trees[r["tree"]]
        op = op_of(r, "plain")
        out = np.empty(r["nq"], np.float32)
        t[tree_key(op)].eval_host_ptr(r["q"].ctypes.data, r["nq"], out.ctypes.data,
                                      request_params(C, W, t, r, op))
        lat.append((time.perf_counter() - t0 - at) * 1e3)
        outs.append(out)
    return time.perf_counter() - t0, np.array(lat), outs


def drive_served(C, W, trees, reqs, server, ids, arrivals, role="served"):
    """Requests submitted to the server at their arrival times (host buffers)."""
    handles = [None] * len(reqs)
    lateness = np.zeros(len(reqs))

    def submitter():
        for k, (r, at) in enumerate(zip(reqs, arrivals)):
            wait_until(t0, at)
            lateness[k] = (time.perf_counter() - t0 - at) * 1e3
            t = trees[r["tree"]]
            op = op_of(r, role)
            handles[k] = server.submit(ids[(r["tree"], tree_key(op))], r["q"],
                                       request_params(C, W, t, r, op))

    t0 = time.perf_counter()
    th = threading.Thread(target=submitter)
    th.start()
    th.join()
    lat = []
    for k, h in enumerate(handles):
        h.wait()
        lat.append(h.info["latency_ms"] + lateness[k])
    return time.perf_counter() - t0, np.array(lat), [h.results for h in handles]


def serving_error(kernel, est, ref):
    """Relative error against FP64: gravity |e|/|ref|; winding number
    |e|/max(|ref|, 1); smooth distance the error of D = -log(S)/alpha, the
    distance the sum S stands for (a non-positive estimate of S counts as an
    infinite error)."""
    est = est.astype(np.float64)
    if kernel == "wn":
        return np.abs(est - ref) / np.maximum(np.abs(ref), 1.0)
    if kernel == "gravity":
        return np.abs(est - ref) / np.abs(ref)
    ok = ref > 0
    d_ref = -np.log(ref[ok]) / SERVING_ALPHA
    with np.errstate(divide="ignore", invalid="ignore"):
        d_est = np.where(est[ok] > 0, -np.log(np.maximum(est[ok], 1e-300)) / SERVING_ALPHA,
                         np.inf)
    return np.abs(d_est - d_ref) / np.abs(d_ref)


def serving_references(trees, reqs, per_kernel=30, n_max=1024, seed=5):
    """FP64 brute-force values (the oracle's GPU FP64 kernel) for the first
    n_max queries of `per_kernel` seeded requests of each kernel."""
    rng = np.random.default_rng(seed)
    pick = []
    for kern in SERVING_KERNELS:
        idx = [k for k, r in enumerate(reqs) if r["kernel"] == kern]
        pick += [int(k) for k in rng.permutation(idx)[:per_kernel]]
    refs = {}
    for k in pick:
        r = reqs[k]
        t = trees[r["tree"]]
        n = min(r["nq"], n_max)
        refs[k] = fp64_reference(t["pts"], t["nrm"], t["m"], r["kernel"],
                                 np.ascontiguousarray(r["q"][:n]),
                                 alpha=SERVING_ALPHA if r["kernel"] == "smooth" else 1.0)
    return refs


def median_errors(C, W, trees, reqs, refs, kernel, op):
    """(median, p99) error of an operating point over the picked requests of one
    kernel (blocking calls on the first queries of each)."""
    errs = []
    for k, ref in refs.items():
        r = reqs[k]
        if r["kernel"] != kernel:
            continue
        t = trees[r["tree"]]
        v, _ = t[tree_key(op)].eval(r["q"][:len(ref)], request_params(C, W, t, r, op))
        errs.append(serving_error(kernel, v, ref))
    e = np.concatenate(errs)
    return float(np.median(e)), float(np.percentile(e, 99))


def device_batch(C, W, torch, trees, reqs, role=None, op_for=None):
    """Batch entries for every request with its queries resident on the device,
    at its role's operating point (or op_for(r))."""
    entries, keep = [], []
    for r in reqs:
        t = trees[r["tree"]]
        op = op_for(r) if op_for else op_of(r, role)
        dq = torch.from_numpy(np.ascontiguousarray(r["q"].T)).cuda()
        out = torch.empty(r["nq"], dtype=torch.float32, device="cuda")
        entries.append((t[tree_key(op)], request_params(C, W, t, r, op), dq.data_ptr(),
                        r["nq"], out.data_ptr(), 0, 0))
        keep += [dq, out]
    return entries, keep


def batch_ms(C, torch, entries, repeats=3):
    """Event-timed median of sbh_eval_batch over the entries (one untimed run first)."""
    C.eval_batch(entries)
    torch.cuda.synchronize()
    ts = []
    for _ in range(repeats):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        C.eval_batch(entries)
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    return statistics.median(ts)


def serving_calibrate(C, W, torch, trees, reqs, refs):
    """The calibration ladders: per kernel, the median / p99 error and the
    batched throughput (all requests of the kernel, queries resident) of every
    Barnes-Hut theta, every stochastic budget factor and brute force; and the
    operating points chosen from them."""
    out = {}
    for kern in SERVING_KERNELS:
        sub = [r for r in reqs if r["kernel"] == kern]
        nq = sum(r["nq"] for r in sub)
        rows = []
        ops = ([("barnes_hut", th) for th in CAL_THETAS] +
               [("stochastic", sc) for sc in CAL_SCALES] + [("brute_force", None)])
        for op in ops:
            med, p99 = median_errors(C, W, trees, reqs, refs, kern, op)
            entries, keep = device_batch(C, W, torch, trees, sub, op_for=lambda r: op)
            ms = batch_ms(C, torch, entries, repeats=1 if op[0] == "brute_force" else 3)
            del entries, keep
            rows.append({"op": list(op), "median_rel_err": med, "p99_rel_err": p99,
                         "batched_queries_per_s": nq / (ms / 1e3)})
        meets = [x for x in rows if x["median_rel_err"] <= MATCH_TARGET]
        bh = [x for x in meets if x["op"][0] == "barnes_hut"]
        sb = [x for x in meets if x["op"][0] == "stochastic"]
        out[kern] = {
            "ladder": rows,
            "plain": max(bh, key=lambda x: x["op"][1])["op"] if bh else ["brute_force", None],
            "stochastic": min(x["op"][1] for x in sb) if sb else None,
            "served": max(meets, key=lambda x: x["batched_queries_per_s"])["op"] if meets else None,
        }
    return out


def run_serving_replicas(args, world, rank, local):
    """Serving under torchrun: replicas only (the path has no exchange step).
    Every rank holds its own copy of the 64 trees on its own GPU and serves the
    same request stream; `value` is the device-resident batch and `e2e` the
    server at saturation, each as all ranks' queries over the slowest rank's
    time.  The plain path, the latency sweep and the CPU baseline are the
    single-GPU line's."""
    import datetime

    import torch
    import torch.distributed as dist

    import sbh_capi as C
    import sbh_workloads as W
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    trees, reqs = serving_setup(C, device=local)
    total_q = sum(r["nq"] for r in reqs)
    entries, keep = device_batch(C, W, torch, trees, reqs, "served")
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    dist.barrier()
    with ClockSampler(local) as clocks:
        dev_ms = sum(timed_device(lambda: C.eval_batch(entries, stream=stream.cuda_stream),
                                  stream, flush, args.warmup, args.steps))
    del entries, keep
    server = C.Server(device=local, slots=3, slot_queries=SERVER_SLOT_QUERIES,
                      max_requests_per_batch=4096)
    ids = {}
    for i, t in enumerate(trees):
        ids[(i, "sbh")] = server.add_tree(t["sbh"])
        ids[(i, "bh")] = server.add_tree(t["bh"])
    drive_served(C, W, trees, reqs[:50], server, ids, np.zeros(50))
    dist.barrier()
    served_s, _, _ = drive_served(C, W, trees, reqs, server, ids, np.zeros(len(reqs)))
    server.close()
    dev_ms, served_ms = max_over_ranks([dev_ms, served_s * 1e3], dist, dev)
    dist.destroy_process_group()
    if rank != 0:
        return None
    return {
        "metric": METRIC, "value": whole_job_rate(world, total_q, dev_ms, args.steps),
        "unit": "queries/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dev_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded generators; the reference publishes no dataset)",
        "config": dict(serving_config(len(reqs), total_q), parallelism=f"replicas x{world}"),
        "e2e": {"value": world * total_q / (served_ms / 1e3), "unit": "queries/s",
                "h2d_bytes_per_step": world * sum(r["nq"] * 4 * trees[r["tree"]]["dim"]
                                                  for r in reqs),
                "d2h_bytes_per_step": world * total_q * 4, "ms_per_step": served_ms,
                "path": "every rank's server (C ABI, host buffers), the stream submitted at "
                        "t = 0; slowest rank"},
        "clocks": clocks.summary(),
        "gpu_launches": args.steps * 9,
    }


def run_serving(args):
    import torch

    import sbh_capi as C
    import sbh_workloads as W
    world, rank, local = dist_setup()
    if world > 1 and not args.calibrate:
        return run_serving_replicas(args, world, rank, local)
    t_setup = time.perf_counter()
    trees, reqs = serving_setup(C)
    if args.calibrate:
        refs = serving_references(trees, reqs, per_kernel=50)
        return {"calibration": serving_calibrate(C, W, torch, trees, reqs, refs),
                "target": MATCH_TARGET, "requests_per_kernel": 50,
                "reference": "FP64 brute force on the GPU, first 1,024 queries per request"}
    refs = serving_references(trees, reqs)
    total_q = sum(r["nq"] for r in reqs)

    # Accuracy at the matched operating points, and of stochastic BH at the
    # requests' own budgets for comparison.
    acc = {}
    for kern in SERVING_KERNELS:
        m = MATCHED[kern]
        row = {}
        for role in ("plain", "served", "served_stochastic"):
            op = op_of({"kernel": kern}, role)
            med, p99 = median_errors(C, W, trees, reqs, refs, kern, op)
            row[role] = {"op": list(op), "median_rel_err": med, "p99_rel_err": p99}
        med, p99 = median_errors(C, W, trees, reqs, refs, kern, ("stochastic", 1.0))
        row["stochastic_at_drawn_budgets"] = {"median_rel_err": med, "p99_rel_err": p99}
        row["stochastic_meets_target"] = m["stochastic"] is not None
        acc[kern] = row
    matched = all(max(a[r]["median_rel_err"] for r in ("plain", "served", "served_stochastic"))
                  <= MATCH_TARGET for a in acc.values())

    # Batch schedule for the served path, autotuned on the first 256 requests (untimed).
    entries, keep = device_batch(C, W, torch, trees, reqs[:256], "served")
    tuning, best_ms, start_ms = C.batch_autotune(entries, stream=0, repeats=2)
    torch.cuda.synchronize()
    del entries, keep

    # value: the whole request stream as one batched evaluation with every
    # request's queries resident in HBM, at the served operating points.
    n_direct = sum(1 for r in reqs if op_of(r, "served")[0] == "stochastic" and
                   tuning.direct_queries > 0 and r["nq"] >= tuning.direct_queries)
    entries, keep = device_batch(C, W, torch, trees, reqs, "served")
    stream = torch.cuda.current_stream()
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    with ClockSampler(0) as clocks:
        dev_ms = timed_device(lambda: C.eval_batch(entries, stream=stream.cuda_stream), stream,
                              flush, args.warmup, args.steps)
    del entries, keep
    dev_total_ms = float(sum(dev_ms))
    breakdown, roofline = serving_breakdown(C, W, torch, trees, reqs, stream, flush)
    entries, keep = device_batch(C, W, torch, trees, reqs, "served_stochastic")
    dev_sbh_ms = statistics.mean(timed_device(
        lambda: C.eval_batch(entries, stream=stream.cuda_stream), stream, flush, 1,
        max(2, args.steps // 4)))
    del entries, keep

    server = C.Server(slots=3, slot_queries=SERVER_SLOT_QUERIES, max_requests_per_batch=4096,
                      tuning=tuning)
    ids = {}
    for i, t in enumerate(trees):
        ids[(i, "sbh")] = server.add_tree(t["sbh"])
        ids[(i, "bh")] = server.add_tree(t["bh"])
    setup_s = time.perf_counter() - t_setup
    # Warm-up of every path on a slice of the stream.
    warm = reqs[:50]
    drive_plain(C, W, trees, warm, np.zeros(len(warm)))
    drive_served(C, W, trees, warm, server, ids, np.zeros(len(warm)))
    # Plain per-call capacity: every request queued at t = 0 (the first pass also
    # grows every tree's cached workspace to its largest request).
    drive_plain(C, W, trees, reqs, np.zeros(len(reqs)))
    plain_mk, plain_lat, _ = drive_plain(C, W, trees, reqs, np.zeros(len(reqs)))
    plain_rps = len(reqs) / plain_mk
    # Served capacity (e2e): the same stream submitted at t = 0, host buffers.
    served_mk, served_lat, _ = drive_served(C, W, trees, reqs, server, ids, np.zeros(len(reqs)))
    sbh_mk, sbh_lat, _ = drive_served(C, W, trees, reqs, server, ids, np.zeros(len(reqs)),
                                      role="served_stochastic")
    rates = {}
    rng = np.random.default_rng(5)
    for factor in (0.5, 1.0, 2.0):
        rate = factor * plain_rps
        gaps = rng.exponential(1.0 / rate, len(reqs))
        arrivals = np.cumsum(gaps) - gaps[0]
        row = {"arrival_rate_rps": rate}
        for name, fn in (("plain", lambda: drive_plain(C, W, trees, reqs, arrivals)),
                         ("served", lambda: drive_served(C, W, trees, reqs, server, ids,
                                                         arrivals))):
            mk, lat, _ = fn()
            row[name] = {"queries_per_s": total_q / mk, "p50_ms": float(np.percentile(lat, 50)),
                         "p99_ms": float(np.percentile(lat, 99)), "makespan_s": mk}
        rates[f"rate_x{factor}"] = row
    stats = server.stats()
    server.close()
    served_qps = total_q / served_mk
    plain_qps = total_q / plain_mk
    cpu = None
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        if O.ref_available():
            cq, cs, cn, _ = reference_serving_sample(trees, reqs, args.cpu_seconds)
            cores = O.ref_hardware_concurrency()
            cpu = {"value": cq / cs, "unit": "queries/s", "cores": cores, "kind": "reference",
                   "sample": f"the first {cn} requests of the stream ({int(cq)} queries, at most "
                             f"{REF_QUERIES_PER_REQUEST} per request), src/sbh.cpp evalBarnesHut "
                             f"at each kernel's plain operating point (beta = inf for exact), "
                             f"its thread pool ({cores} threads), {cs:.1f} s"}
    return {
        "metric": METRIC, "value": total_q / (dev_total_ms / args.steps / 1e3),
        "unit": "queries/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dev_total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded generators; the reference publishes no dataset)",
        "config": serving_config(len(reqs), total_q),
        "e2e": {"value": served_qps, "unit": "queries/s",
                "h2d_bytes_per_step": sum(r["nq"] * 4 * trees[r["tree"]]["dim"] for r in reqs),
                "d2h_bytes_per_step": total_q * 4, "ms_per_step": served_mk * 1e3,
                "path": "sbh_server_submit / sbh_server_wait (C ABI) with host buffers, every "
                        "request of the stream submitted at t = 0",
                "p50_ms": float(np.percentile(served_lat, 50)),
                "p99_ms": float(np.percentile(served_lat, 99))},
        "served_over_plain": served_qps / plain_qps,
        "plain": {"queries_per_s": plain_qps, "requests_per_s": plain_rps,
                  "p50_ms": float(np.percentile(plain_lat, 50)),
                  "p99_ms": float(np.percentile(plain_lat, 99)),
                  "path": "one blocking sbh_eval per request (host buffers) at each kernel's "
                          "plain operating point"},
        "served_stochastic": {
            "what": "the server with stochastic BH wherever it meets the target (gravity at the "
                    "drawn budgets x MATCHED factor), the served points elsewhere",
            "queries_per_s": total_q / sbh_mk, "over_plain": (total_q / sbh_mk) / plain_qps,
            "p50_ms": float(np.percentile(sbh_lat, 50)),
            "p99_ms": float(np.percentile(sbh_lat, 99)),
            "device_batch_queries_per_s": total_q / (dev_sbh_ms / 1e3)},
        "matched": {"target_median_rel_err": MATCH_TARGET, "all_within_target": matched,
                    "operating_points": MATCHED, "accuracy": acc,
                    "reference": "FP64 brute force on the GPU (the oracle's libsbh_bf64.so), "
                                 "first 1,024 queries of 30 seeded requests per kernel"},
        "latency_at_rates": rates,
        "breakdown": breakdown, "roofline": roofline,
        "server_stats": stats, "clocks": clocks.summary(),
        "autotune": {"tuning": tuning.as_dict(), "tuned_ms": best_ms, "default_ms": start_ms},
        "setup_s": setup_s,
        "cpu_baseline": cpu,
        # per batch step: the graph's 9 kernels (query boxes, keys, three scan
        # kernels, scatter, one persistent kernel per method class) plus 8 (sort
        # and sampler) per stochastic request sent to its own launch
        "gpu_launches": args.steps * (9 + 8 * n_direct),
    }


def serving_breakdown(C, W, torch, trees, reqs, stream, flush):
    """Each kernel's requests batched alone at their served operating points
    (device-resident, CUDA events): where the served batch's time goes, and the
    roofline of the largest part.  A part whose served point is brute force is
    bound by its arithmetic pipes: its pairs per second against pair_pipe_bound;
    a traversal part is issue-bound and reported in queries/s."""
    parts = {}
    for kern in SERVING_KERNELS:
        sub = [r for r in reqs if r["kernel"] == kern]
        entries, keep = device_batch(C, W, torch, trees, sub, "served")
        ms = statistics.mean(timed_device(lambda: C.eval_batch(entries, stream=stream.cuda_stream),
                                          stream, flush, 2, 3))
        del entries, keep
        op = MATCHED[kern]["served"]
        parts[kern] = {"op": list(op), "ms": ms, "queries": sum(r["nq"] for r in sub),
                       "pairs": sum(r["nq"] * trees[r["tree"]]["n"] for r in sub)}
    top = max(parts, key=lambda k: parts[k]["ms"])
    p = parts[top]
    if p["op"][0] == "brute_force":
        rates = C.measure_pipe_rates(0)
        peak, mufu_per_pair, fp32_per_pair = pair_pipe_bound(rates, top)
        achieved = p["pairs"] / (p["ms"] / 1e3)
        roof = {"bound": "sfu", "kernel": "batch_eval_kernel (brute-force class), " + top,
                "achieved": achieved, "peak": peak, "unit": "pairs/s", "frac": achieved / peak,
                "peak_source": "measured MUFU rsqrt rate (sbh_measure_pipe_rates) / "
                               f"{mufu_per_pair} MUFU ops per pair (3D operation counts; "
                               f"{fp32_per_pair} FP32 lane ops against the measured FFMA rate "
                               f"bind less): {rates['rsqrt_per_clk_sm']:.2f}/clk/SM at "
                               f"{rates['sm_clock_mhz']:.0f} MHz",
                "kernel_ms": p["ms"], "pairs_per_launch": p["pairs"],
                "traffic": DRAM_TRAFFIC.get("served_smooth") if top == "smooth" else None,
                "note": f"the {top} requests batched alone; share of the summed parts "
                        f"{p['ms'] / sum(x['ms'] for x in parts.values()):.2f}"}
    else:
        roof = {"bound": "issue", "kernel": "batch_eval_kernel, " + top,
                "achieved": p["queries"] / (p["ms"] / 1e3), "peak": None, "unit": "queries/s",
                "frac": None, "kernel_ms": p["ms"], "traffic": None}
    return parts, roof


def serving_config(n_requests, total_q):
    return {"workload": "serving: 32 resident trees (16 3D, 16 2D; Gaussian mixtures, torus, "
                        "sphere and circle surfaces; 1e4..2e6 points), 1500 seeded requests, "
                        "gravity / winding number / smooth distance (alpha 100), 1..1e5 "
                        "queries log-uniform, budgets 64/256/1024; served (continuous batching) "
                        "vs plain per-call evaluation, both at each kernel's operating point of "
                        "median relative error <= 1e-3 vs FP64",
            "operating_points": {k: {"plain": list(v["plain"]), "served": list(v["served"]),
                                     "stochastic_budget_factor": v["stochastic"]}
                                 for k, v in MATCHED.items()},
            "requests": n_requests, "queries": total_q,
            "server": {"slots": 3, "slot_queries": SERVER_SLOT_QUERIES},
            "l2": "512 MiB buffer written between timed batch steps"}


REF_QUERIES_PER_REQUEST = 2048


def reference_serving_sample(trees, reqs, budget_s, start=0, ref_trees=None):
    """The reference's CPU plugin (src/sbh.cpp evalBarnesHut, compiled unmodified
    in oracle/_ref, its own thread pool) on consecutive requests of the stream
    from `start`, each at its kernel's plain operating point (Barnes-Hut at the
    matched theta, or beta = inf -- the reference's own exact evaluation,
    python/example.py:76-82 -- where the plain point is exact), until
    `budget_s` seconds of evaluation: (queries, seconds, requests, next start).
    A request's first REF_QUERIES_PER_REQUEST queries stand for it (per-query
    work is independent).  Reference trees (Octree1 / Quadtree1, alpha 100) are
    built on first use; builds are not timed."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    ref_trees = {} if ref_trees is None else ref_trees
    nq = secs = 0.0
    done = 0
    k = start
    while secs < budget_s and done < len(reqs):
        r = reqs[k % len(reqs)]
        t = trees[r["tree"]]
        if r["tree"] not in ref_trees:
            ref_trees[r["tree"]] = O.RefTree(t["pts"], t["nrm"], t["m"], t["lo"], t["hi"],
                                             alpha=SERVING_ALPHA, dim_split_log=1)
        method, theta = MATCHED[r["kernel"]]["plain"]
        beta = 1.0 / theta if method == "barnes_hut" else np.inf
        q = np.ascontiguousarray(r["q"][:REF_QUERIES_PER_REQUEST])
        _, s = ref_trees[r["tree"]].plugin_bh(SERVING_KID[r["kernel"]], q, beta)
        nq += len(q)
        secs += s
        done += 1
        k += 1
    return nq, secs, done, k


def run_reference_serving(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not O.ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libsbh_ref.so is not built"}
    trees, reqs = serving_setup(None, device_trees=False)
    ref_trees = {}
    k = 0
    for _ in range(args.warmup):
        _, _, _, k = reference_serving_sample(trees, reqs, 0.2, k, ref_trees)
    tq = ts = 0.0
    nreq = 0
    for _ in range(args.steps):
        q, s, n, k = reference_serving_sample(trees, reqs, args.ref_step_seconds, k, ref_trees)
        tq += q
        ts += s
        nreq += n
    value = tq / ts
    cores = O.ref_hardware_concurrency()
    sample = (f"{nreq} consecutive requests of the 1500-request stream ({int(tq)} queries, at "
              f"most {REF_QUERIES_PER_REQUEST} per request), src/sbh.cpp evalBarnesHut per request "
              f"at each kernel's plain operating point (beta = inf where it is exact), its thread "
              f"pool ({cores} threads); tree builds excluded")
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "queries/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ts / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded generators; the reference publishes no dataset)",
        "config": serving_config(len(reqs), sum(r["nq"] for r in reqs)),
        "cpu_baseline": {"value": value, "unit": "queries/s", "cores": cores,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


# ------------------------------------------------- served smooth distance

def run_served_smooth(args):
    """The serving stream's smooth-distance requests (alpha 100) at their served
    operating point, exact summation, as one device-resident batch: the largest
    part of the served batch, where the batched brute-force class kernel runs
    alone.  `--requests N` keeps the first N of them (a small case for
    profiling); only the trees they name are built (host build + upload)."""
    import torch

    import sbh_capi as C
    import sbh_workloads as W
    trees, reqs = serving_setup(C, device_trees=False)
    sub = [r for r in reqs if r["kernel"] == "smooth"]
    if args.requests > 0:
        sub = sub[:args.requests]
    for ti in sorted({r["tree"] for r in sub}):
        t = trees[ti]
        t["bh"] = C.GpuTree(C.HostTree(t["pts"], t["nrm"], t["m"], t["lo"], t["hi"],
                                       dim_split_log=1))
    entries, keep = device_batch(C, W, torch, trees, sub, "served")
    stream = torch.cuda.current_stream()
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    with ClockSampler(0) as clocks:
        ms = timed_device(lambda: C.eval_batch(entries, stream=stream.cuda_stream), stream, flush,
                          args.warmup, args.steps)
    kms = statistics.mean(ms)
    pairs = float(sum(r["nq"] * trees[r["tree"]]["n"] for r in sub))
    pairs3 = float(sum(r["nq"] * trees[r["tree"]]["n"] for r in sub if trees[r["tree"]]["dim"] == 3))
    rates = C.measure_pipe_rates(0)
    peak = (pairs3 / pair_pipe_bound(rates, "smooth", 3)[0] +
            (pairs - pairs3) / pair_pipe_bound(rates, "smooth", 2)[0])
    peak = pairs / peak
    achieved = pairs / (kms / 1e3)
    nq = sum(r["nq"] for r in sub)
    return {
        "metric": "batched brute-force smooth-distance pairs/s (the serving stream's smooth "
                  "requests, exact summation)",
        "value": achieved, "unit": "pairs/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": kms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generators)",
        "config": {"workload": f"served smooth distance: {len(sub)} requests of the serving "
                               f"stream (alpha 100, {nq} queries, {pairs:.3e} pairs) as one "
                               "sbh_eval_batch, queries resident, L2 flushed between steps"},
        "queries_per_s": nq / (kms / 1e3),
        "roofline": {"bound": "sfu", "kernel": "batch_eval_kernel (brute-force class)",
                     "achieved": achieved, "peak": peak, "unit": "pairs/s",
                     "frac": achieved / peak,
                     "peak_source": "pair_pipe_bound per request dimension: measured MUFU rate "
                                    f"{rates['rsqrt_per_clk_sm']:.2f}/clk/SM at "
                                    f"{rates['sm_clock_mhz']:.0f} MHz, 1.75 MUFU ops per pair",
                     "traffic": None if args.requests else DRAM_TRAFFIC.get("served_smooth")},
        "clocks": clocks.summary(),
        "gpu_launches": args.steps * 9,
    }


# ---------------------------------------------------------------- batching

def run_batching(args):
    import torch

    import sbh_capi as C
    import sbh_workloads as W
    rng = np.random.default_rng(44)
    probs = []
    for i in range(256):
        n = int(np.exp(rng.uniform(np.log(1024), np.log(1 << 20))))
        pts, nrm, m = W.gaussian_mixture(n, seed=1000 + i)
        lo, hi = W.padded_box(pts)
        host = C.HostTree(pts, nrm, m, lo, hi, dim_split_log=2)
        gpu = C.GpuTree(host)
        budget = int(rng.choice([64, 128, 256, 512]))
        samples = W.samples_for_budget(budget, gpu.info.root_children)
        dq = torch.from_numpy(np.ascontiguousarray(pts.T)).cuda()
        dm = torch.from_numpy(m).cuda()
        out = torch.empty(n, dtype=torch.float32, device="cuda")
        p = C.params(method=C.STOCHASTIC, kernel=C.GRAVITY, samples_per_subdomain=samples, seed=i)
        probs.append(dict(host=host, gpu=gpu, dq=dq, dm=dm, out=out, n=n, p=p))
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    entries = [(b["gpu"], b["p"], b["dq"].data_ptr(), b["n"], b["out"].data_ptr(), 0,
                b["dm"].data_ptr()) for b in probs]
    total_q = sum(b["n"] for b in probs)
    self_t = [(-b["dm"] / 0.1) for b in probs]

    def batched():
        C.eval_batch(entries, stream=sh)

    def sequential():
        for b, st in zip(probs, self_t):
            b["gpu"].eval_device(b["dq"].data_ptr(), b["n"], b["out"].data_ptr(), b["p"], stream=sh)
            b["out"].sub_(st)

    res = {}
    # The autotuner picks the batch schedule (CTAs per SM, sampler unit size,
    # bucket size) on this batch, untimed; the timed runs use its choice.
    default_tuning = C.get_batch_tuning()
    best, best_ms, start_ms = C.batch_autotune(entries, stream=sh, repeats=2)
    res["autotune"] = {"tuning": best.as_dict(), "tuned_ms": best_ms, "default_ms": start_ms,
                       "default_tuning": default_tuning.as_dict()}
    clocks = None
    for name, fn in (("one_batch_launch", batched), ("sequential_plain_calls", sequential)):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        ts = []
        sampler = ClockSampler(0)
        sampler.__enter__()
        for _ in range(max(1, args.steps // 4)):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        sampler.__exit__(None, None, None)
        clocks = clocks or sampler.summary()
        ms = statistics.mean(ts)
        res[name] = {"ms": ms, "queries_per_s": total_q / (ms / 1e3), "problems_per_s": 256 / (ms / 1e3)}
    return {
        "metric": METRIC, "value": res["one_batch_launch"]["queries_per_s"], "unit": "queries/s",
        "n_gpus": 1, "steps": max(1, args.steps // 4), "warmup": args.warmup,
        "ms_per_step": res["one_batch_launch"]["ms"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generators)",
        "config": {"workload": "batching: 256 3D gravity problems, 1,024..1,048,576 sources "
                               "log-uniform, queries = sources (self term excluded), stochastic "
                               "BH budget 64-512, Octree2", "queries": total_q},
        "batching": res, "clocks": clocks,
        "gpu_launches": 4 * max(1, args.steps // 4),
    }


# ---------------------------------------------------------- differentiation

def run_differentiation(args):
    """Smooth distance (alpha 100, max-shifted) forward and backward through the
    autograd wrapper: stochastic BH (budget 128, Octree2/Quadtree2) and
    deterministic BH (theta 0.5, Octree1/Quadtree1), 3D torus and 2D circle."""
    import torch

    import sbh_capi as C
    import sbh_torch
    import sbh_workloads as W
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    cases = []
    pts3, nrm3, a3 = W.torus_surface(524288, seed=301, jitter=1e-3)
    q3 = W.uniform_queries(1 << 20, seed=302, dim=3, lo=-1.0, hi=1.0)
    pts2, nrm2, a2 = W.circle_points(262144, seed=303, jitter=1e-3)
    q2 = W.uniform_queries(1 << 20, seed=304, dim=2, lo=-1.5, hi=1.5)
    for dim, pts, nrm, a, q in ((3, pts3, nrm3, a3, q3), (2, pts2, nrm2, a2, q2)):
        lo, hi = W.padded_box(pts)
        trees = {dsl: C.GpuTree(C.HostTree(pts, nrm, a, lo, hi, alpha=100.0, dim_split_log=dsl))
                 for dsl in (1, 2)}
        cases.append((dim, trees, q))
    res = {}
    total_q = 0
    total_ms = {"stochastic": 0.0, "barnes_hut": 0.0}
    clocks = None
    for dim, trees, q in cases:
        nq = q.shape[0]
        total_q += nq
        tq = torch.from_numpy(q).to(dev).requires_grad_(True)
        gout = torch.ones(nq, dtype=torch.float32, device=dev)
        sub = q[:4096]
        ref_v, ref_g, _ = trees[1].eval_grad(sub, C.params(method=C.BRUTE_FORCE,
                                                            kernel=C.SMOOTH_DIST))
        for method, tree, kw in (("stochastic", trees[2], {"budget": 128, "seed": 7}),
                                 ("barnes_hut", trees[1], {"beta": 2.0})):
            def step():
                tq.grad = None
                d = sbh_torch.smooth_distance(tree, tq, method=method, **kw)
                d.backward(gout)
                return d

            for _ in range(args.warmup):
                flush.zero_()
                step()
            tree.check(stream.cuda_stream)
            torch.cuda.synchronize(dev)
            ev = []
            with ClockSampler(0) as cs:
                for _ in range(args.steps):
                    flush.zero_()
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    step()
                    e1.record(stream)
                    ev.append((e0, e1))
                torch.cuda.synchronize(dev)
            clocks = cs.summary() if clocks is None else clocks
            tree.check(stream.cuda_stream)
            ms = statistics.mean(a.elapsed_time(b) for a, b in ev)
            total_ms[method] += ms
            # accuracy on the first 4096 queries against compensated brute force
            p = C.params(method={"stochastic": C.STOCHASTIC, "barnes_hut": C.BARNES_HUT}[method],
                         kernel=C.SMOOTH_DIST, beta=kw.get("beta", 2.0), seed=7,
                         samples_per_subdomain=W.samples_for_budget(
                             128, tree.info.root_children))
            v, g, _ = tree.eval_grad(sub, p)
            ok = np.isfinite(v)
            d_err = np.abs(v[ok] - ref_v[ok]) / np.maximum(np.abs(ref_v[ok]), 1e-30)
            g_err = (np.linalg.norm(g[ok] - ref_g[ok], axis=1) /
                     np.maximum(np.linalg.norm(ref_g[ok], axis=1), 1e-30))
            res[f"{dim}d_{method}"] = {
                "fwd_bwd_ms": ms, "queries_per_s": nq / (ms / 1e3),
                "median_rel_err_D": float(np.median(d_err)),
                "median_rel_err_grad": float(np.median(g_err)),
                "nonfinite_frac": float(1.0 - ok.mean()),
                "samples_per_subdomain": int(p.samples_per_subdomain) if method == "stochastic"
                else None}
    value = total_q / (total_ms["stochastic"] / 1e3)
    return {
        "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms["stochastic"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generators)",
        "config": {"workload": "differentiation: smooth distance alpha 100 (max-shifted), forward "
                               "+ backward through torch.autograd; 3D torus 524,288 points "
                               "(jitter 1e-3), 2D circle 262,144 points, 1,048,576 queries each; "
                               "stochastic BH budget 128 (value) and BH theta 0.5",
                   "l2": "flushed between steps (512 MiB write)",
                   "accuracy_reference": "compensated FP32 brute force on the GPU, 4096 queries"},
        "differentiation": res, "clocks": clocks,
        "gpu_launches": 6,
    }


# -------------------------------------------------------------- tree build

def run_tree_build(args):
    """Tree construction, 1,048,576 torus points, Octree2 and Octree1 (leaf 1):
    the GPU build (sbh_gpu_tree_build) against the host build + upload and the
    reference's own build (src/sbh.cpp's Octree constructors, compiled in
    oracle/_ref), all producing the same tree."""
    import torch

    import sbh_capi as C
    import sbh_workloads as W
    pts, nrm, a = W.torus_surface(1 << 20, seed=2024)
    lo, hi = W.padded_box(pts)
    res = {}
    for dsl in (2, 1):
        C.GpuTree.build(pts[:4096], nrm[:4096], a[:4096], lo, hi, dim_split_log=dsl)  # warm-up
        gpu_s = []
        for _ in range(max(3, args.steps // 4)):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            g = C.GpuTree.build(pts, nrm, a, lo, hi, dim_split_log=dsl)
            torch.cuda.synchronize()
            gpu_s.append(time.perf_counter() - t0)
            assert g.built_on_device
            del g
        t0 = time.perf_counter()
        h = C.HostTree(pts, nrm, a, lo, hi, dim_split_log=dsl)
        t1 = time.perf_counter()
        g = C.GpuTree(h)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        res[f"octree{dsl}"] = {"gpu_build_s": statistics.median(gpu_s), "host_build_s": t1 - t0,
                               "upload_s": t2 - t1, "nodes": g.info.num_nodes}
    ref = None
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        if O.ref_available():
            t0 = time.perf_counter()
            O.RefTree(pts, nrm, a, lo, hi, dim_split_log=2)
            ref = time.perf_counter() - t0
    v = res["octree2"]
    return {
        "metric": "tree build points/s", "value": (1 << 20) / v["gpu_build_s"],
        "unit": "points/s", "n_gpus": 1, "steps": max(3, args.steps // 4), "warmup": 1,
        "ms_per_step": v["gpu_build_s"] * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generators)",
        "config": {"workload": "tree build: 1,048,576 torus points, leaf size 1; wall clock "
                               "from host arrays to a device-resident tree"},
        "tree_build": res,
        "cpu_baseline": None if ref is None else {
            "value": (1 << 20) / ref, "unit": "points/s", "cores": 1, "kind": "reference",
            "sample": "the reference's Octree2 constructor on the same 1,048,576 points "
                      "(single-threaded, as the reference builds)"},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload",
                    choices=sorted(WORKLOADS) + ["serving", "batching", "differentiation",
                                                 "tree_build", "served_smooth"],
                    default="serving")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--ref-sample", type=int, default=4096)
    ap.add_argument("--ref-step-seconds", type=float, default=4.0)
    ap.add_argument("--nq", type=int, default=0, help="override the query count (profiling)")
    ap.add_argument("--requests", type=int, default=0,
                    help="served_smooth: keep the first N smooth-distance requests (profiling)")
    ap.add_argument("--budget", type=int, default=0,
                    help="override the sampled paths per query of a stochastic workload")
    ap.add_argument("--stage-leaves", action="store_true",
                    help="Barnes-Hut workloads: copy accepted leaves' points to shared memory "
                         "with bulk asynchronous copies (SBH_FLAG_STAGE_LEAVES)")
    ap.add_argument("--calibrate", action="store_true",
                    help="serving: print the accuracy ladders the matched operating points "
                         "are chosen from, instead of timing")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    systems = {"serving": run_serving, "batching": run_batching,
               "differentiation": run_differentiation, "tree_build": run_tree_build,
               "served_smooth": run_served_smooth}
    if args.workload in systems and args.impl == "ours":
        out = systems[args.workload](args)
        if out is not None:
            print(json.dumps(out), flush=True)
        return
    if args.workload == "serving":
        out = run_reference_serving(args)
        if out is not None:
            print(json.dumps(out), flush=True)
        return
    if args.workload in systems:
        ap.error("--impl reference runs the serving and single-configuration workloads only")
    wl = dict(WORKLOADS[args.workload])
    wl["name"] = args.workload
    wl["resized"] = bool(args.nq or args.budget)
    if args.nq:
        wl["nq"] = args.nq
        wl["desc"] += f" [query count overridden: {args.nq}]"
    if args.budget and wl["method"] == "stochastic":
        wl["budget"] = args.budget
        wl["desc"] += f" [budget overridden: {args.budget} paths/query]"
    out = run_reference(args, wl) if args.impl == "reference" else run_ours(args, wl)
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
