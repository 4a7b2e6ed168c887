"""bench.py's host logic on the CPU: the multi-process path (gloo, world size 2)
and the clock sampler.

The timed path shards by replica (every rank evaluates its own query batch
against its own copy of the tree; no data-path collective), so the host logic
under test is the job-time reduction (maximum over ranks), the whole-job rate,
and the launch contract of the reference arm (rank 0 prints the only line).
"""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT

sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    # rank 0 is slower in the first value, rank 1 in the second
    mine = [100.0 + 50.0 * (rank == 0), 7.0 + 3.0 * (rank == 1)]
    got = bench.max_over_ranks(mine, dist, "cpu")
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, got))


def test_max_over_ranks_with_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0] == res[1] == [150.0, 10.0]


def test_whole_job_rate_and_single_process():
    assert bench.max_over_ranks([1.5, 2.0], None, "cpu") == [1.5, 2.0]
    # 2 ranks x 1000 queries, 4 steps in 8 ms (slowest rank): 2000 / 2 ms
    assert bench.whole_job_rate(2, 1000, 8.0, 4) == pytest.approx(1e6)


def test_reference_arm_under_two_ranks():
    """Launched as the driver launches it (torch.distributed.run, 2 processes):
    rank 0 times the reference's CPU path and prints one JSON line; rank 1
    exits 0 without output."""
    import oracle as O
    if not O.ref_available():
        pytest.skip("reference build (oracle/_ref) absent")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "plain_small_bh",
           "--steps", "1", "--warmup", "3", "--ref-sample", "64", "--ref-step-seconds", "0.05"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [line for line in r.stdout.splitlines() if line.startswith("{")]
    assert len(lines) == 1
    out = json.loads(lines[0])
    assert out["impl"] == "reference" and out["n_gpus"] == 2 and out["value"] > 0
    assert out["cpu_baseline"]["kind"] == "reference"


def test_clock_sampler_reads_nvml_by_pci_match(monkeypatch):
    """The sampler finds the CUDA device's NVML handle by PCI numbers, polls
    clocks and reasons, and reports the median clock and every active reason."""
    import time
    import types

    import torch

    calls = []
    fake = types.ModuleType("pynvml")
    fake.NVML_CLOCK_SM = 1
    for i, (name, attr) in enumerate(bench.ClockSampler.REASONS):
        setattr(fake, attr, 1 << (i + 1))

    class Pci:
        def __init__(self, d, b, v):
            self.domain, self.bus, self.device = d, b, v

    devices = [Pci(0, 0x1B, 0), Pci(0, 0x2C, 0)]
    fake.nvmlInit = lambda: None
    fake.nvmlDeviceGetCount = lambda: len(devices)
    fake.nvmlDeviceGetHandleByIndex = lambda i: ("handle", i)
    fake.nvmlDeviceGetPciInfo = lambda h: devices[h[1]]

    def clock(h, kind):
        calls.append(h)
        return 1800 if h[1] == 1 else 0

    fake.nvmlDeviceGetClockInfo = clock
    fake.nvmlDeviceGetMaxClockInfo = lambda h, kind: 1965
    fake.nvmlDeviceGetCurrentClocksEventReasons = lambda h: fake.nvmlClocksEventReasonSwPowerCap
    monkeypatch.setitem(sys.modules, "pynvml", fake)
    props = types.SimpleNamespace(pci_domain_id=0, pci_bus_id=0x2C, pci_device_id=0)
    monkeypatch.setattr(torch.cuda, "get_device_properties", lambda i: props)
    with bench.ClockSampler(0) as s:
        time.sleep(0.05)
    out = s.summary()
    assert out["samples"] > 3 and out["sm_mhz"] == 1800 and out["sm_max_mhz"] == 1965
    assert out["reasons"] == ["sw_power_cap"]
    assert all(h == ("handle", 1) for h in calls)
