"""The N > 1 path of bench.py on CPU: two gloo ranks (no GPU).

Each rank searches its own instance of the workload (seeds offset by rank, no collective
in the data path, "weak" scaling); the job time is the max over ranks and the job
throughput counts every rank's queries. Here each rank runs the oracle's grid search in
place of the CUDA search, so the host-side logic is exercised end to end.
"""
import os
import socket
import time

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    import datetime
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import torch
    import torch.distributed as dist
    import bench
    import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        cfg = bench.make_workload("radius_uniform_1e5", 0.05, rank)
        t0 = time.perf_counter()
        rows = oracle.grid_search_batched(cfg["points"], cfg["offsets"], mode=cfg["mode"],
                                          r=cfg["radius"], k=cfg["k"], threads=1)
        ms = (time.perf_counter() - t0) * 1e3 + 10.0 * rank   # rank 1 is the slower one
        ms_max = bench.reduce_max(ms, dist)
        sig = torch.tensor([float(np.asarray(cfg["points"], np.float64).sum()), float(cfg["n_queries"])],
                           dtype=torch.float64)
        gathered = [torch.zeros_like(sig) for _ in range(world)]
        dist.all_gather(gathered, sig)
        q.put((rank, ms, ms_max, [g.tolist() for g in gathered], int((rows >= 0).sum()),
               bench.job_throughput(cfg["n_queries"], world, ms_max)))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks_weak_scaling():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        r = q.get(timeout=300)
        res[r[0]] = r
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, ms0, max0, g0, hits0, thr0), (_, ms1, max1, g1, hits1, thr1) = res[0], res[1]
    # every rank sees the same job time: the slowest rank's
    assert max0 == max1 == pytest.approx(max(ms0, ms1))
    # the ranks searched different instances (independent seeds) of the same shape
    assert g0 == g1 and g0[0][0] != g0[1][0]
    assert hits0 > 0 and hits1 > 0
    # whole-job throughput counts both ranks' queries
    assert thr0 == pytest.approx(2 * g0[0][1] / (max0 * 1e-3))


@pytest.mark.gpu
def test_bench_two_ranks_run_the_cuda_path(tmp_path):
    """bench.py under torchrun with two ranks sharing the one GPU (gloo for the host-side
    max over ranks): every rank runs the library's CUDA search on its own instance, and
    rank 0 prints one line with the job throughput of both ranks."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = {**os.environ, "RTNN_BENCH_BACKEND": "gloo",
           "RTNN_AUTOTUNE_CACHE": str(tmp_path / "autotune.json")}
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(root, "bench.py"), "--gpus", "2", "--steps", "2", "--warmup", "3",
           "--scale", "0.005", "--no-other-workloads", "--no-e2e", "--cpu-seconds", "1"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=900, cwd=root, env=env)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["n_gpus"] == 2 and d["value"] > 0 and d["identical_sets"] is True
    assert d["gpu_launches"] > 0 and d["cpu_baseline"] is None   # the CPU sample is N=1 only
