"""bench.py's multi-process path on CPU: two gloo ranks run the same rank
setup and max-over-ranks timing that `bench.py --gpus N` runs under torchrun
with NCCL, and the whole-job rate counts every rank's work."""
import os
import socket

import pytest
import torch.multiprocessing as mp

import bench


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, q):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    r, w, local, dist = bench.dist_setup(world, backend="gloo")
    try:
        slowest = bench.max_over_ranks(10.0 + 5.0 * r, dist, device="cpu")  # rank r "took" 10 + 5r ms
        rate = bench.job_rate(w, 3, 1000, slowest / 1000.0)
        q.put((r, w, local, slowest, rate))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for r, (rank, world, local, slowest, rate) in enumerate(got):
        assert (rank, world, local) == (r, 2, r)
        assert slowest == 15.0  # the max over ranks, on every rank
        assert rate == pytest.approx(2 * 3 * 1000 / 0.015)


def test_single_process_needs_no_group(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert bench.dist_setup(1) == (0, 1, 0, None)
    assert bench.max_over_ranks(3.5, None) == 3.5
    with pytest.raises(SystemExit):
        bench.dist_setup(2)


def test_level_traffic_matches_its_profile():
    """The DRAM bytes bench.py reports as roofline.traffic come from a
    committed ncu summary; the constant and the summary agree."""
    for workload, tr in bench.LEVEL_TRAFFIC.items():
        assert workload in bench.WORKLOADS
        path = os.path.join(bench.REPO, tr["profile"])
        text = open(path).read()
        assert f"{tr['bytes']:,} bytes" in text, (workload, path)
        assert tr["launches"] > 0 and tr["window_bits"] >= 10 and tr["threads"] in (128, 256, 512)
