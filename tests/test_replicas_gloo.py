"""Host logic of multi-GPU runs (independent replicas, no data-path collective) on CPU ranks.

bench.py --gpus N runs one replica per rank; the job time is the maximum over ranks and the
job throughput is all ranks' units over that time.  Two gloo ranks on 127.0.0.1 check the
reduction and the aggregate; the reference arm must leave ranks other than 0 idle.
"""
import os
import socket
import types

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        t = bench.max_over_ranks(1.0 + 2.5 * rank, world, device="cpu")   # this rank's seconds
        v = bench.job_throughput(100.0, world, t)
        dist.barrier()
    finally:
        dist.destroy_process_group()
    with open(os.path.join(out_dir, f"r{rank}.txt"), "w") as f:
        f.write(f"{t!r} {v!r}")


def test_max_over_ranks_and_throughput_two_gloo_ranks(tmp_path):
    mp = pytest.importorskip("torch.multiprocessing")
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    for r in range(world):
        t, v = (float(x) for x in (tmp_path / f"r{r}.txt").read_text().split())
        assert t == 3.5                       # the slowest rank's time, seen by every rank
        assert v == pytest.approx(200.0 / 3.5)  # 2 ranks x 100 units / 3.5 s


def test_single_rank_needs_no_process_group():
    import bench
    assert bench.max_over_ranks(2.25, 1) == 2.25
    assert bench.job_throughput(10.0, 1, 2.0) == 5.0


def test_reference_arm_idle_on_other_ranks(monkeypatch, capsys):
    import bench
    monkeypatch.setenv("RANK", "1")
    args = types.SimpleNamespace(n=64, ref_layers=1, steps=3, warmup=3, gpus=2)
    assert bench.run_reference(args) == 0
    assert capsys.readouterr().out == ""
