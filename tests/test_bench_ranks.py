"""The multi-rank path of bench.py on CPU: two gloo ranks take the max of
their timings with one all-reduce, the whole-job rate counts every rank's
units, and the reference arm does no work on ranks other than 0."""
import importlib.util
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        b = _bench()
        t = b.max_over_ranks([1.0 + rank, 10.0 - rank, 0.5 * (rank + 1)], world, "cpu")
        out[rank] = (t, b.job_rate(5, world, t[0]))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_rate_with_two_gloo_ranks():
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank_main, args=(2, _free_port(), out), nprocs=2, start_method="spawn", join=True)
    for rank in (0, 1):
        t, rate = out[rank]
        assert t == [2.0, 10.0, 1.0]
        assert rate == pytest.approx(2 * 5 / 2.0)


def test_single_rank_needs_no_process_group():
    b = _bench()
    assert b.max_over_ranks([3.0, 4.0], 1, "cpu") == [3.0, 4.0]
    assert b.job_rate(5, 1, 2.0) == 2.5


def test_reference_arm_is_silent_on_other_ranks(monkeypatch, capsys):
    b = _bench()
    monkeypatch.setenv("RANK", "1")

    class Args:
        steps, warmup, gpus = 1, 1, 2

    assert b.run_reference(Args()) == 0
    assert capsys.readouterr().out == ""
