"""The replica path of bench.py at world size 2, on CPU with gloo: the step time every rank
reports is the slowest rank's, whatever the order in which ranks finish, and the reference
arm does no work on ranks other than 0."""
import importlib.util
import os
import socket

from conftest import ROOT


def _bench():
    spec = importlib.util.spec_from_file_location("bench_ranks", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench = _bench()
        # rank r measured (r + 1) * 1.5 ms; two rounds, the second with the order reversed
        a = bench.max_over_ranks((rank + 1) * 1.5, dist, device="cpu")
        b = bench.max_over_ranks((world - rank) * 0.25, dist, device="cpu")
        q.put((rank, a, b))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_step_time_is_the_slowest_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    world, port = 2, _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=5) for _ in range(world))
    assert got == [(0, 3.0, 0.5), (1, 3.0, 0.5)]


def test_single_process_is_its_own_maximum():
    assert _bench().max_over_ranks(1.25, None) == 1.25


def test_reference_arm_is_idle_off_rank_zero(capsys):
    bench = _bench()

    class Args:
        steps, warmup = 2, 3

    assert bench.reference_arm(Args(), 1, 2) == 0
    assert capsys.readouterr().out == ""
