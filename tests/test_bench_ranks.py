"""The multi-rank path of bench.py on CPU: two gloo ranks, each with its own device time,
agree on the slowest one; the whole-job rate counts every rank's units over that time; the
reference arm runs on rank 0 only."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms = 100.0 + 50.0 * rank
    m = bench.max_over_ranks_ms(ms, world, "cpu")
    dist.barrier()
    out[rank] = (m, bench.whole_job_rate(world, 32, 5, m))
    dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_slowest_time():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as man:
        out = man.dict()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0] == res[1]
    m, rate = res[0]
    assert m == 150.0
    assert abs(rate - 2 * 32 * 5 / 0.15) < 1e-9


def test_reference_arm_only_on_rank_zero(capsys, monkeypatch):
    sys.path.insert(0, ROOT)
    import bench

    monkeypatch.setenv("RANK", "1")
    bench.run_reference(bench.parse_args.__globals__["argparse"].Namespace(gpus=2, steps=1, warmup=0))
    assert capsys.readouterr().out == ""
