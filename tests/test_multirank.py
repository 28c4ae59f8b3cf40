"""The N > 1 host logic of bench.py on CPU ranks (gloo, world size 2).

`bench.py --gpus N` runs one independent replica of the step per GPU (the
step does not shard: replicas only).  What the ranks share is host logic: the
slowest rank's time (all-reduce MAX), the whole-job throughput over it, and
the reference arm, which rank 0 alone runs and prints."""
import contextlib
import io
import multiprocessing as mp
import os
import socket
from argparse import Namespace
from datetime import timedelta


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist
    import bench
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
        r, w, _ = bench.dist_env()
        ms = bench.max_over_ranks(10.0 + 3.0 * r, w)  # rank 1 is the slowest
        value = bench.job_value(1000, 5, w, ms)
        # the reference arm with a stand-in for the timed CPU sample
        bench.cpu_reference_sample = lambda a, threads, steps, warmup, budget, rebuild_at: {
            "seconds": 1.0, "steps": steps, "warmup": warmup, "particles": 10, "fluid": 5,
            "rebuilds": int(rebuild_at >= 0), "threads": threads, "workload": "stand-in", "value": 123.0}
        args = Namespace(steps=5, warmup=3, ref_seconds=1.0, ref_single_steps=1, gpus=w, scene="dam_small")
        out = io.StringIO()
        with contextlib.redirect_stdout(out):
            bench.run_reference_arm(args, r, w)
        dist.barrier()
        dist.destroy_process_group()
        q.put((r, ms, value, out.getvalue()))
    except Exception as e:  # reported to the parent, which fails the test
        q.put((rank, None, None, repr(e)))


def test_two_ranks_max_time_job_value_and_reference_arm():
    import json
    import bench
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = {}
    for _ in range(2):
        r, ms, value, text = q.get(timeout=180)
        res[r] = (ms, value, text)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in (0, 1):
        assert res[r][0] == 13.0, res[r]
        assert abs(res[r][1] - 1000 * 5 * 2 / 0.013) < 1e-6 * res[r][1]
    line = json.loads(res[0][2].strip())
    assert line["impl"] == "reference" and line["value"] == 123.0 and line["n_gpus"] == 2
    assert line["steps"] == 5 and line["warmup"] == 3 and "1 neighbour rebuild" in line["cpu_baseline"]["sample"]
    assert line["cpu_baseline"]["single_thread"]["steps"] == 1
    assert line["config"] == bench.bench_config("stand-in", "fp64")
    assert line["e2e"]["h2d_bytes_per_step"] == 0
    assert res[1][2] == ""  # the other ranks do no work and print nothing
