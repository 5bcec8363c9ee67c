"""The multi-GPU path of `bench.py` (independent replicas, one scan per rank, no exchange step)
on CPU: two gloo ranks launched as torchrun would (RANK / WORLD_SIZE / LOCAL_RANK, rendezvous on
127.0.0.1) take the maximum of their timed regions and report the whole job's patterns over it;
each rank makes its own scan; under the reference arm only rank 0 works."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    from ptyrs_b200 import sim
    from ptyrs_b200.replicas import Replicas, job_value
    group = Replicas("gloo", timeout_s=60)
    group.barrier()
    ms = 100.0 + 50.0 * rank          # this rank's timed region
    top = group.max(ms)
    s = sim.make_scan("rpie64", seed=rank, scale=0.05)   # the per-rank scan bench.py makes
    group.barrier()
    out.put((rank, top, job_value(len(s["counts"]), group.world, 3, top),
             float(s["counts"].sum())))
    group.close()


def test_two_gloo_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, top0, v0, c0), (r1, top1, v1, c1) = got
    assert (r0, r1) == (0, 1)
    assert top0 == top1 == 150.0
    frames = len(np.arange(400)[:max(2, int(400 * 0.05))])
    assert v0 == v1 == frames * 2 * 3 / 0.150
    assert c0 != c1      # each rank reconstructs its own seeded scan


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("LOCAL_RANK", "1")

    class Args:
        workload, scale, steps, warmup = "ml256", 1.0, 1, 0

    assert bench.reference_arm(Args, bench.WORKLOADS["ml256"]) is None
    assert capsys.readouterr().out == ""
