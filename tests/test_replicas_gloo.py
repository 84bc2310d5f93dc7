"""The multi-GPU path of bench.py is replicas only: every rank runs its own
discharge / deck / request stream with its own seed, no collective touches
the data path, and the whole-job figures are the slowest rank's time and the
summed work.  This covers that host logic with two gloo ranks on the CPU."""
import os
import socket
import sys

import numpy as np
import torch.distributed as td
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "aurora-pic_b200"))
    import bench
    from apic import workloads as W
    td.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r timed 10 + r ms over 1000 (r + 1) particle-steps
        t, work = bench._reduce(td, 10.0 + rank, 1000.0 * (rank + 1), device="cpu")
        # replica inputs: the seed of rank r is the bench's 7 + r
        wl = W.ccp_helium(particles_per_cell=4, cells=16, seed=7 + rank, table_rows=64)
        head = wl.species[0].x[:8].tolist()
        out.put((rank, t, work, head))
        td.barrier()
    finally:
        td.destroy_process_group()


def test_two_gloo_replicas_reduce_max_time_and_total_work():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, work, _ in res:
        assert t == 11.0  # the slowest rank
        assert work == 3000.0  # 1000 + 2000
    # each replica loads its own particles
    assert not np.allclose(res[0][3], res[1][3])


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")

    class Args:
        workload = "ccp1d"
    bench.run_reference(Args())  # returns at once, prints nothing
    assert capsys.readouterr().out == ""
