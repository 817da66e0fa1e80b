"""Replica bookkeeping of multi-GPU runs (bench.py --gpus N), on CPU with the
gloo backend and two ranks: barrier, maximum of the per-rank times and the
whole-job rate."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(os.path.dirname(here), "fesom-c_b200"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    from fesomc import replicas
    ws, r, local = replicas.dist_env()
    reps = replicas.Replicas(ws, "gloo", timeout_s=30)
    reps.barrier()
    t = 1.0 + r                 # rank 1 is the slow one
    tmax = reps.max(t)
    rate = replicas.whole_job_rate(100, 10, ws, tmax)
    reps.close()
    with open(os.path.join(out_dir, f"rank{r}.txt"), "w") as f:
        f.write(f"{ws} {local} {tmax} {rate}\n")


def test_two_gloo_replicas(tmp_path):
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    for r in range(2):
        ws, local, tmax, rate = (tmp_path / f"rank{r}.txt").read_text().split()
        assert int(ws) == 2 and int(local) == r
        assert float(tmax) == 2.0
        assert float(rate) == pytest.approx(100 * 10 * 2 / 2.0)


def test_single_process_needs_no_group():
    from fesomc import replicas
    reps = replicas.Replicas(1, "gloo")
    reps.barrier()
    assert reps.max(3.5) == 3.5
    assert replicas.whole_job_rate(7, 3, 1, 2.0) == pytest.approx(10.5)
    reps.close()
