"""Ensemble host logic on CPU: the member generator (seeded perturbations of
the cfg0 estuary), the longest-processing-time plan that deals members out
to GPUs, and that plan agreed by two gloo ranks."""
import ast
import math
import os
import socket

import numpy as np
import pytest


def test_lpt_partition_covers_and_balances():
    from fesomc import ensemble
    rng = np.random.default_rng(3)
    costs = [int(c) for c in rng.integers(1, 1000, 48)]
    for bins in (1, 2, 3, 8):
        plan = ensemble.lpt_partition(costs, bins)
        flat = sorted(i for b in plan for i in b)
        assert flat == list(range(48))
        loads = [sum(costs[i] for i in b) for b in plan]
        # LPT bound: no bin exceeds the mean by more than the largest member
        assert max(loads) <= sum(costs) / bins + max(costs)
        for b in plan:                                   # largest first within a bin
            assert [costs[i] for i in b] == sorted((costs[i] for i in b), reverse=True)
    assert ensemble.lpt_partition(costs, 4) == ensemble.lpt_partition(list(costs), 4)
    with pytest.raises(ValueError):
        ensemble.lpt_partition(costs, 0)


def test_member_draws_follow_the_spec():
    from fesomc import cases
    draws = [cases.ensemble_draw(i) for i in range(48)]
    nodes = np.array([(d["nx"] + 1) * (d["ny"] + 1) for d in draws])
    assert nodes.min() >= 0.9 * 20_000 and nodes.max() <= 1.1 * 250_000
    assert len(set(nodes)) >= 40                         # sizes differ
    assert {d["nsigma"] for d in draws} == {11, 21}
    for d in draws:
        assert 0.96 <= d["m2_amp"] <= 1.44
        assert -15.0 <= d["m2_phase_deg"] <= 15.0
        assert math.hypot(*d["stress"]) <= 0.2
        assert 0.0 <= d["noise_sigma"] <= 1.0
        assert 2.0 < (d["nx"] + 1) / (d["ny"] + 1) < 3.0
    assert cases.ensemble_draw(5) == cases.ensemble_draw(5)
    assert cases.ensemble_draw(5, seed=1) != cases.ensemble_draw(5)


def test_small_members_build(built):
    from fesomc import cases
    a = cases.ensemble_member(0, nodes_range=(300, 900))
    b = cases.ensemble_member(1, nodes_range=(300, 900))
    for c, i in ((a, 0), (b, 1)):
        d = cases.ensemble_draw(i, nodes_range=(300, 900))
        assert c.mesh.N == (d["nx"] + 1) * (d["ny"] + 1)
        assert c.mesh.NS == d["nsigma"]
        f = c.forcing_fn(1, c.params.time_jd0)
        assert np.allclose(f["taux"], d["stress"][0]) and np.allclose(f["tauy"], d["stress"][1])
        assert f["ampt"][: c.mesh.c.nobn].min() == pytest.approx(d["m2_amp"])


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
    import torch.distributed as dist
    from fesomc import cases, ensemble, replicas
    ws, r, _ = replicas.dist_env()
    reps = replicas.Replicas(ws, "gloo", timeout_s=30)
    costs = [(d["nx"] + 1) * (d["ny"] + 1) * (d["nsigma"] - 1)
             for d in (cases.ensemble_draw(i) for i in range(48))]
    mine = ensemble.lpt_partition(costs, ws)[r]
    got = [None] * ws
    dist.all_gather_object(got, mine)
    reps.close()
    with open(os.path.join(out_dir, f"rank{r}.txt"), "w") as f:
        f.write(repr(got) + "\n")


def test_two_gloo_ranks_share_the_members(tmp_path):
    pytest.importorskip("torch")
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    views = [ast.literal_eval((tmp_path / f"rank{r}.txt").read_text()) for r in range(2)]
    assert views[0] == views[1]
    a, b = views[0]
    assert sorted(a + b) == list(range(48)) and not set(a) & set(b)
