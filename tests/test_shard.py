"""The path across ranks (gliomasolver_b200.shard), on CPU with gloo.

The step runs as independent replicas; a TMCMC stage shards its samples over
the ranks.  Here two gloo ranks each solve their share of a small stage with
the oracle's forward map (the C restatement of the reference's step), gather
per-sample results to rank 0 and reduce a duration with the max over ranks;
rank 0 checks that the gathered results equal a one-process run of the whole
stage and that every sample was solved exactly once.
"""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

from gliomasolver_b200.shard import gather_results, max_over_ranks, stage_shards


def test_stage_shards_cover_and_balance():
    rng = np.random.default_rng(0)
    steps = rng.integers(50, 15000, 101)
    for world in (1, 2, 3, 8):
        shards = stage_shards(steps, world)
        assert len(shards) == world
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(steps)))
        loads = [int(steps[s].sum()) for s in shards]
        # longest-processing-time-first: no rank exceeds another by more than one sample
        assert max(loads) - min(loads) <= steps.max()
        assert shards == stage_shards(list(steps), world)
    assert stage_shards([], 2) == [[], []]
    with pytest.raises(ValueError):
        stage_shards([1], 0)


def test_single_process_helpers():
    assert max_over_ranks(3.5) == 3.5
    assert gather_results({2: 1.0}) == {2: 1.0}


def _stage():
    """A small stage: 7 samples on one 16^3 anatomy with uneven horizons."""
    from gliomasolver_b200.anatomy import make_anatomy, tumor_ic
    from gliomasolver_b200.schedule import make_schedule

    n = 16
    pw, pg, _ = make_anatomy(n, 3)
    rng = np.random.default_rng(5)
    stage = []
    for i in range(7):
        x0 = tuple(rng.uniform(0.4, 0.6, 3))
        s = make_schedule(float(rng.uniform(0.05, 0.3)), float(rng.uniform(0.01, 0.2)), float(rng.uniform(2, 12)),
                          25.6, n // 8, "f64")
        stage.append((tumor_ic(n, x0, pw, pg), s))
    return pw, pg, stage


def _solve(pw, pg, c0, s):
    from oracle import oracle as O

    u = O.rd_steps_dense(pw, pg, c0, s.Dw, s.Dg, s.rho, s.h, s.dt, s.nsteps)
    return float(np.sum(u * u))


def _rank_main(rank, world, port, out_path):
    import torch.distributed as dist

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        pw, pg, stage = _stage()
        mine = stage_shards([s.nsteps for _, s in stage], world)[rank]
        local = {i: _solve(pw, pg, *stage[i]) for i in mine}
        merged = gather_results(local)
        worst = max_over_ranks(1.5 + rank)
        if rank == 0:
            np.save(out_path, np.array([worst] + [merged[i] for i in range(len(stage))] + [len(merged)]))
        else:
            assert merged is None
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_solve_a_stage():
    pw, pg, stage = _stage()
    want = [_solve(pw, pg, c0, s) for c0, s in stage]
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "rank0.npy")
        mp.start_processes(_rank_main, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
        got = np.load(out)
    assert got[0] == 2.5                       # max over ranks
    assert got[-1] == len(stage)               # every sample once
    assert np.array_equal(got[1:-1], want)     # same results as one process
