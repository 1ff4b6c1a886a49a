"""The multi-rank path on CPU: two gloo ranks shard the batch and reduce the timing.

Each rank evaluates its shard of the stacked shape batch with the oracle;
the shards' results, concatenated in rank order, must equal the result of
one process evaluating the whole batch, and the timing reduction must
return the maximum over ranks.
"""

import os

import numpy as np
import pytest
import torch.multiprocessing as mp

from subsetix_b200.distributed import shard


def test_shard_covers_every_unit_once():
    for total in (0, 1, 7, 128, 1000):
        for world in (1, 2, 3, 8):
            got = [shard(total, r, world) for r in range(world)]
            assert sum(c for _, c in got) == total
            assert all(got[r][0] + got[r][1] == got[r + 1][0] for r in range(world - 1))
            assert max(c for _, c in got) - min(c for _, c in got) <= 1
    with pytest.raises(ValueError):
        shard(4, 2, 2)


def _ops(copies, first):
    from oracle import oracle as O
    from subsetix_b200 import synth

    shapes = synth.shape_operands(256)
    leaves = [O.ISet(*synth.stack_rows(s, copies, 256, first=first)) for s in shapes]
    spec = ("symmetric_difference", ("difference", ("union", "A", "B"), ("intersection", "C", "D")), "E")
    return O.evaluate(spec, dict(zip("ABCDE", leaves)))


def _rank(rank, world, port, copies, out):
    import torch
    import torch.distributed as dist

    from subsetix_b200.distributed import max_over_ranks

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        first, count = shard(world * copies, rank, world)
        res = _ops(count, first)
        out[rank] = (res.begin.tolist(), res.end.tolist(), res.row_offsets.tolist(), first, count)
        out[f"max{rank}"] = max_over_ranks(10.0 + rank)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_match_one_process():
    world, copies = 2, 3
    port = 29500 + (os.getpid() % 2000)
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, port, copies, out), nprocs=world, join=True)
        results = dict(out)
    whole = _ops(world * copies, 0)
    begin = np.concatenate([results[r][0] for r in range(world)])
    end = np.concatenate([results[r][1] for r in range(world)])
    np.testing.assert_array_equal(begin, whole.begin)
    np.testing.assert_array_equal(end, whole.end)
    # row offsets of the shards, rebased, tile the whole batch's offsets
    offs = [np.asarray(results[0][2])]
    for r in range(1, world):
        offs.append(np.asarray(results[r][2])[1:] + offs[-1][-1])
    np.testing.assert_array_equal(np.concatenate(offs), whole.row_offsets)
    assert results["max0"] == results["max1"] == 10.0 + world - 1
