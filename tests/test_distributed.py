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


# ---------------------------------------------------------------------------------------------------------------
# Row slabs of one domain: halo exchange for dilation and upwind, mass reduction
# ---------------------------------------------------------------------------------------------------------------

def _global_set(height=40, width=60):
    from tests.gpu_util import rand_set

    b, e, off, rows = rand_set(height, 2.5, seed=17, max_col=width, row0=0)
    keep = np.diff(off) > 0
    keep[::7] = True  # some empty rows stay listed
    sel = np.nonzero(keep)[0]
    counts = np.diff(off)[sel]
    new_off = np.zeros(sel.size + 1, np.int64)
    np.cumsum(counts, out=new_off[1:])
    idx = np.concatenate([np.arange(off[r], off[r + 1]) for r in sel]) if sel.size else np.zeros(0, np.int64)
    return (b[idx].astype(np.int32), e[idx].astype(np.int32), new_off.astype(np.int32), rows[sel].astype(np.int32))


def _np(t):
    return np.asarray(t.numpy() if hasattr(t, "numpy") else t)


def _slab_rank(rank, world, port, out):
    import torch
    import torch.distributed as dist

    from oracle import oracle as O
    from subsetix_b200.distributed import mass_allreduce, slab_dilate, slab_rows, slab_upwind, take_rows

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        H, W = 40, 60
        g = [torch.as_tensor(a) for a in _global_set(H, W)]
        r0, r1 = slab_rows(H, rank, world)
        slab = take_rows(*g, r0, r1)

        def dilate(b, e, off, rows, hx, hy):
            res = O.dilate(O.ISet(_np(b), _np(e), _np(off), _np(rows)), hx, hy)
            return tuple(torch.as_tensor(x) for x in res)

        d = slab_dilate(slab, r0, r1, 1, 2, rank, world, dilate)
        out[f"dil{rank}"] = tuple(_np(x).tolist() for x in d)

        full = O.ISet(*(_np(x) for x in g))
        cell = O.cell_offsets(full)
        vals = np.random.default_rng(3).uniform(0, 1, int(cell[-1])).astype(np.float64)
        sb, sv = take_rows(*g, r0, r1, values=torch.as_tensor(vals), cell_offsets=torch.as_tensor(cell))
        scell = torch.zeros(int(sb[0].numel()) + 1, dtype=torch.int32)
        scell[1:] = torch.cumsum(sb[1] - sb[0], 0)

        def step(b, e, off, rows, v, c):
            f = O.Field(O.ISet(_np(b), _np(e), _np(off), _np(rows)), _np(v), _np(c))
            return torch.as_tensor(O.upwind(f, width=W, height=H, a=0.8, b=-0.6, dt=0.01, dx=0.05, dy=0.05,
                                            dtype=np.float64))

        res = slab_upwind(sb, sv, scell, r0, r1, rank, world, 10, step)
        out[f"up{rank}"] = _np(res).tolist()
        v = _np(res)
        s = c = 0.0
        for x in v.tolist():
            t = s + x
            c += ((s - t) + x) if abs(s) >= abs(x) else ((x - t) + s)
            s = t
        out[f"mass{rank}"] = mass_allreduce(s, c)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_row_slabs_match_one_process(world):
    from oracle import oracle as O

    port = 31500 + (os.getpid() % 1500) + world
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_slab_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    H, W = 40, 60
    g = O.ISet(*_global_set(H, W))
    # dilation (halo_y = 2): the slabs' rows, in rank order, are the global result's rows
    want = O.dilate(g, 1, 2)
    b = np.concatenate([res[f"dil{r}"][0] for r in range(world)])
    e = np.concatenate([res[f"dil{r}"][1] for r in range(world)])
    rows = np.concatenate([res[f"dil{r}"][3] for r in range(world)])
    np.testing.assert_array_equal(b, want.begin)
    np.testing.assert_array_equal(e, want.end)
    np.testing.assert_array_equal(rows, want.rows)
    # ten upwind steps with one halo row per side per step
    cell = O.cell_offsets(g)
    v = np.random.default_rng(3).uniform(0, 1, int(cell[-1])).astype(np.float64)
    for _ in range(10):
        v = O.upwind(O.Field(g, v, cell), width=W, height=H, a=0.8, b=-0.6, dt=0.01, dx=0.05, dy=0.05,
                     dtype=np.float64)
    got = np.concatenate([res[f"up{r}"] for r in range(world)])
    np.testing.assert_array_equal(got, v)
    # the mass reduction: identical on every rank, equal to the compensated global sum
    masses = [res[f"mass{r}"] for r in range(world)]
    assert len(set(masses)) == 1
    assert abs(masses[0] - O.mass_kahan(v, 1.0)) <= 1e-14 * abs(masses[0])
