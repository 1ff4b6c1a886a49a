"""Work across ranks (one process per GPU).

Two decompositions:

* Independent units (sets, expressions, whole simulations of a batch) are
  split into contiguous shards, one per rank, with no data-path collective;
  the only communication is the timing reduction, the maximum over ranks.
* One large domain is split into row slabs.  Set algebra is row-local and
  needs nothing from the neighbours.  Dilation by ``halo_y`` reads ``halo_y``
  rows on either side (``subsetix_cupy/morphology.py:225-248``) and an upwind
  step one row (``subsetix_cupy/interval_stencil.py:17-57``), so before those
  a rank receives its neighbours' boundary rows (point-to-point send/recv of
  interval rows and, for fields, their values), computes on its slab plus
  the halo, and keeps its own rows.  The mass integral's partial sums are
  all-gathered and added in rank order, so every rank gets the same FP64
  total whatever the reduction tree.

The exchange works on whatever device the tensors live on: NCCL between
GPUs, gloo between CPU processes.  Data lands in local buffers; nothing reads
a peer's memory.
"""

from __future__ import annotations

from typing import Callable, List, Optional, Sequence, Tuple


def shard(total: int, rank: int, world: int) -> Tuple[int, int]:
    """``(first, count)`` of rank ``rank``'s contiguous share of ``total`` units (sizes differ by at most one)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    if total < 0:
        raise ValueError("total must be non-negative")
    base, extra = divmod(int(total), int(world))
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of ``value`` over the ranks of the default process group (the value itself when there is none)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------------------------------------------
# Row slabs of one domain
# ---------------------------------------------------------------------------------------------------------------

def _dist():
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        raise RuntimeError("row-slab operations need an initialised process group")
    return dist


def slab_rows(height: int, rank: int, world: int) -> Tuple[int, int]:
    """Rows ``[r0, r1)`` of rank ``rank``'s slab of a ``height``-row domain."""
    first, count = shard(height, rank, world)
    return first, first + count


def take_rows(begin, end, row_offsets, rows, lo: int, hi: int, values=None, cell_offsets=None):
    """The rows of a set with ids in ``[lo, hi)`` as a new set (and the values of those cells)."""
    import torch

    r = rows
    a = int(torch.searchsorted(r, torch.tensor([lo], dtype=r.dtype, device=r.device)).item())
    b = int(torch.searchsorted(r, torch.tensor([hi], dtype=r.dtype, device=r.device)).item())
    i0, i1 = int(row_offsets[a].item()), int(row_offsets[b].item())
    out = (begin[i0:i1].clone(), end[i0:i1].clone(), (row_offsets[a:b + 1] - i0).clone(), rows[a:b].clone())
    if values is None:
        return out
    c0, c1 = int(cell_offsets[i0].item()), int(cell_offsets[i1].item())
    return out, values[c0:c1].clone()


def _pack(part, values=None):
    """One int32 message: [rows, intervals, cells, rows..., counts..., begins..., ends...] (+ value bits)."""
    import torch

    b, e, off, rows = part
    counts = (off[1:] - off[:-1]).to(torch.int32)
    nv = 0 if values is None else int(values.numel())
    head = torch.tensor([int(rows.numel()), int(b.numel()), nv], dtype=torch.int32, device=b.device)
    pieces = [head, rows.to(torch.int32), counts, b.to(torch.int32), e.to(torch.int32)]
    if values is not None:
        pieces.append(values.contiguous().view(torch.int32))
    return torch.cat(pieces)


def _unpack(msg, value_dtype=None):
    import torch

    nr, ni, nv = (int(x) for x in msg[:3].tolist())
    p = 3
    rows = msg[p:p + nr]
    p += nr
    counts = msg[p:p + nr]
    p += nr
    b = msg[p:p + ni]
    p += ni
    e = msg[p:p + ni]
    p += ni
    off = torch.zeros(nr + 1, dtype=torch.int32, device=msg.device)
    if nr:
        off[1:] = torch.cumsum(counts, 0)
    values = None
    if value_dtype is not None:
        words = nv * torch.empty(0, dtype=value_dtype).element_size() // 4
        values = msg[p:p + words].clone().view(value_dtype)
    return (b.clone(), e.clone(), off, rows.clone()), values


def _swap(send_down, send_up, rank: int, world: int, group=None):
    """Send to rank-1 / rank+1 and receive from them (sizes first); returns (from below, from above)."""
    import torch

    dist = _dist()
    dev = (send_down if send_down is not None else send_up).device
    ops, sizes = [], {}
    for peer, msg in ((rank - 1, send_down), (rank + 1, send_up)):
        if 0 <= peer < world:
            n = torch.tensor([int(msg.numel())], dtype=torch.int64, device=dev)
            got = torch.empty(1, dtype=torch.int64, device=dev)
            ops += [dist.P2POp(dist.isend, n, peer, group), dist.P2POp(dist.irecv, got, peer, group)]
            sizes[peer] = got
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    ops, bufs = [], {}
    for peer, msg in ((rank - 1, send_down), (rank + 1, send_up)):
        if 0 <= peer < world:
            buf = torch.empty(int(sizes[peer].item()), dtype=torch.int32, device=dev)
            ops += [dist.P2POp(dist.isend, msg, peer, group), dist.P2POp(dist.irecv, buf, peer, group)]
            bufs[peer] = buf
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    return bufs.get(rank - 1), bufs.get(rank + 1)


def _concat_sets(parts):
    import torch

    parts = [p for p in parts if p is not None]
    b = torch.cat([p[0] for p in parts])
    e = torch.cat([p[1] for p in parts])
    rows = torch.cat([p[3] for p in parts])
    offs, base = [parts[0][2][:1]], 0
    for p in parts:
        offs.append(p[2][1:] + base)
        base += int(p[0].numel())
    return b, e, torch.cat(offs).to(torch.int32), rows


def with_halo(slab, r0: int, r1: int, halo: int, rank: int, world: int, values=None, cell_offsets=None,
              group=None):
    """The slab ``[r0, r1)`` extended by ``halo`` rows of each neighbour's slab (and their values).

    Every rank must call this together (it exchanges with rank - 1 and
    rank + 1).  Returns the extended set (rows still sorted), or with
    ``values`` the pair (set, values) in cell order.
    """
    b, e, off, rows = slab
    if values is None:
        down = _pack(take_rows(b, e, off, rows, r0, r0 + halo))
        up = _pack(take_rows(b, e, off, rows, r1 - halo, r1))
        from_below, from_above = _swap(down, up, rank, world, group)
        lo = _unpack(from_below)[0] if from_below is not None else None
        hi = _unpack(from_above)[0] if from_above is not None else None
        return _concat_sets([lo, slab, hi])
    dpart, dvals = take_rows(b, e, off, rows, r0, r0 + halo, values, cell_offsets)
    upart, uvals = take_rows(b, e, off, rows, r1 - halo, r1, values, cell_offsets)
    from_below, from_above = _swap(_pack(dpart, dvals), _pack(upart, uvals), rank, world, group)
    lo = _unpack(from_below, values.dtype) if from_below is not None else (None, None)
    hi = _unpack(from_above, values.dtype) if from_above is not None else (None, None)
    import torch

    ext = _concat_sets([lo[0], slab, hi[0]])
    vals = torch.cat([v for v in (lo[1], values, hi[1]) if v is not None])
    return ext, vals


def slab_dilate(slab, r0: int, r1: int, halo_x: int, halo_y: int, rank: int, world: int,
                dilate: Callable, group=None):
    """Box dilation of the global set restricted to rows ``[r0, r1)`` (the first and last slab also keep
    the rows the dilation adds below and above the domain).

    ``dilate(b, e, off, rows, halo_x, halo_y)`` dilates a local set (the
    product's ``dilate_interval_set`` on GPUs, any equal implementation
    elsewhere).  Output row ``y`` depends on input rows ``y - halo_y .. y +
    halo_y``, all present after the halo exchange.
    """
    if halo_y > r1 - r0:
        raise ValueError(f"a slab of {r1 - r0} rows cannot supply a halo of {halo_y} rows")
    ext = with_halo(slab, r0, r1, halo_y, rank, world, group=group) if halo_y > 0 else slab
    out = dilate(*ext, halo_x, halo_y)
    # the dilation is unbounded: rows below the domain belong to the first slab, rows above it to the last
    lo = r0 if rank > 0 else -(1 << 31)
    hi = r1 if rank < world - 1 else (1 << 31) - 1
    return take_rows(*out, lo, hi)


def slab_upwind(slab, values, cell_offsets, r0: int, r1: int, rank: int, world: int, steps: int,
                step: Callable, group=None):
    """``steps`` upwind steps of the global field restricted to rows ``[r0, r1)``.

    ``step(b, e, off, rows, values, cell_offsets)`` returns the new values of
    one upwind step of a local field with the global domain's width, height
    and spacing.  Each step receives one boundary row (intervals and values)
    from each neighbour first.
    """
    import torch

    b, e, off, rows = slab
    n_own = int(values.numel())
    for _ in range(int(steps)):
        (xb, xe, xoff, xrows), xv = with_halo(slab, r0, r1, 1, rank, world, values=values,
                                              cell_offsets=cell_offsets, group=group)
        xcell = torch.zeros(int(xb.numel()) + 1, dtype=torch.int32, device=xb.device)
        if xb.numel():
            xcell[1:] = torch.cumsum(xe - xb, 0)
        new = step(xb, xe, xoff, xrows, xv, xcell)
        # own cells follow the rows received from below
        lo = int(torch.searchsorted(xrows, torch.tensor([r0], dtype=xrows.dtype, device=xrows.device)).item())
        c0 = int(xcell[int(xoff[lo].item())].item())
        values = new[c0:c0 + n_own].clone()
    return values


def mass_allreduce(partial_sum: float, partial_comp: float = 0.0, group=None) -> float:
    """FP64 total of compensated partial sums, added in rank order on every rank (deterministic)."""
    import torch

    dist = _dist()
    world = dist.get_world_size(group)
    mine = torch.tensor([float(partial_sum), float(partial_comp)], dtype=torch.float64)
    backend = dist.get_backend(group)
    if backend == "nccl":
        mine = mine.cuda()
    parts = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(parts, mine, group=group)
    s = c = 0.0
    for p in parts:
        ps, pc = (float(x) for x in p.cpu())
        t = s + ps
        c += ((s - t) + ps) if abs(s) >= abs(ps) else ((ps - t) + s)
        c += pc
        s = t
    return s + c


__all__ = ["shard", "max_over_ranks", "slab_rows", "take_rows", "with_halo", "slab_dilate", "slab_upwind",
           "mass_allreduce"]
