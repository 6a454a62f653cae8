"""Several GPUs: replicas over disjoint pixel ranges.

Pixels are independent, so N GPUs (one process each, torch.distributed for
the plumbing) invert disjoint contiguous pixel ranges of a cube with no
collective in the data path; the results are gathered on one rank on the
host.  This replaces the reference's per-stream pixel slices
(`displsPixels` / `sendCountPixels`, gmilos.cu:1008-1060) one level up.

The gather runs over a gloo group on CPU tensors, whatever the default
backend, so it needs no device memory and works in CPU-only tests.
"""
import datetime

import numpy as np


def pixel_range(npix, rank, world):
    """Contiguous range [start, stop) of `rank` in a balanced split of npix
    pixels over `world` ranks: the first npix % world ranks take one pixel
    more; ranks past npix get an empty range."""
    if world < 1 or not 0 <= rank < world or npix < 0:
        raise ValueError("bad partition: npix %d, rank %d of %d" % (npix, rank, world))
    base, extra = divmod(npix, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def host_group(timeout_s=None):
    """A gloo group over all ranks for host-side traffic (a new group, so the
    default group may be NCCL).  timeout_s bounds every operation on it."""
    import torch.distributed as dist
    kw = {} if timeout_s is None else {"timeout": datetime.timedelta(seconds=timeout_s)}
    return dist.new_group(backend="gloo", **kw)


def gather_rows(local, npix, group=None, dst=0):
    """Gather the rows of each rank's pixel range into one [npix, ...] array
    on rank `dst` (None on the others).  `local` holds this rank's rows in
    order; every rank passes the same npix and row shape."""
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    start, stop = pixel_range(npix, rank, world)
    local = np.ascontiguousarray(local)
    if local.shape[0] != stop - start:
        raise ValueError("rank %d holds %d rows, its range has %d" % (rank, local.shape[0], stop - start))
    rows = -(-npix // world)               # the largest range
    pad = np.zeros((rows,) + local.shape[1:], dtype=local.dtype)
    pad[: local.shape[0]] = local
    # gloo moves no unsigned integers wider than a byte: carry them as the
    # signed type of the same width
    wire = {np.dtype(np.uint32): np.int32, np.dtype(np.uint64): np.int64, np.dtype(np.uint16): np.int16}
    t = torch.from_numpy(pad.view(wire.get(pad.dtype, pad.dtype)))
    if rank == dst:
        parts = [torch.empty_like(t) for _ in range(world)]
        dist.gather(t, gather_list=parts, dst=dist.get_global_rank(group, dst) if group else dst, group=group)
        out = np.empty((npix,) + local.shape[1:], dtype=local.dtype)
        for r, p in enumerate(parts):
            a, b = pixel_range(npix, r, world)
            out[a:b] = p.numpy().view(local.dtype)[: b - a]
        return out
    dist.gather(t, dst=dist.get_global_rank(group, dst) if group else dst, group=group)
    return None


def invert_sharded(engine, iquv, group=None, dst=0, outputs=("model64", "chi2", "iters", "status")):
    """Invert this rank's pixel range of the cube `iquv` ([P][4][nl], the
    whole cube on every rank) with `engine` and gather the named outputs on
    rank `dst`: a dict of [P, ...] arrays there, None elsewhere."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    npix = len(iquv)
    start, stop = pixel_range(npix, rank, world)
    out = engine.invert(iquv[start:stop])
    result = {}
    for k in outputs:
        v = out[k]
        v = v.cpu().numpy() if hasattr(v, "cpu") else np.asarray(v)
        result[k] = gather_rows(v, npix, group=group, dst=dst)
    return result if rank == dst else None


def max_over_ranks(value, group=None):
    """The largest `value` over all ranks (the timing rule for several
    GPUs: a step takes as long as its slowest rank)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
