"""Neighbour lists over several GPUs, one process per GPU.

The build shards without exchanging pairs:

* One large system is split by **rows**: rank r owns the atoms
  ``[lo_r, hi_r)`` and produces the rows ``i`` in that range.  Every rank
  bins all atoms (binning is cheap next to the pair passes), so the only
  collectives are an all-gather of positions (24 B per atom) and one of the
  per-rank pair totals, from which each rank learns where its slice starts in
  the global list.  Because the engine emits rows in ascending ``i`` and a
  row's pairs in the reference's order, the concatenation of the ranks'
  slices in rank order IS the single-GPU list, bit for bit.
* Many independent systems are split by an estimate of their cost; each rank
  builds its own systems with ``NeighbourListBatch`` and no collective at all.

The reference builds one list per process and has no multi-device mode
(src/libneighbours/neighbour_list.cc:99-204); this module is an addition.
Collectives go through ``torch.distributed`` (NCCL on GPUs, gloo on CPU).
"""

from collections import namedtuple

import numpy as np

ShardedList = namedtuple("ShardedList", "arrays atom_range pair_offset total_pairs")
ShardedList.__doc__ = """One rank's slice of a row-split neighbour list.

arrays: the requested quantities for rows atom_range[0] <= i < atom_range[1]
    (torch CUDA tensors, request order, a bare tensor for one character).
atom_range: (lo, hi), this rank's rows.
pair_offset: index of this slice's first pair in the global list.
total_pairs: length of the global list."""


# ---------------------------------------------------------------------------
# partitioning (host only)
# ---------------------------------------------------------------------------

def partition_rows(nat, world_size, weights=None):
    """Contiguous row ranges, one per rank, covering [0, nat).

    Without weights every rank gets nat // world_size atoms (the first
    nat % world_size ranks one more).  With per-atom weights (e.g. the
    neighbour counts of a previous step) the cut points split the cumulative
    weight evenly, which balances the pairs rather than the atoms.
    """
    nat = int(nat)
    world_size = int(world_size)
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    if nat < 0:
        raise ValueError("nat must be >= 0")
    if weights is None:
        base, extra = divmod(nat, world_size)
        cuts = [0]
        for r in range(world_size):
            cuts.append(cuts[-1] + base + (1 if r < extra else 0))
    else:
        w = np.asarray(weights, dtype=np.float64)
        if w.shape != (nat,):
            raise ValueError("weights must have one entry per atom")
        if np.any(w < 0):
            raise ValueError("weights must be non-negative")
        cum = np.concatenate([[0.0], np.cumsum(w)])
        total = cum[-1]
        cuts = [0]
        for r in range(1, world_size):
            target = total * r / world_size
            c = int(np.searchsorted(cum, target, side="left"))
            cuts.append(min(max(c, cuts[-1]), nat))
        cuts.append(nat)
    return [(cuts[r], cuts[r + 1]) for r in range(world_size)]


def system_cost(nat, cell, cutoff):
    """Pair-count estimate n * rho * (4/3) pi rc^3 of one system, the quantity
    the batch partition balances.  A zero-volume (non-periodic, flat) cell
    falls back to n^2."""
    nat = int(nat)
    cell = np.asarray(cell, dtype=np.float64).reshape(3, 3)
    vol = abs(float(np.linalg.det(cell)))
    rc = float(np.max(np.asarray(cutoff, dtype=np.float64)))
    if vol <= 1e-12:
        return float(nat) * float(nat)
    rho = nat / vol
    return nat * min(rho * (4.0 / 3.0) * np.pi * rc ** 3, float(nat))


def partition_systems(costs, world_size):
    """Assign systems to ranks by longest-processing-time-first: systems in
    descending cost (ties by index) each go to the currently lightest rank
    (ties to the lowest rank).  Returns, per rank, its system indices in
    ascending order.  Deterministic, so every rank computes the same plan
    without communicating."""
    world_size = int(world_size)
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    costs = [float(c) for c in costs]
    order = sorted(range(len(costs)), key=lambda s: (-costs[s], s))
    load = [0.0] * world_size
    parts = [[] for _ in range(world_size)]
    for s in order:
        r = min(range(world_size), key=lambda k: (load[k], k))
        parts[r].append(s)
        load[r] += costs[s]
    return [sorted(p) for p in parts]


# ---------------------------------------------------------------------------
# collectives
# ---------------------------------------------------------------------------

def _dist():
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        raise RuntimeError("torch.distributed is not initialised")
    return dist


def _all_gather_sizes(n, device, group):
    """Every rank's integer n, as a Python list in rank order."""
    import torch
    dist = _dist()
    ws = dist.get_world_size(group)
    t = torch.tensor([int(n)], dtype=torch.int64, device=device)
    out = [torch.empty_like(t) for _ in range(ws)]
    dist.all_gather(out, t, group=group)
    return [int(x.item()) for x in out]


def _all_gather_rows(local, sizes, group):
    """Concatenate every rank's rows of `local` (same trailing shape and
    dtype on all ranks, row counts `sizes`) on every rank.  Ragged sizes are
    padded to the largest for the collective and cut back afterwards."""
    import torch
    dist = _dist()
    m = max(sizes) if sizes else 0
    pad = torch.zeros((m,) + tuple(local.shape[1:]), dtype=local.dtype,
                      device=local.device)
    pad[:local.shape[0]] = local
    bufs = [torch.empty_like(pad) for _ in sizes]
    dist.all_gather(bufs, pad.contiguous(), group=group)
    return torch.cat([b[:n] for b, n in zip(bufs, sizes)], dim=0)


def gather_positions(local_positions, group=None):
    """All-gather of the ranks' position slices (rank order).  Returns
    (positions of all atoms, this rank's (lo, hi))."""
    dist = _dist()
    rank = dist.get_rank(group)
    sizes = _all_gather_sizes(local_positions.shape[0], local_positions.device, group)
    full = _all_gather_rows(local_positions, sizes, group)
    lo = sum(sizes[:rank])
    return full, (lo, lo + sizes[rank])


def global_pair_offset(n_local, device, group=None):
    """(index of this rank's first pair in the global list, global length)
    from one all-gather of the ranks' pair counts."""
    dist = _dist()
    rank = dist.get_rank(group)
    sizes = _all_gather_sizes(n_local, device, group)
    return sum(sizes[:rank]), sum(sizes)


def gather_pairs(arrays, group=None):
    """Every rank's slice concatenated in rank order, on every rank: the
    single-GPU list.  `arrays` is a sequence of tensors with the same number
    of rows (this rank's pairs)."""
    if not arrays:
        return []
    n = int(arrays[0].shape[0])
    sizes = _all_gather_sizes(n, arrays[0].device, group)
    return [_all_gather_rows(a, sizes, group) for a in arrays]


# ---------------------------------------------------------------------------
# builds
# ---------------------------------------------------------------------------

def neighbour_list_rows(quantities, positions, cell, pbc, cutoff, atom_range, *,
                        numbers=None, cell_origin=None):
    """The rows lo <= i < hi of ``neighbour_list(quantities, positions=...,
    cell=..., pbc=..., cutoff=...)`` for device positions (torch CUDA
    float64 (n, 3)), as torch tensors on that device.  Pairs keep their
    global atom indices."""
    from . import _matscipy_neighbours as _ext
    from .neighbours import _host_metadata, _resolve_cutoff
    pos_t = _ext.import_device_positions(positions)
    nat = pos_t.shape[0]
    lo, hi = (int(atom_range[0]), int(atom_range[1]))
    if not (0 <= lo <= hi <= nat):
        raise ValueError(f"atom range [{lo}, {hi}) outside [0, {nat})")
    if cell is None:
        raise ValueError("cell must be given for device-resident positions.")
    co, ce, inv, pb, nums = _host_metadata(cell, pbc, numbers, cell_origin, nat)
    cut, nums = _resolve_cutoff(cutoff, nums)
    origin, ce, inv, pbc8 = _ext.coerce_geometry(co, ce, inv, pb)
    rc, per_atom, per_type_sq, ncut = _ext.resolve_cutoff(cut, nat)
    flags = _ext.quantity_flags(quantities)
    bufs = _ext.run_device(quantities, origin, ce, inv, pbc8, pos_t, None, rc,
                           per_atom, per_type_sq, ncut, nums, flags,
                           pos_t.device.index, atom_range=(lo, hi))
    return [bufs[ch] for ch in quantities]


def neighbour_list_sharded(quantities, local_positions, cell, pbc, cutoff, *,
                           numbers=None, cell_origin=None, group=None, gather=False):
    """Row-split build of one system across the ranks of `group`.

    Each rank passes its own contiguous slice of the atoms (rank order; torch
    CUDA float64 (n_r, 3) on its GPU) and, when `numbers` is used, the
    numbers of ALL atoms.  Returns a ShardedList with this rank's rows; with
    gather=True its arrays are instead the whole list (every rank's slice,
    all-gathered), identical to a single-GPU ``neighbour_list``.
    """
    full, rows = gather_positions(local_positions, group)
    arrays = neighbour_list_rows(quantities, full, cell, pbc, cutoff, rows,
                                 numbers=numbers, cell_origin=cell_origin)
    n_local = int(arrays[0].shape[0]) if arrays else 0
    off, total = global_pair_offset(n_local, local_positions.device, group)
    if gather:
        arrays = gather_pairs(arrays, group)
        rows = (0, int(full.shape[0]))
        off = 0
    out = arrays[0] if len(quantities) == 1 else tuple(arrays)
    return ShardedList(out, rows, off, total)


def local_systems(systems, world_size, rank, costs=None):
    """This rank's share of a list of independent systems (dicts as taken by
    ``NeighbourListBatch``) under partition_systems.  Returns (global system
    indices, the systems), ready for ``NeighbourListBatch(..., device=...)``."""
    if costs is None:
        costs = [system_cost(np.asarray(s["positions"]).shape[0], s["cell"],
                             s["cutoff"] if np.ndim(s["cutoff"]) == 0
                             else np.max(s["cutoff"]) * 2.0)
                 for s in systems]
    mine = partition_systems(costs, world_size)[int(rank)]
    return mine, [systems[s] for s in mine]
