"""Host side of the multi-GPU split, on CPU: the partitioners, and the
collectives of a row-split build run as two gloo ranks.  The per-rank pair
build is stood in for by the oracle's rows [lo, hi) (the engine needs a GPU);
the test checks that offsets and gathers put the slices back together as the
full list."""
import os
import socket

import numpy as np
import pytest

from conftest import assert_same_lists


def test_partition_rows_covers_contiguously():
    from matscipy_neighbours import distributed as D
    for nat in (0, 1, 5, 97, 1000):
        for ws in (1, 2, 3, 8):
            r = D.partition_rows(nat, ws)
            assert len(r) == ws and r[0][0] == 0 and r[-1][1] == nat
            assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
            sizes = [hi - lo for lo, hi in r]
            assert max(sizes) - min(sizes) <= 1


def test_partition_rows_weighted_balances_weight():
    from matscipy_neighbours import distributed as D
    rng = np.random.default_rng(0)
    w = rng.integers(0, 60, size=5000).astype(float)
    w[:1000] *= 5.0  # a heavy region at the front
    r = D.partition_rows(5000, 4, weights=w)
    loads = [w[lo:hi].sum() for lo, hi in r]
    assert r[0][0] == 0 and r[-1][1] == 5000
    assert max(loads) - min(loads) <= 2 * w.max()
    with pytest.raises(ValueError):
        D.partition_rows(10, 2, weights=np.ones(9))
    with pytest.raises(ValueError):
        D.partition_rows(10, 0)


def test_partition_systems_lpt():
    from matscipy_neighbours import distributed as D
    rng = np.random.default_rng(1)
    costs = rng.uniform(1, 100, size=300)
    parts = D.partition_systems(costs, 8)
    flat = sorted(s for p in parts for s in p)
    assert flat == list(range(300))
    loads = [costs[p].sum() for p in parts]
    # LPT: no rank exceeds the lightest by more than the largest job
    assert max(loads) - min(loads) <= costs.max()
    assert parts == D.partition_systems(list(costs), 8)  # deterministic
    assert D.partition_systems([], 3) == [[], [], []]
    assert D.partition_systems([5.0], 3) == [[0], [], []]


def test_system_cost_orders_by_pairs():
    from matscipy_neighbours import distributed as D
    small = D.system_cost(100, 10 * np.eye(3), 3.0)
    dense = D.system_cost(800, 10 * np.eye(3), 3.0)
    longer = D.system_cost(100, 10 * np.eye(3), 5.0)
    assert dense > small and longer > small
    assert D.system_cost(10, np.zeros((3, 3)), 3.0) == 100.0


# --- two gloo ranks ----------------------------------------------------------

def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _case():
    rng = np.random.default_rng(7)
    cell = np.array([[9.0, 0, 0], [1.0, 8.5, 0], [0.5, 0.3, 9.5]])
    pos = rng.uniform(0, 1, size=(333, 3)) @ cell
    return dict(cell=cell, positions=pos, cutoff=2.6, pbc=(True, True, False))


def _rank_main(rank, world, port, outdir):
    import torch
    import torch.distributed as dist

    import oracle as O
    from matscipy_neighbours import distributed as D
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        w = _case()
        nat = w["positions"].shape[0]
        # uneven slices: rank 0 takes 100 atoms, rank 1 the rest
        cuts = [0, 100, nat]
        local = torch.from_numpy(w["positions"][cuts[rank]:cuts[rank + 1]].copy())
        full, rows = D.gather_positions(local)
        assert rows == (cuts[rank], cuts[rank + 1])
        assert torch.equal(full, torch.from_numpy(w["positions"]))
        # this rank's rows (the engine's job on a GPU)
        allq = O.oracle_neighbour_list("ijdDS", w["cell"], full.numpy(), w["cutoff"],
                                       w["pbc"])
        sel = (allq[0] >= rows[0]) & (allq[0] < rows[1])
        mine = [torch.from_numpy(np.ascontiguousarray(a[sel])) for a in allq]
        off, total = D.global_pair_offset(len(mine[0]), torch.device("cpu"))
        gathered = D.gather_pairs(mine)
        np.savez(os.path.join(outdir, f"rank{rank}.npz"), off=off, total=total,
                 n=len(mine[0]), *[g.numpy() for g in gathered])
        # a rank with no rows at all
        empty = [a[:0] if rank == 1 else a for a in mine]
        g2 = D.gather_pairs(empty)
        n0 = len(mine[0]) if rank == 0 else off
        assert g2[0].shape[0] == n0
        assert torch.equal(g2[0], gathered[0][:n0])
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_row_split(tmp_path, oracle):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.spawn(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    w = _case()
    want = oracle.oracle_neighbour_list("ijdDS", w["cell"], w["positions"], w["cutoff"],
                                        w["pbc"])
    r0 = np.load(tmp_path / "rank0.npz")
    r1 = np.load(tmp_path / "rank1.npz")
    assert int(r0["off"]) == 0 and int(r1["off"]) == int(r0["n"])
    assert int(r0["total"]) == int(r1["total"]) == len(want[0])
    for r in (r0, r1):
        got = tuple(r[f"arr_{k}"] for k in range(5))
        assert_same_lists(got, want, "ijdDS")
