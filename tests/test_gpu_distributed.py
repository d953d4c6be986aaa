"""Row-split and system-split builds on one GPU: the slices that ranks would
build, made one after another, concatenate to the oracle's full list bit for
bit (same arrays, same order)."""
import itertools
import socket

import numpy as np
import pytest

from conftest import assert_same_lists

pytestmark = pytest.mark.gpu

MODES = list(itertools.product(["fp32", "fp64"], ["dense", "morton", "hashed"]))


@pytest.fixture(autouse=True)
def _restore_options():
    from matscipy_neighbours import set_options
    prev = set_options()
    yield
    set_options(precision=prev["precision"], grid=prev["grid"])


def _workloads():
    from matscipy_neighbours import _workloads as W
    rng = np.random.default_rng(3)
    r = rng.uniform(0, 1.6, size=900)
    r[::5] = 0.0
    types = rng.integers(0, 3, size=700).astype(np.int32)
    return [
        ("fcc_bulk_12", W.fcc_bulk(reps=12)),
        ("slab_8k", W.sparse_slab(n=8000)),
        ("diff_lattice_12", W.diff_lattice(shape=(12, 12, 6))),
        ("per_atom_mixed_pbc", dict(cell=12 * np.eye(3),
                                    positions=rng.uniform(0, 12, size=(900, 3)),
                                    cutoff=r, pbc=(True, False, True))),
        ("per_type", dict(cell=11 * np.eye(3), positions=rng.uniform(0, 11, size=(700, 3)),
                          cutoff=np.array([[2.0, 2.5, 3.0], [2.5, 1.0, 0.0],
                                           [3.0, 0.0, 3.5]]),
                          pbc=True, types=types)),
        ("one_dense_cell", dict(cell=40 * np.eye(3),
                                positions=rng.uniform(10, 10.5, size=(1200, 3)),
                                cutoff=3.0, pbc=True)),
    ]


WL = _workloads()


def _expected(oracle, w, q="ijdDS"):
    return oracle.oracle_neighbour_list(q, w["cell"], w["positions"], w["cutoff"],
                                        w["pbc"], types=w.get("types"))


def _rows(w, rng_pair, q="ijdDS"):
    import torch
    from matscipy_neighbours import distributed as D
    pos = torch.from_numpy(np.ascontiguousarray(w["positions"], dtype=np.float64)).cuda()
    pbc = np.broadcast_to(np.asarray(w["pbc"], dtype=bool), (3,))
    out = D.neighbour_list_rows(q, pos, np.asarray(w["cell"], dtype=float), pbc,
                                w["cutoff"], rng_pair, numbers=w.get("types"))
    torch.cuda.synchronize()
    return [t.cpu().numpy() for t in out]


def _concat(parts):
    return tuple(np.concatenate([p[k] for p in parts], axis=0) for k in range(len(parts[0])))


@pytest.mark.parametrize("mode", MODES, ids=["-".join(m) for m in MODES])
@pytest.mark.parametrize("name,w", WL, ids=[n for n, _ in WL])
def test_row_split_concatenates_to_full_list(oracle, name, w, mode):
    import matscipy_neighbours as m
    from matscipy_neighbours import distributed as D
    m.set_options(precision=mode[0], grid=mode[1])
    nat = np.asarray(w["positions"]).shape[0]
    want = _expected(oracle, w)
    for ranges in (D.partition_rows(nat, 4),
                   D.partition_rows(nat, 3, weights=np.bincount(want[0], minlength=nat))):
        parts = []
        for lo, hi in ranges:
            p = _rows(w, (lo, hi))
            assert np.all((p[0] >= lo) & (p[0] < hi))
            parts.append(p)
        assert_same_lists(_concat(parts), want, "ijdDS")


def test_row_ranges_edges(oracle):
    w = WL[0][1]
    nat = np.asarray(w["positions"]).shape[0]
    want = _expected(oracle, w)
    full = _rows(w, (0, nat))
    assert_same_lists(tuple(full), want, "ijdDS")
    for lo, hi in [(0, 0), (nat, nat), (17, 17)]:
        got = _rows(w, (lo, hi))
        assert all(len(a) == 0 for a in got)
    # one row, and a range that starts mid-cell and ends mid-cell
    for lo, hi in [(5, 6), (123, 1234)]:
        got = _rows(w, (lo, hi))
        sel = (want[0] >= lo) & (want[0] < hi)
        assert_same_lists(tuple(got), tuple(a[sel] for a in want), "ijdDS")
    with pytest.raises(ValueError):
        _rows(w, (10, 5))
    with pytest.raises(ValueError):
        _rows(w, (0, nat + 1))


def test_range_does_not_leak_into_later_calls(oracle):
    """A row-split build leaves this thread's plan building full lists."""
    import matscipy_neighbours as m
    w = WL[1][1]
    _rows(w, (10, 20))
    got = m.neighbour_list("ijdDS", positions=np.asarray(w["positions"], dtype=float),
                           cell=w["cell"], pbc=w["pbc"], cutoff=w["cutoff"])
    assert_same_lists(got, _expected(oracle, w), "ijdDS")


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_sharded_single_rank_nccl(oracle):
    """neighbour_list_sharded through a real NCCL group of one rank: the
    all-gathers, offsets and (gather=True) output gather are the identity."""
    import torch
    import torch.distributed as dist
    from matscipy_neighbours import distributed as D
    w = WL[0][1]
    pos = torch.from_numpy(np.asarray(w["positions"], dtype=np.float64)).cuda()
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}",
                            rank=0, world_size=1, device_id=torch.device("cuda", 0))
    try:
        want = _expected(oracle, w)
        sl = D.neighbour_list_sharded("ijdDS", pos, w["cell"], w["pbc"], w["cutoff"])
        assert sl.atom_range == (0, pos.shape[0])
        assert sl.pair_offset == 0 and sl.total_pairs == len(want[0])
        assert_same_lists(tuple(t.cpu().numpy() for t in sl.arrays), want, "ijdDS")
        sl = D.neighbour_list_sharded("ij", pos, w["cell"], w["pbc"], w["cutoff"],
                                      gather=True)
        assert_same_lists(tuple(t.cpu().numpy() for t in sl.arrays), want[:2], "ij")
    finally:
        dist.destroy_process_group()


def test_system_split_batches(oracle):
    """Systems dealt to 3 ranks by partition_systems, each rank's share built
    as one batch: every system matches the oracle."""
    import torch
    from matscipy_neighbours import _workloads as W
    from matscipy_neighbours.batch import NeighbourListBatch
    from matscipy_neighbours import distributed as D
    systems = W.batched_systems(nsys=20, seed=9, nmax=256)
    seen = []
    for rank in range(3):
        ids, mine = D.local_systems(systems, 3, rank)
        seen += ids
        if not mine:
            continue
        b = NeighbourListBatch(mine, "ijdDS", autotune=False)
        b.run()
        torch.cuda.synchronize()
        for k, s in enumerate(ids):
            got = tuple(t.cpu().numpy() for t in b.system(k))
            want = oracle.oracle_neighbour_list("ijdDS", systems[s]["cell"],
                                                systems[s]["positions"],
                                                systems[s]["cutoff"], systems[s]["pbc"])
            assert_same_lists(got, want, "ijdDS")
        b.close()
    assert sorted(seen) == list(range(len(systems)))
