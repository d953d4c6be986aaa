"""Batches: every system's pairs equal the oracle's for that system alone,
through one launch (and a replayed CUDA graph), with in-place position
updates and capacity growth."""
import numpy as np
import pytest

from conftest import assert_same_lists

pytestmark = pytest.mark.gpu


def _systems(nsys=40, seed=3, nmax=256):
    from matscipy_neighbours import _workloads as W
    return W.batched_systems(nsys=nsys, seed=seed, nmax=nmax)


def _check(oracle, b, systems, q="ijdDS"):
    off = b.sys_offsets()
    outs = [t.cpu().numpy() for t in b.results()]
    for s, sd in enumerate(systems):
        got = tuple(o[off[s]:off[s + 1]] for o in outs)
        want = oracle.oracle_neighbour_list(q, sd["cell"], sd["positions"], sd["cutoff"],
                                            sd["pbc"], types=sd.get("numbers"))
        assert_same_lists(got, want, q)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("graph", [True, False])
def test_batch_matches_oracle_per_system(oracle, precision, graph):
    from matscipy_neighbours.batch import NeighbourListBatch
    systems = _systems()
    b = NeighbourListBatch(systems, precision=precision, graph=graph, autotune=False)
    b.run()
    _check(oracle, b, systems)
    b.run()  # replay: same answer
    _check(oracle, b, systems)
    b.close()


def test_batch_scalar_cutoffs_and_grids(oracle):
    from matscipy_neighbours.batch import NeighbourListBatch
    rng = np.random.default_rng(9)
    systems = []
    for k in range(25):
        n = int(rng.integers(1, 300))
        L = float(rng.uniform(6, 20))
        cell = np.diag([L, L * rng.uniform(0.8, 1.2), L])
        cell[1, 0] = rng.uniform(-2, 2)
        systems.append(dict(positions=rng.uniform(0, 1, size=(n, 3)) @ cell, cell=cell,
                            pbc=rng.integers(0, 2, size=3).astype(bool),
                            cutoff=float(rng.uniform(1.5, 4.0))))
    for grid in ("dense", "morton", "hashed"):
        b = NeighbourListBatch(systems, grid=grid, autotune=False)
        b.run()
        _check(oracle, b, systems)
        b.close()


def test_batch_per_type(oracle):
    from matscipy_neighbours.batch import NeighbourListBatch
    rng = np.random.default_rng(5)
    table = np.array([[1.5, 2.5], [2.5, 3.0]])
    systems = []
    for k in range(12):
        n = int(rng.integers(20, 200))
        L = float(rng.uniform(8, 14))
        systems.append(dict(positions=rng.uniform(0, L, size=(n, 3)),
                            cell=L * np.eye(3), pbc=True, cutoff=table,
                            numbers=rng.integers(0, 2, size=n).astype(np.int32)))
    b = NeighbourListBatch(systems, quantities="ijdD", autotune=False)
    b.run()
    _check(oracle, b, systems, q="ijdD")
    b.close()


def test_batch_positions_update_in_place_and_capacity_growth(oracle):
    from matscipy_neighbours.batch import NeighbourListBatch
    systems = _systems(nsys=16, seed=11)
    b = NeighbourListBatch(systems, capacity=1000, autotune=False)  # too small
    b.run()  # grows and rebuilds
    assert b.capacity >= b.npairs
    _check(oracle, b, systems)
    rng = np.random.default_rng(2)
    moved = []
    for s, sd in enumerate(systems):
        d = dict(sd)
        d["positions"] = sd["positions"] + rng.normal(0, 0.3, size=sd["positions"].shape)
        moved.append(d)
    import torch
    new = torch.from_numpy(np.concatenate([m["positions"] for m in moved])).cuda()
    b.positions.copy_(new)
    b.run()
    _check(oracle, b, moved)
    b.close()


def test_batch_autotune_picks_a_config(oracle):
    from matscipy_neighbours.batch import NeighbourListBatch
    systems = _systems(nsys=24, seed=4)
    b = NeighbourListBatch(systems, autotune=True)
    cm, grp, fm = b.config()
    # CTAs per SM: 1, 2 or 4 waves of each kernel's resident CTAs
    assert 1 <= cm <= 64 and grp in (2, 4) and 1 <= fm <= 64
    assert all(isinstance(t, bool) for t in b.tickets())
    lc = b.launch_config()
    assert lc["count_warps"] in (2, 4, 8) and lc["fill_warps"] in (2, 4, 8)
    assert lc["atoms_per_item"] in (16, 32) and lc["count_large_staging"] in (0, 1)
    assert lc["count_group"] == grp and lc["count_ctas_per_sm"] == cm
    assert lc["count_candidates_per_warp"] in (384, 768)
    assert lc["tuned_count_ms"] > 0 and lc["tuned_fill_ms"] > 0
    b.run()
    _check(oracle, b, systems)
    b.close()
