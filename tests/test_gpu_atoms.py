"""The thread-per-atom pair passes (launch config thread_per_atom;
nbl_trav_atoms.cu), chosen by default on dilute grids (fewer atoms than
cells): bit for bit the
oracle's list on sparse and dense systems, every grid layout (the home cell
is recovered from dense, Morton and hashed sort keys), scalar, per-atom and
per-type cutoffs, split rows, the neighbour matrix, quantity subsets,
batches of several systems, the force sink (which keeps the work items) and
the default choice on the sparse slab."""
import ctypes

import numpy as np
import pytest

from conftest import assert_same_lists

pytestmark = pytest.mark.gpu


def _system(n, box, pbc, cutoff, seed, tilt=0.0, kind="scalar", zslab=None):
    rng = np.random.default_rng(seed)
    cell = np.diag([box, box, box]).astype(float)
    cell[1, 0] = tilt * box
    cell[2, 0] = 0.5 * tilt * box
    frac = rng.uniform(0.0, 1.0, size=(n, 3))
    if zslab is not None:
        frac[:, 2] = rng.uniform(zslab[0], zslab[1], size=n)
    w = dict(positions=np.ascontiguousarray(frac @ cell), cell=cell,
             pbc=np.array(pbc), cutoff=cutoff, types=None)
    if kind == "per_atom":
        w["cutoff"] = rng.uniform(0.4 * cutoff, 0.5 * cutoff, size=n)
    elif kind == "per_type":
        w["types"] = rng.integers(0, 2, size=n).astype(np.int32)
        w["cutoff"] = np.array([[0.6, 0.8], [0.8, 1.0]]) * cutoff
    return w


SYSTEMS = {
    "slab_periodic_xy": _system(6000, 80.0, (True, True, False), 4.0, 1, zslab=(0.4, 0.6)),
    "gas_open": _system(3000, 70.0, (False, False, False), 3.5, 2),
    "gas_triclinic": _system(4000, 60.0, (True, True, True), 3.0, 3, tilt=0.3),
    "few_cells": _system(300, 9.0, (True, True, True), 4.2, 4),
    "per_atom": _system(4000, 60.0, (True, False, True), 4.0, 5, kind="per_atom"),
    "per_type": _system(4000, 60.0, (True, True, True), 4.0, 6, kind="per_type"),
    "dense_bulk": _system(4000, 30.0, (True, True, True), 4.5, 7, tilt=0.2),
}


def _want(oracle, w, q="ijdDS"):
    return oracle.oracle_neighbour_list(q, w["cell"], w["positions"], w["cutoff"], w["pbc"],
                                        types=w["types"])


def _run(w, q="ijdDS"):
    import torch
    import matscipy_neighbours as m
    pos = torch.from_numpy(w["positions"]).cuda()
    kw = {} if w["types"] is None else {"numbers": w["types"]}
    out = m.neighbour_list(q, positions=pos, cell=w["cell"], pbc=w["pbc"], cutoff=w["cutoff"],
                           array_namespace=torch, **kw)
    torch.cuda.synchronize()
    out = out if len(q) > 1 else (out,)
    return tuple(t.cpu().numpy() for t in out)


@pytest.fixture
def atoms_on():
    """Thread-per-atom passes forced on (one-launch count phase off)."""
    from matscipy_neighbours import _matscipy_neighbours as ext
    plan = ext.plan_for(0)
    prev = ext.set_options()
    cfg = ext.LaunchConfig(thread_per_atom=1, one_launch_atoms=-1)
    ext.check(ext.lib.nbl_plan_set_launch_config(plan, ctypes.byref(cfg)))
    back = ext.LaunchConfig()
    ext.check(ext.lib.nbl_plan_get_launch_config(plan, ctypes.byref(back)))
    assert back.thread_per_atom == 1
    yield ext
    ext.check(ext.lib.nbl_plan_set_launch_config(plan, ctypes.byref(ext.LaunchConfig())))
    ext.set_options(precision=prev["precision"], grid=prev["grid"])


@pytest.mark.parametrize("grid", ["dense", "morton", "hashed"])
@pytest.mark.parametrize("name", list(SYSTEMS))
def test_every_grid_gives_the_oracles_list(oracle, atoms_on, name, grid):
    w = SYSTEMS[name]
    want = _want(oracle, w)
    assert len(want[0]) > 0
    for precision in ("fp32", "fp64"):
        atoms_on.set_options(precision=precision, grid=grid)
        assert_same_lists(_run(w), want, "ijdDS")


@pytest.mark.parametrize("q", ["i", "j", "D", "d", "S", "Sdj", "ijdD"])
def test_quantity_subsets(oracle, atoms_on, q):
    w = SYSTEMS["gas_triclinic"]
    got = _run(w, q)
    assert_same_lists(got[0] if len(q) == 1 else got, _want(oracle, w, q), q)


def test_host_positions_and_repeated_calls(oracle, atoms_on):
    import matscipy_neighbours as m
    for name in ("slab_periodic_xy", "per_type", "slab_periodic_xy"):
        w = SYSTEMS[name]
        kw = {} if w["types"] is None else {"numbers": w["types"]}
        got = m.neighbour_list("ijdDS", positions=w["positions"], cell=w["cell"], pbc=w["pbc"],
                               cutoff=w["cutoff"], **kw)
        assert_same_lists(got, _want(oracle, w), "ijdDS")


def test_split_rows(oracle, atoms_on):
    import torch
    from matscipy_neighbours.distributed import neighbour_list_rows
    w = SYSTEMS["slab_periodic_xy"]
    want = _want(oracle, w)
    pos = torch.from_numpy(w["positions"]).cuda()
    n = len(pos)
    parts = [neighbour_list_rows("ijdDS", pos, w["cell"], w["pbc"], w["cutoff"], r)
             for r in ((0, 1000), (1000, 1001), (1001, n))]
    torch.cuda.synchronize()
    got = tuple(np.concatenate([p[k].cpu().numpy() for p in parts]) for k in range(5))
    assert_same_lists(got, want, "ijdDS")


def test_neighbour_matrix_and_force_sink(oracle, atoms_on):
    import matscipy_neighbours as m
    w = SYSTEMS["gas_triclinic"]
    i, j, D = _want(oracle, w, "ijD")
    from torch.utils.dlpack import from_dlpack
    cell = np.asarray(w["cell"], dtype=float)
    for K in (64, 3):
        *caps, overflow = atoms_on.neighbour_matrix_dlpack(
            np.zeros(3), cell, np.linalg.inv(cell.T), w["pbc"], w["positions"],
            w["cutoff"], K)
        idx, dist, count = (from_dlpack(c).cpu().numpy() for c in caps)
        assert overflow == (K < 64)
        deg = np.bincount(i, minlength=len(w["positions"]))
        assert np.array_equal(count, deg)
        start = np.concatenate([[0], np.cumsum(deg)])
        for a in range(len(deg)):
            k = min(deg[a], K)
            assert np.array_equal(idx[a, :k], j[start[a]:start[a] + k])
            assert np.array_equal(dist[a, :k].view(np.int64),
                                  D[start[a]:start[a] + k].view(np.int64))
    # the force sink keeps the warp work items and is unaffected by the setting
    d = np.sqrt((D * D).sum(axis=1))
    s6 = (1.0 / (d * d)) ** 3
    coef = -24.0 * s6 * (2.0 * s6 - 1.0) / (d * d)
    f = np.zeros((len(w["positions"]), 3))
    np.add.at(f, i, coef[:, None] * D)
    e = 0.5 * np.sum(4.0 * (s6 * s6 - s6))
    ge, gf = m.lennard_jones(w["positions"], float(w["cutoff"]), cell=w["cell"], pbc=w["pbc"])
    assert np.allclose(gf, f, rtol=1e-12, atol=1e-12 * np.abs(f).max())
    assert abs(ge - e) <= 1e-12 * max(1.0, abs(e))
    # and a list after the force sink is still the oracle's
    assert_same_lists(_run(w), _want(oracle, w), "ijdDS")


def test_batch_of_dilute_systems(oracle):
    """Several dilute systems in one batch take the thread-per-atom passes by
    default (the system of each atom from the atom bases)."""
    from matscipy_neighbours.batch import NeighbourListBatch
    systems = [dict(SYSTEMS[k]) for k in ("slab_periodic_xy", "gas_open", "gas_triclinic")]
    for s in systems:
        s.pop("types")
    want = [_want(oracle, dict(s, types=None)) for s in systems]
    for grid in ("dense", "hashed"):
        b = NeighbourListBatch(systems, precision="fp32", grid=grid, graph=True,
                               autotune=False)
        b.run()
        b.run()
        off = b.sys_offsets()
        outs = [t.cpu().numpy() for t in b.results()]
        b.close()
        for s in range(len(systems)):
            assert_same_lists(tuple(o[off[s]:off[s + 1]] for o in outs), want[s], "ijdDS")


def test_default_choice_on_the_slab(oracle):
    """The default (0) takes the thread-per-atom passes on the sparse slab
    and the warp passes on dense bulk; both give the oracle's list."""
    from matscipy_neighbours import _matscipy_neighbours as ext
    from matscipy_neighbours import _workloads as W
    plan = ext.plan_for(0)
    w = W.sparse_slab(n=20000)
    sw = dict(positions=w["positions"], cell=w["cell"], pbc=w["pbc"], cutoff=w["cutoff"],
              types=np.ascontiguousarray(w["numbers"], dtype=np.int32))
    want = _want(oracle, sw, "ijdD")
    launches = {}
    try:
        for setting in (-1, 0):
            cfg = ext.LaunchConfig(thread_per_atom=setting)
            ext.check(ext.lib.nbl_plan_set_launch_config(plan, ctypes.byref(cfg)))
            ext.lib.nbl_launch_count(1)
            assert_same_lists(_run(sw, "ijdD"), want, "ijdD")
            launches[setting] = ext.lib.nbl_launch_count(1)
    finally:
        ext.check(ext.lib.nbl_plan_set_launch_config(plan, ctypes.byref(ext.LaunchConfig())))
    # the default skips the work-item builder (k_tiles): one launch fewer
    assert launches[0] == launches[-1] - 1


def test_thread_per_atom_out_of_range_is_refused():
    from matscipy_neighbours import _matscipy_neighbours as ext
    plan = ext.plan_for(0)
    for bad in (-2, 2):
        cfg = ext.LaunchConfig(thread_per_atom=bad)
        assert ext.lib.nbl_plan_set_launch_config(plan, ctypes.byref(cfg)) == \
            ext.NBL_ERROR_INVALID_ARGUMENT


def test_default_learns_the_occupied_cells(oracle):
    """The full-size slab has fewer atoms than cells but 2.3 atoms per occupied
    cell: its first call (occupancy unknown) takes the thread-per-atom passes,
    the next one, knowing the occupied cells from the first count, the warp
    passes (one launch more: the work-item builder).  Both give the oracle's
    list."""
    from matscipy_neighbours import _matscipy_neighbours as ext
    from matscipy_neighbours import _workloads as W
    plan = ext.plan_for(0)
    ext.check(ext.lib.nbl_plan_set_launch_config(plan, ctypes.byref(ext.LaunchConfig())))
    w = W.sparse_slab()
    sw = dict(positions=w["positions"], cell=w["cell"], pbc=w["pbc"], cutoff=w["cutoff"],
              types=np.ascontiguousarray(w["numbers"], dtype=np.int32))
    want = _want(oracle, sw, "ijdD")
    _run(SYSTEMS["few_cells"])  # another system's sizes: the slab's occupancy is unknown
    launches = []
    for _ in range(2):
        ext.lib.nbl_launch_count(1)
        assert_same_lists(_run(sw, "ijdD"), want, "ijdD")
        launches.append(ext.lib.nbl_launch_count(1))
    assert launches[1] == launches[0] + 1
