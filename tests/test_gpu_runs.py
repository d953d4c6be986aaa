"""Work items that join several home cells along x ("runs", launch config
cells_per_item; chosen on the device for sparse dense grids): every run
length gives the oracle's list bit for bit, on sparse systems where runs
form -- orthorhombic and triclinic cells, periodic and open x (runs that touch
the box edge wrap their neighbour cells), few cells along x, scalar,
per-atom and per-type cutoffs, split rows, the neighbour matrix, the force
sink and a batch."""
import ctypes

import numpy as np
import pytest

from conftest import assert_same_lists

pytestmark = pytest.mark.gpu


def _sparse(n, box, pbc, cutoff, seed, tilt=0.0, kind="scalar", zslab=None):
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
    "slab_periodic_xy": _sparse(6000, 80.0, (True, True, False), 4.0, 1, zslab=(0.4, 0.6)),
    "gas_open": _sparse(3000, 70.0, (False, False, False), 3.5, 2),
    "gas_triclinic": _sparse(4000, 60.0, (True, True, True), 3.0, 3, tilt=0.3),
    "few_cells_x": _sparse(100, 13.0, (True, True, True), 4.2, 4),
    "per_atom": _sparse(4000, 60.0, (True, False, True), 4.0, 5, kind="per_atom"),
    "per_type": _sparse(4000, 60.0, (True, True, True), 4.0, 6, kind="per_type"),
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
def plan_config():
    from matscipy_neighbours import _matscipy_neighbours as ext
    plan = ext.plan_for(0)
    prev = ext.set_options()
    ext.set_options(precision="fp32", grid="dense")

    def set_cells(n, tile=0):
        cfg = ext.LaunchConfig(atoms_per_item=tile, cells_per_item=n)
        ext.check(ext.lib.nbl_plan_set_launch_config(plan, ctypes.byref(cfg)))
        back = ext.LaunchConfig()
        ext.check(ext.lib.nbl_plan_get_launch_config(plan, ctypes.byref(back)))
        assert back.cells_per_item == n
    yield set_cells
    ext.check(ext.lib.nbl_plan_set_launch_config(plan, ctypes.byref(ext.LaunchConfig())))
    ext.set_options(precision=prev["precision"], grid=prev["grid"])


@pytest.mark.parametrize("name", list(SYSTEMS))
def test_every_run_length_gives_the_oracles_list(oracle, plan_config, name):
    w = SYSTEMS[name]
    want = _want(oracle, w)
    assert len(want[0]) > 0
    for cells in (0, 1, 2, 3, 5, 8):
        for tile in (0, 9):
            plan_config(cells, tile)
            assert_same_lists(_run(w), want, "ijdDS")


def test_runs_with_split_rows(oracle, plan_config):
    import torch
    from matscipy_neighbours.distributed import neighbour_list_rows
    w = SYSTEMS["slab_periodic_xy"]
    want = _want(oracle, w)
    pos = torch.from_numpy(w["positions"]).cuda()
    n = len(pos)
    plan_config(8)
    parts = [neighbour_list_rows("ijdDS", pos, w["cell"], w["pbc"], w["cutoff"], r)
             for r in ((0, 1000), (1000, 1001), (1001, n))]
    torch.cuda.synchronize()
    got = tuple(np.concatenate([p[k].cpu().numpy() for p in parts]) for k in range(5))
    assert_same_lists(got, want, "ijdDS")


def test_runs_neighbour_matrix_and_force_sink(oracle, plan_config):
    import matscipy_neighbours as m
    w = SYSTEMS["gas_triclinic"]
    plan_config(8)
    i, j, D = _want(oracle, w, "ijD")
    idx, dist, count = (np.asarray(x) for x in m.neighbour_matrix(
        positions=w["positions"], cell=w["cell"], pbc=w["pbc"], cutoff=w["cutoff"],
        max_neighbours=64))
    deg = np.bincount(i, minlength=len(w["positions"]))
    assert np.array_equal(count, deg)
    start = np.concatenate([[0], np.cumsum(deg)])
    for a in range(len(deg)):
        assert np.array_equal(idx[a, :deg[a]], j[start[a]:start[a + 1]])
        assert np.array_equal(dist[a, :deg[a]].view(np.int64),
                              D[start[a]:start[a + 1]].view(np.int64))
    d = np.sqrt((D * D).sum(axis=1))
    s6 = (1.0 / (d * d)) ** 3
    coef = -24.0 * s6 * (2.0 * s6 - 1.0) / (d * d)
    f = np.zeros((len(w["positions"]), 3))
    np.add.at(f, i, coef[:, None] * D)
    e = 0.5 * np.sum(4.0 * (s6 * s6 - s6))
    ge, gf = m.lennard_jones(w["positions"], float(w["cutoff"]), cell=w["cell"], pbc=w["pbc"])
    assert np.allclose(gf, f, rtol=1e-12, atol=1e-12 * np.abs(f).max())
    assert abs(ge - e) <= 1e-12 * max(1.0, abs(e))


def test_runs_in_a_batch(oracle):
    from matscipy_neighbours.batch import NeighbourListBatch
    systems = [dict(SYSTEMS[k]) for k in ("slab_periodic_xy", "gas_triclinic", "few_cells_x")]
    for s in systems:
        s.pop("types")
    want = [_want(oracle, dict(s, types=None)) for s in systems]
    b = NeighbourListBatch(systems, precision="fp32", grid="dense", graph=True, autotune=False)
    b.run()
    b.run()
    off = b.sys_offsets()
    outs = [t.cpu().numpy() for t in b.results()]
    b.close()
    for s in range(len(systems)):
        assert_same_lists(tuple(o[off[s]:off[s + 1]] for o in outs), want[s], "ijdDS")


def test_cells_per_item_out_of_range_is_refused():
    from matscipy_neighbours import _matscipy_neighbours as ext
    plan = ext.plan_for(0)
    for bad in (-1, 9):
        cfg = ext.LaunchConfig(cells_per_item=bad)
        assert ext.lib.nbl_plan_set_launch_config(plan, ctypes.byref(cfg)) == \
            ext.NBL_ERROR_INVALID_ARGUMENT
