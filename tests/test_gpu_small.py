"""The one-launch count phase of small systems (nbl_small.cu; by default up to
128 atoms in one CTA, up to 2048 on request in a cluster of CTAs): it is taken when
the system qualifies (one launch for the whole count phase), leaves the same
buffers as the multi-kernel sequence -- the fill, the per-atom counts, the row
offsets and the neighbour matrix that follow give the oracle's results bit
for bit -- and is left for larger systems, sparse grids with many cells, row
slices and batches."""
import ctypes

import numpy as np
import pytest

from conftest import assert_same_lists

pytestmark = pytest.mark.gpu


def _system(n, seed, box=None, kind="scalar", pbc=(True, True, True)):
    rng = np.random.default_rng(seed)
    box = box or (n / 0.085) ** (1.0 / 3.0)
    cell = np.array([[box, 0.0, 0.0], [0.2 * box, box, 0.0], [0.1 * box, -0.15 * box, box]])
    w = dict(positions=np.ascontiguousarray(rng.uniform(0, 1, size=(n, 3)) @ cell), cell=cell,
             pbc=np.array(pbc), cutoff=3.7, types=None)
    if kind == "per_atom":
        w["cutoff"] = rng.uniform(1.0, 1.9, size=n)
    elif kind == "per_type":
        w["types"] = rng.integers(0, 3, size=n).astype(np.int32)
        w["cutoff"] = np.array([[2.0, 2.6, 3.0], [2.6, 3.3, 2.2], [3.0, 2.2, 3.7]])
    return w


def _launches_of_call(ext, w, precision):
    """Kernel launches of one nbl_count + nbl_fill through the C-ABI."""
    import torch
    ext.set_options(precision=precision, grid="auto")
    cell = np.ascontiguousarray(w["cell"], dtype=float)
    inv = np.ascontiguousarray(np.linalg.inv(cell.T))
    pbc = np.ascontiguousarray(np.asarray(w["pbc"], dtype=np.uint8))
    origin = np.zeros(3)
    pos = w["positions"]
    rc, pa, pt, nc = ext.resolve_cutoff(w["cutoff"], len(pos))
    keep = [cell, inv, pbc, origin, pa, pt, w["types"]]
    req = ext.make_request(31, origin, cell, inv, pbc, len(pos), ctypes.c_void_p(pos.ctypes.data),
                           False, rc, pa, pt, nc, w["types"], 0)
    plan = ext.plan_for(0)
    n = ctypes.c_int64()
    ext.check(ext.lib.nbl_count(plan, ctypes.byref(req), None, ctypes.byref(n)))
    bufs = {c: torch.empty((n.value,) + ext._SHAPES[c][0],
                           dtype=torch.int32 if ext._SHAPES[c][1] == np.int32 else torch.float64,
                           device="cuda") for c in "ijdDS"}
    o = ext._outputs_struct(bufs, lambda t: t.data_ptr())
    ext.lib.nbl_launch_count(1)
    ext.check(ext.lib.nbl_count(plan, ctypes.byref(req), None, ctypes.byref(n)))
    ext.check(ext.lib.nbl_fill(plan, ctypes.byref(o), None))
    launches = ext.lib.nbl_launch_count(1)
    torch.cuda.synchronize()
    del keep
    return launches, tuple(bufs[c].cpu().numpy() for c in "ijdDS")


@pytest.fixture
def ext():
    from matscipy_neighbours import _matscipy_neighbours as e
    prev = e.set_options()
    yield e
    e.check(e.lib.nbl_plan_set_launch_config(e.plan_for(0), ctypes.byref(e.LaunchConfig())))
    e.set_options(precision=prev["precision"], grid=prev["grid"])


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("n,kind", [(1, "scalar"), (2, "scalar"), (100, "scalar"),
                                    (128, "per_atom"), (700, "per_atom"), (1500, "per_type"),
                                    (2048, "scalar")])
def test_small_system_is_one_launch_and_matches_the_oracle(oracle, ext, n, kind, precision):
    if n > 128:  # above the default threshold: raise it to the largest allowed
        cfg = ext.LaunchConfig(one_launch_atoms=2048)
        ext.check(ext.lib.nbl_plan_set_launch_config(ext.plan_for(0), ctypes.byref(cfg)))
    w = _system(n, seed=n, kind=kind)
    launches, got = _launches_of_call(ext, w, precision)
    assert launches == 2  # the count phase and the fill
    want = oracle.oracle_neighbour_list("ijdDS", w["cell"], w["positions"], w["cutoff"],
                                        w["pbc"], types=w["types"])
    assert_same_lists(got, want, "ijdDS")


def test_larger_or_sparse_systems_keep_the_multi_kernel_sequence(oracle, ext):
    cfg = ext.LaunchConfig(one_launch_atoms=2048)
    ext.check(ext.lib.nbl_plan_set_launch_config(ext.plan_for(0), ctypes.byref(cfg)))
    for w in (_system(2049, seed=1),                          # too many atoms
              _system(200, seed=2, box=120.0, pbc=(True, True, False))):  # > 16,384 cells
        launches, got = _launches_of_call(ext, w, "fp32")
        assert launches > 2
        want = oracle.oracle_neighbour_list("ijdDS", w["cell"], w["positions"], w["cutoff"],
                                            w["pbc"])
        assert_same_lists(got, want, "ijdDS")


def test_threshold_and_off_switch(ext):
    w = _system(120, seed=3)
    plan = ext.plan_for(0)
    for thr, expect_one in ((0, True), (120, True), (119, False), (-1, False)):
        cfg = ext.LaunchConfig(one_launch_atoms=thr)
        ext.check(ext.lib.nbl_plan_set_launch_config(plan, ctypes.byref(cfg)))
        back = ext.LaunchConfig()
        ext.check(ext.lib.nbl_plan_get_launch_config(plan, ctypes.byref(back)))
        assert back.one_launch_atoms == thr
        launches, _ = _launches_of_call(ext, w, "fp32")
        assert (launches == 2) == expect_one, thr
    for bad in (-2, 2049):
        cfg = ext.LaunchConfig(one_launch_atoms=bad)
        assert ext.lib.nbl_plan_set_launch_config(plan, ctypes.byref(cfg)) == \
            ext.NBL_ERROR_INVALID_ARGUMENT


def test_counts_offsets_and_matrix_after_the_one_cta_count(oracle, ext):
    import matscipy_neighbours as m
    w = _system(125, seed=4)
    i, j, D = oracle.oracle_neighbour_list("ijD", w["cell"], w["positions"], w["cutoff"],
                                           w["pbc"])
    deg = np.bincount(i, minlength=125)
    assert np.array_equal(np.asarray(m.coordination(positions=w["positions"], cell=w["cell"],
                                                    pbc=w["pbc"], cutoff=w["cutoff"])), deg)
    idx, dist, count = (np.asarray(x) for x in m.neighbour_matrix(
        positions=w["positions"], cell=w["cell"], pbc=w["pbc"], cutoff=w["cutoff"],
        max_neighbours=int(deg.max())))
    assert np.array_equal(count, deg)
    start = np.concatenate([[0], np.cumsum(deg)])
    for a in range(125):
        assert np.array_equal(idx[a, :deg[a]], j[start[a]:start[a + 1]])
        assert np.array_equal(dist[a, :deg[a]].view(np.int64),
                              D[start[a]:start[a + 1]].view(np.int64))


def test_non_finite_position_is_a_range_error_on_the_one_cta_path(ext):
    import matscipy_neighbours as m
    pos = np.array([[0.0, 0, 0], [1.0, np.nan, 1]])
    with pytest.raises(RuntimeError):
        m.neighbour_list("ij", positions=pos, cell=5 * np.eye(3), pbc=True, cutoff=1.0)
    out = m.neighbour_list("ij", positions=pos[:1], cell=5 * np.eye(3), pbc=True, cutoff=1.0)
    assert len(out[0]) == 0
