"""nbl_plan_set_launch / nbl_plan_set_launch_config: the launch configuration
of the pair passes (grids, work-item tickets, block size, candidates staged
per warp, atoms per sweep, atoms per work item) is a tuning knob only.  Every
configuration gives the same arrays, bit for bit -- the oracle's -- and bad
values are refused."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lib():
    from matscipy_neighbours import _matscipy_neighbours as ext
    fn = ext.lib.nbl_plan_set_launch
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    fn.restype = ctypes.c_int
    return ext, fn


@pytest.mark.parametrize("cutoff_kind", ["scalar", "per_atom"])
def test_launch_configurations_give_identical_lists(cutoff_kind):
    import torch
    from matscipy_neighbours import _workloads as W
    from matscipy_neighbours import neighbour_list
    ext, set_launch = _lib()
    w = W.fcc_bulk(reps=7, cutoff=4.2)
    pos = torch.from_numpy(np.ascontiguousarray(w["positions"])).cuda()
    cutoff = w["cutoff"]
    if cutoff_kind == "per_atom":
        cutoff = np.random.default_rng(5).uniform(1.6, 2.4, size=pos.shape[0])

    def run():
        out = neighbour_list("ijdDS", positions=pos, cell=w["cell"], pbc=w["pbc"],
                             cutoff=cutoff, array_namespace=torch)
        torch.cuda.synchronize()
        return out

    plan = ext.plan_for(0)
    ref = run()
    assert ref[0].numel() > 0
    try:
        for cfg in [(1, 4, 1), (1, 2, 3), (6, 2, 5), (12, 4, 10), (64, 4, 64)]:
            assert set_launch(plan, *cfg) == 0
            got = run()
            for a, b in zip(ref, got):
                assert torch.equal(a, b), cfg
    finally:
        set_launch(plan, 0, 0, 0)


def test_launch_configuration_rejects_bad_values():
    ext, set_launch = _lib()
    plan = ext.plan_for(0)
    for cfg in [(-1, 4, 0), (0, 3, 0), (0, 4, -2), (65, 4, 0), (0, 4, 65)]:
        assert set_launch(plan, *cfg) == ext.NBL_ERROR_INVALID_ARGUMENT, cfg
    assert set_launch(plan, 0, 0, 0) == 0


def _dense_cells():
    """Cells with more candidates than one staging of the count holds (so the
    large staging and multi-pass sweeps both run) plus an ordinary lattice."""
    from matscipy_neighbours import _workloads as W
    rng = np.random.default_rng(17)
    cluster = dict(positions=rng.uniform(0.0, 6.0, size=(900, 3)), cell=18.0 * np.eye(3),
                   pbc=np.array([True, True, True]), cutoff=2.9)
    return [("cluster", cluster), ("fcc", W.fcc_bulk(reps=5, cutoff=4.0))]


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("name,w", _dense_cells(), ids=[n for n, _ in _dense_cells()])
def test_every_launch_shape_gives_the_oracles_list(oracle, name, w, precision):
    import itertools

    import torch
    from matscipy_neighbours import neighbour_list, set_options
    from conftest import assert_same_lists
    ext, _ = _lib()
    plan = ext.plan_for(0)
    want = oracle.oracle_neighbour_list("ijdDS", w["cell"], w["positions"], w["cutoff"],
                                        w["pbc"])
    pos = torch.from_numpy(np.ascontiguousarray(w["positions"])).cuda()
    prev = set_options(precision=precision)
    tried = 0
    try:
        for cw, big, grp, fw, tile, strided in itertools.product(
                (2, 4, 8), (0, 1), (2, 4), (2, 4, 8), (32, 16, 7), (0, 1)):
            if precision == "fp64" and grp == 2:
                continue
            cfg = ext.LaunchConfig(0, 0, strided, 1 - strided, cw, fw, grp, big, tile)
            assert ext.lib.nbl_plan_set_launch_config(plan, ctypes.byref(cfg)) == 0
            got = neighbour_list("ijdDS", positions=pos, cell=w["cell"], pbc=w["pbc"],
                                 cutoff=w["cutoff"], array_namespace=torch)
            torch.cuda.synchronize()
            assert_same_lists(tuple(t.cpu().numpy() for t in got), want, "ijdDS")
            back = ext.LaunchConfig()
            ext.check(ext.lib.nbl_plan_get_launch_config(plan, ctypes.byref(back)))
            assert back.as_dict() == cfg.as_dict()
            tried += 1
    finally:
        set_options(precision=prev["precision"])
        ext.check(ext.lib.nbl_plan_set_launch_config(plan, ctypes.byref(ext.LaunchConfig())))
    assert tried >= 108


def test_launch_config_rejects_bad_values():
    ext, _ = _lib()
    plan = ext.plan_for(0)
    bad = [dict(count_warps=3), dict(fill_warps=16), dict(count_group=3),
           dict(count_large_staging=2), dict(atoms_per_item=33), dict(atoms_per_item=-1),
           dict(count_ctas_per_sm=65)]
    for b in bad:
        cfg = ext.LaunchConfig(**b)
        assert ext.lib.nbl_plan_set_launch_config(plan, ctypes.byref(cfg)) == \
            ext.NBL_ERROR_INVALID_ARGUMENT, b
    assert ext.lib.nbl_plan_set_launch_config(plan, ctypes.byref(ext.LaunchConfig())) == 0
