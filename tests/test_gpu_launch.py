"""nbl_plan_set_launch: the grids of the pair passes are a tuning knob only.
Every launch configuration gives the same arrays, bit for bit, and bad
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
