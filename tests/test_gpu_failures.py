"""Error paths, made to fail on the host (nbl_debug_inject) so that no GPU is
ever faulted: a device workspace that cannot grow must come back as
NBL_ERROR_OUT_OF_MEMORY (Python MemoryError) and leave the plan usable and
leak-free; a hashed cell table with fewer slots than occupied cells must make
the bounded probe give up and the call return NBL_ERROR_INTERNAL (Python
RuntimeError) instead of hanging.  The reference aborts the process on device
errors instead (src/libneighbours/device.hh:68-74).  After each failure the
same request succeeds and matches the oracle bit for bit."""
import ctypes

import numpy as np
import pytest

from conftest import assert_same_lists

pytestmark = pytest.mark.gpu

INJECT_ALLOC_FAILURES = 1
INJECT_HASH_CAPACITY = 2


def _ext():
    from matscipy_neighbours import _matscipy_neighbours as ext
    ext.lib.nbl_debug_inject.argtypes = [ctypes.c_int, ctypes.c_int64]
    ext.lib.nbl_debug_inject.restype = ctypes.c_int
    return ext


@pytest.fixture(autouse=True)
def _clear_injections():
    ext = _ext()
    prev = ext.set_options()
    yield
    ext.check(ext.lib.nbl_debug_inject(INJECT_ALLOC_FAILURES, 0))
    ext.check(ext.lib.nbl_debug_inject(INJECT_HASH_CAPACITY, 0))
    ext.set_options(precision=prev["precision"], grid=prev["grid"])


def _system(n=3000, seed=0):
    rng = np.random.default_rng(seed)
    L = (n / 0.08) ** (1.0 / 3.0)
    cell = np.array([[L, 0.0, 0.0], [0.1 * L, L, 0.0], [0.0, 0.2 * L, L]])
    return dict(positions=np.ascontiguousarray(rng.uniform(0, 1, size=(n, 3)) @ cell),
                cell=cell, pbc=np.array([True, True, False]), cutoff=3.5)


def _request(ext, w, keep):
    cell = np.ascontiguousarray(w["cell"])
    inv = np.ascontiguousarray(np.linalg.inv(cell.T))
    pbc = np.ascontiguousarray(w["pbc"].astype(np.uint8))
    origin = np.zeros(3)
    pos = w["positions"]
    keep.extend([cell, inv, pbc, origin, pos])
    return ext.make_request(31, origin, cell, inv, pbc, len(pos),
                            ctypes.c_void_p(pos.ctypes.data), False, w["cutoff"], None,
                            None, 0, None, 0)


def test_workspace_allocation_failure_is_memory_error_and_recovers(oracle):
    import torch
    ext = _ext()
    torch.cuda.set_device(0)
    w = _system()
    keep = []
    req = _request(ext, w, keep)
    n = ctypes.c_int64()
    # one complete call first, so that the library's module (and its static
    # device data) is loaded before free memory is measured
    plan = ctypes.c_void_p()
    ext.check(ext.lib.nbl_plan_create(0, ctypes.byref(plan)))
    ext.check(ext.lib.nbl_count(plan, ctypes.byref(req), None, ctypes.byref(n)))
    ext.check(ext.lib.nbl_plan_destroy(plan))
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    free0 = torch.cuda.mem_get_info()[0]
    plan = ctypes.c_void_p()
    ext.check(ext.lib.nbl_plan_create(0, ctypes.byref(plan)))
    try:
        ext.check(ext.lib.nbl_debug_inject(INJECT_ALLOC_FAILURES, 1))
        st = ext.lib.nbl_count(plan, ctypes.byref(req), None, ctypes.byref(n))
        assert st == ext.NBL_ERROR_OUT_OF_MEMORY
        assert b"injected" in ext.lib.nbl_last_error()
        with pytest.raises(MemoryError):
            ext.check(st)
        # nothing of the failed call is kept: a fill now has no count to use
        o = ext.Outputs()
        assert ext.lib.nbl_fill(plan, ctypes.byref(o), None) == ext.NBL_ERROR_INVALID_ARGUMENT
        # the same request succeeds once memory is available again
        ext.check(ext.lib.nbl_count(plan, ctypes.byref(req), None, ctypes.byref(n)))
        outs = {"i": torch.empty(n.value, dtype=torch.int32, device="cuda"),
                "j": torch.empty(n.value, dtype=torch.int32, device="cuda"),
                "D": torch.empty((n.value, 3), dtype=torch.float64, device="cuda"),
                "d": torch.empty(n.value, dtype=torch.float64, device="cuda"),
                "S": torch.empty((n.value, 3), dtype=torch.int32, device="cuda")}
        o = ext._outputs_struct(outs, lambda t: t.data_ptr())
        ext.check(ext.lib.nbl_fill(plan, ctypes.byref(o), None))
        ext.check(ext.lib.nbl_check(plan, None))
        got = tuple(outs[q].cpu().numpy() for q in "ijdDS")
        want = oracle.oracle_neighbour_list("ijdDS", w["cell"], w["positions"], w["cutoff"],
                                            w["pbc"])
        assert_same_lists(got, want, "ijdDS")
        del outs
    finally:
        ext.check(ext.lib.nbl_plan_destroy(plan))
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    # no device memory left behind by the failed call or the retry (the
    # plan's pinned host staging is host memory; allow driver granularity)
    assert abs(torch.cuda.mem_get_info()[0] - free0) < (8 << 20)


def test_public_api_raises_memory_error_then_works(oracle):
    import matscipy_neighbours as m
    ext = _ext()
    w = _system(n=2000, seed=3)
    ext.check(ext.lib.nbl_plan_trim(ext.plan_for(0)))  # the next call must grow
    ext.check(ext.lib.nbl_debug_inject(INJECT_ALLOC_FAILURES, 1))
    with pytest.raises(MemoryError):
        m.neighbour_list("ijdDS", positions=w["positions"], cell=w["cell"], pbc=w["pbc"],
                         cutoff=w["cutoff"])
    got = m.neighbour_list("ijdDS", positions=w["positions"], cell=w["cell"], pbc=w["pbc"],
                           cutoff=w["cutoff"])
    want = oracle.oracle_neighbour_list("ijdDS", w["cell"], w["positions"], w["cutoff"],
                                        w["pbc"])
    assert_same_lists(got, want, "ijdDS")


def _sparse(n=400, seed=5):
    rng = np.random.default_rng(seed)
    return dict(positions=rng.uniform(0, 200, size=(n, 3)), cell=200.0 * np.eye(3),
                pbc=np.array([True, True, True]), cutoff=4.0)


def test_hash_probe_runs_out_and_reports_internal_error(oracle):
    import matscipy_neighbours as m
    ext = _ext()
    w = _sparse()
    m.set_options(grid="hashed")
    ext.check(ext.lib.nbl_debug_inject(INJECT_HASH_CAPACITY, 16))  # << occupied cells
    with pytest.raises(RuntimeError, match="device-side bound"):
        m.neighbour_list("ijdDS", positions=w["positions"], cell=w["cell"], pbc=w["pbc"],
                         cutoff=w["cutoff"])
    ext.check(ext.lib.nbl_debug_inject(INJECT_HASH_CAPACITY, 0))
    got = m.neighbour_list("ijdDS", positions=w["positions"], cell=w["cell"], pbc=w["pbc"],
                           cutoff=w["cutoff"])
    want = oracle.oracle_neighbour_list("ijdDS", w["cell"], w["positions"], w["cutoff"],
                                        w["pbc"])
    assert_same_lists(got, want, "ijdDS")


def test_hash_probe_runs_out_in_a_batch(oracle):
    from matscipy_neighbours.batch import NeighbourListBatch
    ext = _ext()
    systems = [_sparse(n=300, seed=s) for s in range(4)]
    ext.check(ext.lib.nbl_debug_inject(INJECT_HASH_CAPACITY, 64))
    b = NeighbourListBatch(systems, grid="hashed", graph=False, autotune=False,
                           capacity=1 << 16)
    try:
        with pytest.raises(RuntimeError, match="device-side bound"):
            b.run()
    finally:
        b.close()
    ext.check(ext.lib.nbl_debug_inject(INJECT_HASH_CAPACITY, 0))
    b = NeighbourListBatch(systems, grid="hashed", graph=False, autotune=False)
    b.run()
    off = b.sys_offsets()
    outs = [t.cpu().numpy() for t in b.results()]
    b.close()
    for s, sd in enumerate(systems):
        want = oracle.oracle_neighbour_list("ijdDS", sd["cell"], sd["positions"],
                                            sd["cutoff"], sd["pbc"])
        assert_same_lists(tuple(o[off[s]:off[s + 1]] for o in outs), want, "ijdDS")
