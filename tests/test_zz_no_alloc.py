"""nbl_neighbour_list_noalloc: the entry point for callers that cannot allocate
device memory at call time (for example an MD engine whose time-step loop
forbids allocation, or a host whose pool allocator has already reserved the
device memory).  It takes all scratch from a static array inside the library;
the caller provides inputs and output buffers.

Checks, through the C-ABI, that two calls in a row return exactly what the
existing entry point (nbl_count + nbl_fill) returns -- the second call on a
smaller system, so stale contents of the shared scratch would show -- and
that requests beyond the stated limits are refused with a clear error.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lib():
    from matscipy_neighbours import _matscipy_neighbours as ext
    fn = ext.lib.nbl_neighbour_list_noalloc
    fn.argtypes = [ctypes.POINTER(ext.Request), ctypes.POINTER(ext.Outputs),
                   ctypes.c_int64, ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return ext, fn


def _system(n, seed, per_atom=False):
    rng = np.random.default_rng(seed)
    L = (n / 0.085) ** (1.0 / 3.0)
    cell = np.array([[L, 0.0, 0.0], [0.15 * L, L, 0.0], [0.05 * L, 0.1 * L, L]])
    pos = rng.uniform(0, 1, size=(n, 3)) @ cell
    cutoff = rng.uniform(1.0, 2.2, size=n) if per_atom else 4.0
    return pos, cell, cutoff


def _request(ext, pos_t, cell, cutoff, keep):
    origin = np.zeros(3)
    inv = np.ascontiguousarray(np.linalg.inv(cell.T))
    pbc = np.ones(3, dtype=np.uint8)
    rc, pa, pt, nc = ext.resolve_cutoff(cutoff, pos_t.shape[0])
    keep.extend([origin, inv, pbc, cell, pa])
    return ext.make_request(31, origin, cell, inv, pbc, pos_t.shape[0],
                            ctypes.c_void_p(pos_t.data_ptr()), True, rc, pa, pt, nc,
                            None, 0)


def _outputs(torch, n):
    return {"i": torch.empty(n, dtype=torch.int32, device="cuda"),
            "j": torch.empty(n, dtype=torch.int32, device="cuda"),
            "D": torch.empty((n, 3), dtype=torch.float64, device="cuda"),
            "d": torch.empty(n, dtype=torch.float64, device="cuda"),
            "S": torch.empty((n, 3), dtype=torch.int32, device="cuda")}


def _existing(ext, torch, pos_t, cell, cutoff):
    keep = []
    req = _request(ext, pos_t, cell, cutoff, keep)
    plan = ext.plan_for(0)
    n = ctypes.c_int64()
    stream = torch.cuda.current_stream()
    ext.check(ext.lib.nbl_count(plan, ctypes.byref(req), ctypes.c_void_p(stream.cuda_stream),
                                ctypes.byref(n)))
    outs = _outputs(torch, int(n.value))
    o = ext._outputs_struct(outs, lambda t: t.data_ptr())
    ext.check(ext.lib.nbl_fill(plan, ctypes.byref(o), ctypes.c_void_p(stream.cuda_stream)))
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in outs.items()}


def _noalloc(ext, fn, torch, pos_t, cell, cutoff, capacity):
    keep = []
    req = _request(ext, pos_t, cell, cutoff, keep)
    outs = _outputs(torch, capacity)
    o = ext._outputs_struct(outs, lambda t: t.data_ptr())
    n = ctypes.c_int64()
    stream = torch.cuda.current_stream()
    st = fn(ctypes.byref(req), ctypes.byref(o), capacity, ctypes.byref(n),
            ctypes.c_void_p(stream.cuda_stream))
    torch.cuda.synchronize()
    got = {k: v[: int(n.value)].cpu().numpy() for k, v in outs.items()}
    return st, int(n.value), got


def test_noalloc_matches_existing_entry_point_twice():
    import torch
    ext, fn = _lib()
    torch.cuda.set_device(0)
    for n, seed, per_atom in [(20000, 1, False), (3000, 2, True)]:
        pos, cell, cutoff = _system(n, seed, per_atom)
        pos_t = torch.from_numpy(pos).cuda()
        want = _existing(ext, torch, pos_t, cell, cutoff)
        npairs = len(want["i"])
        st, got_n, got = _noalloc(ext, fn, torch, pos_t, cell, cutoff, npairs + 64)
        assert st == ext.NBL_SUCCESS, ext.lib.nbl_last_error()
        assert got_n == npairs
        for k in "ijDdS":
            assert got[k].shape == want[k].shape
            assert np.array_equal(got[k], want[k]), k


def test_noalloc_refuses_requests_beyond_its_limits():
    import torch
    ext, fn = _lib()
    pos, cell, cutoff = _system(40000, 3)
    pos_t = torch.from_numpy(pos).cuda()
    st, _, _ = _noalloc(ext, fn, torch, pos_t, cell, cutoff, 16)
    assert st == ext.NBL_ERROR_INVALID_ARGUMENT
    assert b"limit" in ext.lib.nbl_last_error()
    pos, cell, cutoff = _system(2000, 4)
    pos_t = torch.from_numpy(pos).cuda()
    st, n, _ = _noalloc(ext, fn, torch, pos_t, cell, cutoff, 16)
    assert st == ext.NBL_ERROR_CAPACITY and n > 16
