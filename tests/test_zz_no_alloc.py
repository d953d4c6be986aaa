"""nbl_neighbour_list_noalloc: the entry point for callers that cannot allocate
device memory at call time (for example an MD engine whose time-step loop
forbids allocation, or a host whose pool allocator has already reserved the
device memory).  It takes all scratch from a static array inside the library;
the caller provides inputs and output buffers.

Checks, through the C-ABI, that calls in a row return exactly what the
existing entry point (nbl_count + nbl_fill) returns and what the CPU oracle
returns -- each later call on a different system, so stale contents of the
shared scratch would show -- over both precisions, device and host
positions, scalar, per-atom and per-type cutoffs, and a sparse system whose
grid is too large for the static scratch and falls back to the hashed table;
and that requests beyond the stated limits are refused with a clear error.
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


def _system(n, seed, kind="scalar"):
    rng = np.random.default_rng(seed)
    L = (n / 0.085) ** (1.0 / 3.0)
    cell = np.array([[L, 0.0, 0.0], [0.15 * L, L, 0.0], [0.05 * L, 0.1 * L, L]])
    pos = rng.uniform(0, 1, size=(n, 3)) @ cell
    types = None
    pbc = (True, True, True)
    if kind == "per_atom":
        cutoff = rng.uniform(1.0, 2.2, size=n)
    elif kind == "per_type":
        cutoff = np.array([[2.5, 3.0], [3.0, 3.6]])
        types = rng.integers(0, 2, size=n).astype(np.int32)
    elif kind == "sparse":
        # a thin slab in a large open box: 10^6 cells for a few thousand atoms
        cell = np.diag([300.0, 300.0, 300.0])
        pos = np.column_stack([rng.uniform(0, 300, size=(n, 2)),
                               rng.uniform(140, 160, size=n)])
        pbc = (True, True, False)
        cutoff = 3.0
    else:
        cutoff = 4.0
    return dict(positions=np.ascontiguousarray(pos), cell=cell, cutoff=cutoff,
                types=types, pbc=pbc)


def _request(ext, w, pos_ptr, on_device, precision, keep):
    ext.set_options(precision=precision, grid="auto")
    origin = np.zeros(3)
    cell = np.ascontiguousarray(w["cell"], dtype=float)
    inv = np.ascontiguousarray(np.linalg.inv(cell.T))
    pbc = np.ascontiguousarray(np.asarray(w["pbc"], dtype=np.uint8))
    nat = w["positions"].shape[0]
    rc, pa, pt, nc = ext.resolve_cutoff(w["cutoff"], nat)
    types = w["types"]
    keep.extend([origin, inv, pbc, cell, pa, pt, types])
    return ext.make_request(31, origin, cell, inv, pbc, nat, pos_ptr, on_device, rc, pa,
                            pt, nc, types, 0)


def _outputs(torch, n):
    return {"i": torch.empty(n, dtype=torch.int32, device="cuda"),
            "j": torch.empty(n, dtype=torch.int32, device="cuda"),
            "D": torch.empty((n, 3), dtype=torch.float64, device="cuda"),
            "d": torch.empty(n, dtype=torch.float64, device="cuda"),
            "S": torch.empty((n, 3), dtype=torch.int32, device="cuda")}


def _existing(ext, torch, w, precision):
    keep = []
    pos_t = torch.from_numpy(w["positions"]).cuda()
    req = _request(ext, w, ctypes.c_void_p(pos_t.data_ptr()), True, precision, keep)
    plan = ext.plan_for(0)
    n = ctypes.c_int64()
    sp = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    ext.check(ext.lib.nbl_count(plan, ctypes.byref(req), sp, ctypes.byref(n)))
    outs = _outputs(torch, int(n.value))
    o = ext._outputs_struct(outs, lambda t: t.data_ptr())
    ext.check(ext.lib.nbl_fill(plan, ctypes.byref(o), sp))
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in outs.items()}


def _noalloc(ext, fn, torch, w, capacity, precision="fp32", host=False):
    keep = []
    if host:
        pos_ptr = ctypes.c_void_p(w["positions"].ctypes.data)
    else:
        pos_t = torch.from_numpy(w["positions"]).cuda()
        keep.append(pos_t)
        pos_ptr = ctypes.c_void_p(pos_t.data_ptr())
    req = _request(ext, w, pos_ptr, not host, precision, keep)
    outs = _outputs(torch, capacity)
    o = ext._outputs_struct(outs, lambda t: t.data_ptr())
    n = ctypes.c_int64()
    st = fn(ctypes.byref(req), ctypes.byref(o), capacity, ctypes.byref(n),
            ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    # no synchronisation here: the entry point returns with its work finished
    got = {k: v[: int(n.value)].cpu().numpy() for k, v in outs.items()}
    return st, int(n.value), got


def _same(a, b):
    if a.shape != b.shape or a.dtype != b.dtype:
        return False
    if a.dtype.kind == "f":
        return np.array_equal(a.view(np.int64), b.view(np.int64))
    return np.array_equal(a, b)


CALLS = [
    # (atoms, seed, cutoff kind, precision, host positions)
    (20000, 1, "scalar", "fp32", False),
    (3000, 2, "per_atom", "fp32", False),
    (12000, 5, "per_type", "fp64", True),
    (6000, 6, "sparse", "fp32", False),
    (2500, 7, "scalar", "fp64", True),
]


def test_noalloc_matches_existing_entry_point_and_oracle_calls_in_a_row(oracle):
    import torch
    ext, fn = _lib()
    torch.cuda.set_device(0)
    prev = ext.set_options()
    try:
        for n, seed, kind, precision, host in CALLS:
            w = _system(n, seed, kind)
            want = _existing(ext, torch, w, precision)
            ref = oracle.oracle_neighbour_list("ijDdS", w["cell"], w["positions"],
                                               w["cutoff"], w["pbc"], types=w["types"])
            npairs = len(want["i"])
            st, got_n, got = _noalloc(ext, fn, torch, w, npairs + 64, precision, host)
            assert st == ext.NBL_SUCCESS, ext.lib.nbl_last_error()
            assert got_n == npairs
            for k, r in zip("ijDdS", ref):
                assert _same(got[k], want[k]), (kind, k)
                assert _same(got[k], r), (kind, k)
    finally:
        ext.set_options(precision=prev["precision"], grid=prev["grid"])


def test_noalloc_refuses_requests_beyond_its_limits():
    import torch
    ext, fn = _lib()
    w = _system(40000, 3)
    st, _, _ = _noalloc(ext, fn, torch, w, 16)
    assert st == ext.NBL_ERROR_INVALID_ARGUMENT
    assert b"limit" in ext.lib.nbl_last_error()
    w = _system(2000, 4)
    st, n, _ = _noalloc(ext, fn, torch, w, 16)
    assert st == ext.NBL_ERROR_CAPACITY and n > 16
