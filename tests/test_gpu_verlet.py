"""The reused (Verlet) list: while no atom moved more than skin / 2 since the
build, the refreshed list holds exactly the pair set neighbour_list returns at
the cutoff, with D and d equal to 1e-12; a larger move rebuilds."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _canon(i, j, S, D, d):
    key = np.lexsort((S[:, 2], S[:, 1], S[:, 0], j, i))
    return i[key], j[key], S[key], D[key], d[key]


def _check(vl, pos_t, w, oracle):
    import torch
    i, j, d, D, S = [t.cpu().numpy() for t in vl.update(pos_t)]
    assert np.all(np.diff(i) >= 0)
    pos = pos_t.cpu().numpy()
    wi, wj, wd, wD, wS = oracle.oracle_neighbour_list("ijdDS", w["cell"], pos, vl.cutoff,
                                                      w["pbc"])
    a = _canon(i, j, S, D, d)
    b = _canon(wi, wj, wS, wD, wd)
    for x, y in zip(a[:3], b[:3]):
        assert np.array_equal(x, y)
    assert np.allclose(a[3], b[3], rtol=0, atol=1e-12)
    assert np.allclose(a[4], b[4], rtol=0, atol=1e-12)


@pytest.mark.parametrize("pbc", [(True, True, True), (True, False, True)])
def test_verlet_refresh_matches_rebuilt_list(oracle, pbc):
    import torch
    from matscipy_neighbours import _workloads as W
    from matscipy_neighbours.verlet import VerletList
    w = dict(W.fcc_bulk(reps=6))
    w["pbc"] = np.array(pbc)
    rng = np.random.default_rng(3)
    pos = torch.from_numpy(np.ascontiguousarray(w["positions"])).cuda()
    vl = VerletList(cutoff=4.0, skin=0.8, cell=w["cell"], pbc=w["pbc"])
    _check(vl, pos, w, oracle)
    assert vl.builds == 1
    for _ in range(4):  # random walk, each step well inside skin / 2 in total
        pos = pos + torch.from_numpy(rng.normal(0, 0.02, size=pos.shape)).cuda()
        _check(vl, pos, w, oracle)
    assert vl.builds == 1 and vl.refreshes == 4
    pos = pos + torch.from_numpy(rng.normal(0, 0.5, size=pos.shape)).cuda()
    _check(vl, pos, w, oracle)
    assert vl.builds == 2


def test_verlet_single_quantity_and_errors():
    import torch
    from matscipy_neighbours.verlet import VerletList
    rng = np.random.default_rng(1)
    pos = torch.from_numpy(rng.uniform(0, 8, size=(300, 3))).cuda()
    vl = VerletList(cutoff=2.0, skin=0.4, cell=8 * np.eye(3), quantities="d")
    d = vl.update(pos)
    assert d.dim() == 1 and bool((d < 2.0).all())
    with pytest.raises(ValueError):
        VerletList(cutoff=2.0, skin=-1.0, cell=np.eye(3))


def test_verlet_refresh_call_paths():
    """nbl_verlet_refresh counts only (out NULL), refuses a capacity below the
    kept count, and gives the same rows whether it writes before (capacity >=
    stored pairs) or after (capacity = kept) reading the count."""
    import ctypes
    import torch
    from matscipy_neighbours import _matscipy_neighbours as _ext
    from matscipy_neighbours import _workloads as W
    from matscipy_neighbours.neighbours import neighbour_list
    from matscipy_neighbours.verlet import _lib
    lib = _lib()
    w = W.fcc_bulk(reps=5)
    pos = torch.from_numpy(np.ascontiguousarray(w["positions"])).cuda()
    i, j, S = neighbour_list("ijS", positions=pos, cell=w["cell"], pbc=w["pbc"], cutoff=4.5,
                             array_namespace=torch)
    pos2 = pos + torch.from_numpy(np.random.default_rng(2).normal(0, 0.05, pos.shape)).cuda()
    cell = np.ascontiguousarray(w["cell"], dtype=np.float64)
    pbc = np.ones(3, dtype=np.uint8)
    npairs = int(i.shape[0])
    stream = torch.cuda.current_stream()
    sp = ctypes.c_void_p(stream.cuda_stream)
    P = ctypes.c_void_p

    def call(o, cap):
        n = ctypes.c_int64()
        st = lib.nbl_verlet_refresh(npairs, P(i.data_ptr()), P(j.data_ptr()), P(S.data_ptr()),
                                    P(pos2.data_ptr()), P(cell.ctypes.data), P(pbc.ctypes.data),
                                    4.0, o, cap, ctypes.byref(n), sp)
        return st, int(n.value)

    st, kept = call(None, 0)
    assert st == 0 and 0 < kept < npairs

    def outputs(m):
        t = {"i": torch.empty(m, dtype=torch.int32, device="cuda"),
             "j": torch.empty(m, dtype=torch.int32, device="cuda"),
             "D": torch.empty((m, 3), dtype=torch.float64, device="cuda"),
             "d": torch.empty(m, dtype=torch.float64, device="cuda"),
             "S": torch.empty((m, 3), dtype=torch.int32, device="cuda")}
        o = _ext.Outputs()
        o.first, o.second = t["i"].data_ptr(), t["j"].data_ptr()
        o.distvec, o.absdist, o.shift = t["D"].data_ptr(), t["d"].data_ptr(), t["S"].data_ptr()
        return t, o

    t_small, o_small = outputs(kept - 1)
    st, n = call(ctypes.byref(o_small), kept - 1)
    assert st == _ext.NBL_ERROR_CAPACITY and n == kept
    t_exact, o_exact = outputs(kept)
    st, n = call(ctypes.byref(o_exact), kept)
    assert st == 0 and n == kept
    t_all, o_all = outputs(npairs)
    st, n = call(ctypes.byref(o_all), npairs)
    assert st == 0 and n == kept
    torch.cuda.synchronize()
    for k in "ijDdS":
        assert torch.equal(t_exact[k], t_all[k][:kept])
    # the kept rows are the stored rows with d < cutoff, in the stored order
    D = pos2[j.long()] - pos2[i.long()] + S.double() @ torch.from_numpy(cell).cuda()
    keep = (D * D).sum(1) < 16.0
    assert torch.equal(t_all["i"][:kept], i[keep]) and torch.equal(t_all["j"][:kept], j[keep])
    assert torch.equal(t_all["S"][:kept], S[keep])
