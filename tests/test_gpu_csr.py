"""CSR helpers on the device (nbl_first_neighbours, nbl_triplet_list) against
the oracle's restatement of the reference's first_neighbours.cc and
triplet_list.cc: the same arrays, element for element."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lists(oracle):
    from matscipy_neighbours import _workloads as W
    out = []
    for name, w in (("plain_small", W.plain_small()), ("fcc_bulk_6", W.fcc_bulk(reps=6)),
                    ("diff_lattice_8", W.diff_lattice(shape=(8, 8, 6)))):
        i, d = oracle.oracle_neighbour_list("id", w["cell"], w["positions"], w["cutoff"],
                                            w["pbc"])
        out.append((name, len(w["positions"]), i, d, 0.75 * float(np.max(w["cutoff"]))))
    # rows before the first atom with pairs, empty rows inside and at the end
    i = np.array([2, 2, 2, 5, 7, 7, 7, 7], dtype=np.int32)
    out.append(("gaps", 10, i, np.linspace(1.0, 3.0, len(i)), 2.0))
    out.append(("empty", 4, np.zeros(0, dtype=np.int32), np.zeros(0), 1.0))
    return out


@pytest.mark.parametrize("k", range(5))
def test_first_neighbours_and_triplets_match_oracle(oracle, k):
    import torch
    from matscipy_neighbours import _matscipy_neighbours as ext
    from matscipy_neighbours import neighbours
    name, n, i, d, cut = _lists(oracle)[k]
    want_seed = oracle.oracle_first_neighbours(n, i)
    it = torch.from_numpy(i).cuda()
    seed = ext.first_neighbours(n, it)
    assert seed.is_cuda
    assert np.array_equal(seed.cpu().numpy(), want_seed), name
    seed_h = want_seed
    for use_cut in (False, True):
        if use_cut:
            want = oracle.oracle_triplet_list(seed_h, d, cut)
            got = neighbours.triplet_list(seed, torch.from_numpy(d).cuda(), cut)
        else:
            want = oracle.oracle_triplet_list(seed_h)
            got = neighbours.triplet_list(seed)
        assert got[0].is_cuda and got[1].is_cuda
        assert np.array_equal(got[0].cpu().numpy(), want[0]), (name, use_cut)
        assert np.array_equal(got[1].cpu().numpy(), want[1]), (name, use_cut)


def test_triplet_capacity_and_errors():
    import ctypes

    import torch
    from matscipy_neighbours import _matscipy_neighbours as ext
    f = torch.tensor([0, 3, 5], dtype=torch.int32, device="cuda")
    n = ctypes.c_int64()
    ij = torch.empty(2, dtype=torch.int32, device="cuda")
    ik = torch.empty(2, dtype=torch.int32, device="cuda")
    st = ext.lib.nbl_triplet_list(3, ctypes.c_void_p(f.data_ptr()), None, 0.0,
                                  ctypes.c_void_p(ij.data_ptr()), ctypes.c_void_p(ik.data_ptr()),
                                  2, ctypes.byref(n), None)
    assert st == ext.NBL_ERROR_CAPACITY and n.value == 8
    with pytest.raises(TypeError):
        ext.triplet_list(f, torch.ones(5, dtype=torch.float64, device="cuda"))
