"""The public API on the GPU: device (torch) positions in and out, DLPack
capsules, device override, coordination, the dense matrix, error classes."""
import numpy as np
import pytest

from conftest import assert_same_lists

pytestmark = pytest.mark.gpu


def _config(N=2000, L=12.0, seed=1):
    rng = np.random.default_rng(seed)
    return (np.ascontiguousarray(rng.uniform(0.0, L, size=(N, 3))),
            np.diag([L, L, L]).astype(float), np.ones(3, dtype=bool))


def test_host_path_matches_oracle(oracle):
    import matscipy_neighbours as m
    pos, cell, pbc = _config()
    got = m.neighbour_list("ijdDS", positions=pos, cell=cell, pbc=pbc, cutoff=1.0)
    want = oracle.oracle_neighbour_list("ijdDS", cell, pos, 1.0, pbc)
    assert all(isinstance(a, np.ndarray) for a in got)
    assert_same_lists(got, want, "ijdDS")


def test_torch_in_torch_out(oracle):
    import torch
    import matscipy_neighbours as m
    pos, cell, pbc = _config(N=3000, seed=5)
    t = torch.from_numpy(pos).cuda()
    got = m.neighbour_list("ijdDS", positions=t, cell=cell, pbc=pbc, cutoff=1.0,
                           array_namespace=torch)
    assert all(isinstance(a, torch.Tensor) and a.is_cuda for a in got)
    want = oracle.oracle_neighbour_list("ijdDS", cell, pos, 1.0, pbc)
    assert_same_lists([a.cpu().numpy() for a in got], want, "ijdDS")


def test_device_dlpack_capsules():
    import torch
    import matscipy_neighbours as m
    from matscipy_neighbours import DLPackTensor
    pos, cell, pbc = _config(N=1500, seed=8)
    caps = m.neighbour_list("ij", positions=torch.from_numpy(pos).cuda(), cell=cell,
                            pbc=pbc, cutoff=1.0, array_namespace="dlpack")
    assert all(isinstance(c, DLPackTensor) for c in caps)
    assert caps[0].__dlpack_device__() == (2, 0)
    i, j = (torch.from_dlpack(c) for c in caps)
    assert i.is_cuda and i.dtype == torch.int32


def test_host_dlpack_capsules_free_without_consumer():
    import matscipy_neighbours as m
    pos, cell, pbc = _config(N=500, seed=4)
    caps = m.neighbour_list("i", positions=pos, cell=cell, pbc=pbc, cutoff=1.0,
                            array_namespace="dlpack")
    del caps


def test_host_array_namespace_numpy_matches_fast_path():
    import matscipy_neighbours as m
    pos, cell, pbc = _config(seed=2)
    a = m.neighbour_list("ijS", positions=pos, cell=cell, pbc=pbc, cutoff=1.0)
    b = m.neighbour_list("ijS", positions=pos, cell=cell, pbc=pbc, cutoff=1.0,
                         array_namespace=np)
    assert_same_lists(b, a, "ijS")


def test_device_override_host_in_gpu_out(oracle):
    import torch
    import matscipy_neighbours as m
    pos, cell, pbc = _config(N=2500, seed=7)
    i, j = m.neighbour_list("ij", positions=pos, cell=cell, pbc=pbc, cutoff=1.0,
                            device="cuda", array_namespace=torch)
    assert i.is_cuda
    want = oracle.oracle_neighbour_list("ij", cell, pos, 1.0, pbc)
    assert_same_lists((i.cpu().numpy(), j.cpu().numpy()), want, "ij")


def test_device_wrong_dtype_raises_type_error():
    import torch
    import matscipy_neighbours as m
    pos = torch.rand(400, 3, dtype=torch.float32, device="cuda")
    with pytest.raises(TypeError):
        m.neighbour_list("ij", positions=pos, cell=np.diag([12.0] * 3),
                         cell_origin=np.zeros(3), pbc=False, cutoff=2.5,
                         array_namespace=torch)


def test_device_positions_need_a_cell():
    import torch
    import matscipy_neighbours as m
    with pytest.raises(ValueError):
        m.neighbour_list("ij", positions=torch.zeros(3, 3, dtype=torch.float64,
                                                     device="cuda"), cutoff=1.0)


def test_coordination_device_and_host(oracle):
    import torch
    import matscipy_neighbours as m
    pos, cell, pbc = _config(N=3000, seed=10)
    want = oracle.oracle_counts(cell, pos, 1.3, pbc)
    c_host = m.coordination(positions=pos, cell=cell, pbc=pbc, cutoff=1.3)
    assert isinstance(c_host, np.ndarray) and np.array_equal(c_host, want)
    c_dev = m.coordination(positions=torch.from_numpy(pos).cuda(), cell=cell, pbc=pbc,
                           cutoff=1.3, array_namespace=torch)
    assert c_dev.is_cuda and np.array_equal(c_dev.cpu().numpy(), want)


def test_matrix_matches_pairs(oracle):
    import torch
    import matscipy_neighbours as m
    pos, cell, pbc = _config(seed=11)
    n = len(pos)
    i, j, D = oracle.oracle_neighbour_list("ijD", cell, pos, 1.0, pbc)
    idx, dist, count = m.neighbour_matrix(positions=pos, cell=cell, pbc=pbc, cutoff=1.0,
                                          max_neighbours=64)
    assert idx.shape == (n, 64) and dist.shape == (n, 64, 3)
    assert np.array_equal(count, np.bincount(i, minlength=n))
    off = np.concatenate([[0], np.cumsum(count)])
    for a in range(0, n, 37):
        k = count[a]
        assert np.array_equal(idx[a, :k], j[off[a]:off[a + 1]])
        assert np.array_equal(dist[a, :k], D[off[a]:off[a + 1]])
        assert not idx[a, k:].any() and not dist[a, k:].any()
    idx_t, dist_t, count_t = m.neighbour_matrix(positions=torch.from_numpy(pos).cuda(),
                                                cell=cell, pbc=pbc, cutoff=1.0,
                                                max_neighbours=64, array_namespace=torch)
    assert np.array_equal(idx_t.cpu().numpy(), idx)
    assert np.array_equal(dist_t.cpu().numpy(), dist)


def test_matrix_overflow_raises():
    import matscipy_neighbours as m
    pos, cell, pbc = _config(seed=12)
    with pytest.raises(ValueError):
        m.neighbour_matrix(positions=pos, cell=cell, pbc=pbc, cutoff=1.5,
                           max_neighbours=2)


def test_repeated_calls_reuse_workspace(oracle):
    import matscipy_neighbours as m
    for seed, N in [(1, 3000), (2, 100), (3, 5000), (4, 10)]:
        pos, cell, pbc = _config(N=N, seed=seed)
        got = m.neighbour_list("ijdDS", positions=pos, cell=cell, pbc=pbc, cutoff=1.2)
        want = oracle.oracle_neighbour_list("ijdDS", cell, pos, 1.2, pbc)
        assert_same_lists(got, want, "ijdDS")
