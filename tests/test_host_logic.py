"""Host-side logic of the binding and the public API that runs before any
device work: argument coercion, cutoff resolution and the reference's error
classes (bind_py_neighbours.cc:97-195, neighbours.py:145-288)."""
import numpy as np
import pytest

from matscipy_neighbours import _matscipy_neighbours as ext
from matscipy_neighbours import neighbours as nb


def test_quantity_flags():
    assert ext.quantity_flags("ijdDS") == 31
    assert ext.quantity_flags("") == 0
    assert ext.quantity_flags("D") == 4
    with pytest.raises(ValueError):
        ext.quantity_flags("x")
    with pytest.raises(TypeError):
        ext.quantity_flags("ié")


def test_resolve_cutoff_forms():
    assert ext.resolve_cutoff(2.5, 10) == (2.5, None, None, 0)
    rc, pa, pt, nc = ext.resolve_cutoff(np.array([0.4, 0.4, 1.2]), 3)
    assert rc == 2.4 and pa is not None and pt is None and nc == 0
    rc, pa, pt, nc = ext.resolve_cutoff(np.array([[2.0, 3.0], [3.0, 4.0]]), 5)
    assert rc == 4.0 and nc == 2 and np.array_equal(pt, [[4.0, 9.0], [9.0, 16.0]])
    with pytest.raises(TypeError):
        ext.resolve_cutoff(np.ones(9), 10)
    with pytest.raises(TypeError):
        ext.resolve_cutoff(np.ones((2, 3)), 10)
    # A Python int is not a float: the reference coerces it to an array of
    # depth 0 and raises.
    with pytest.raises(ValueError):
        ext.resolve_cutoff(3, 10)


def test_geometry_coercion_errors():
    with pytest.raises(ValueError):
        ext.coerce_geometry(np.zeros(3), np.eye(2), np.eye(3), [True] * 3)
    o, c, inv, p = ext.coerce_geometry([0, 0, 0], np.eye(3), np.eye(3), [1, 0, 1])
    assert p.dtype == np.uint8 and list(p) == [1, 0, 1]


def test_type_length_mismatch_is_type_error():
    with pytest.raises(TypeError):
        ext.neighbour_list("ij", np.zeros(3), np.eye(3), np.eye(3),
                           np.array([True] * 3), np.zeros((4, 3)), 1.0,
                           np.zeros(3, dtype=np.int32))


def test_missing_cutoff_and_positions():
    with pytest.raises(ValueError):
        nb.neighbour_list("ij", positions=np.zeros((2, 3)))
    with pytest.raises(ValueError):
        nb.neighbour_list("ij", cutoff=1.0)
    with pytest.raises(ValueError):
        nb.neighbour_matrix(positions=np.zeros((2, 3)), cutoff=1.0)


def test_resolve_device():
    assert nb._resolve_device(None, True) == (True, -1)
    assert nb._resolve_device("cpu", False) == (False, -1)
    assert nb._resolve_device("cuda", False) == (True, -1)
    assert nb._resolve_device(1, False) == (True, 1)
    assert nb._resolve_device(("cuda", 2), False) == (True, 2)
    with pytest.raises(ValueError):
        nb._resolve_device("tpu", False)


def test_dict_cutoff_matrix():
    m, nums = nb._resolve_cutoff({(1, 2): 3.0, (2, 2): 1.5}, np.array([1, 2, 2]))
    assert m.shape == (3, 3)
    assert m[1, 2] == m[2, 1] == 3.0 and m[2, 2] == 1.5 and m[1, 1] == 0.0


def test_host_metadata_defaults():
    co, ce, inv, pb, nums = nb._host_metadata(None, None, None, None, 2,
                                              positions=np.array([[0.0, 0, 0],
                                                                  [1.0, 2, 3]]))
    assert np.array_equal(ce, np.diag([1.0, 2.0, 3.0]))
    assert not pb.any() and np.array_equal(nums, [1, 1])
    assert np.allclose(inv, np.linalg.inv(ce.T))


# first_neighbours / get_jump_indicies / triplet_list known answers
# (tests/test_extension.py:277-336 of the reference).
def test_first_neighbours_known_answers():
    f = ext.first_neighbours
    assert list(f(5, [1, 1, 1, 1, 3, 3, 3])) == [-1, 0, 4, 4, 7, 7]
    assert list(f(6, [0, 1, 2, 3, 4, 5])) == [0, 1, 2, 3, 4, 5, 6]
    assert list(f(8, [0, 1, 2, 3, 5, 6])) == [0, 1, 2, 3, 4, 4, 5, 6, 6]
    assert list(f(8, [0, 1, 2, 3, 3, 5, 6])) == [0, 1, 2, 3, 5, 5, 6, 7, 7]
    assert list(f(5, [])) == [0] * 6


def test_jump_indices_known_answers():
    assert list(ext.get_jump_indicies(
        [0, 0, 0, 1, 1, 1, 1, 1, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4])) == [0, 3, 8, 11, 15, 19]
    assert list(ext.get_jump_indicies([0])) == [0, 1]


def test_triplets_known_answers():
    first_i = np.array([0, 2, 6, 10], dtype=np.int32)
    ij, ik = ext.triplet_list(first_i)
    assert list(ij) == [0, 1, 2, 2, 2, 3, 3, 3, 4, 4, 4, 5, 5, 5, 6, 6, 6, 7, 7, 7, 8, 8, 8,
                        9, 9, 9]
    assert list(ik) == [1, 0, 3, 4, 5, 2, 4, 5, 2, 3, 5, 2, 3, 4, 7, 8, 9, 6, 8, 9, 6, 7, 9,
                        6, 7, 8]
    ij, ik = ext.triplet_list(first_i, np.array([2.2] * 4 + [3.0] * 2 + [2.0] * 4), 2.6)
    assert list(ij) == [0, 1, 2, 3, 6, 6, 6, 7, 7, 7, 8, 8, 8, 9, 9, 9]
    assert list(ik) == [1, 0, 3, 2, 7, 8, 9, 6, 8, 9, 6, 7, 9, 6, 7, 8]
    with pytest.raises(TypeError):
        ext.triplet_list(first_i, np.ones(10))


def test_mic():
    cell = 10.0 * np.eye(3)
    dr = np.array([[6.0, -7.0, 1.0]])
    assert np.allclose(nb.mic(dr, cell), [[-4.0, 3.0, 1.0]])
    assert np.allclose(nb.mic(dr, cell, pbc=[False, True, True]), [[6.0, 3.0, 1.0]])
