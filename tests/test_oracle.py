"""The CPU oracle, pinned to the reference: golden digests produced by the
reference's own core, the reference tests' known answers, an independent
brute force, and (where the reference sources were compiled) a direct
comparison with the reference core."""
import numpy as np
import pytest

from _cases import digest, golden_cases

CASES = golden_cases()


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_oracle_matches_reference_golden(oracle, case):
    out = oracle.oracle_neighbour_list(case["quantities"], case["cell"],
                                       case["positions"], case["cutoff"], case["pbc"],
                                       types=case["types"])
    assert len(out[0]) == case["npairs"]
    for q, a in zip(case["quantities"], out):
        assert digest(a) == case["digest"][q], q
        if q in case["full"]:
            assert np.array_equal(a, case["full"][q])


# Known answers of the reference's tests (tests/test_extension.py:102-119,
# 211-231; tests/test_core.cc:32-120).
def test_unit_cube_counts(oracle):
    i, j, D, S = oracle.oracle_neighbour_list("ijDS", np.eye(3), [[0.5, 0.5, 0.5]], 1.1)
    assert np.bincount(i)[0] == 6
    assert (D == S).all()
    i = oracle.oracle_neighbour_list("i", np.eye(3), [[0.5, 0.5, 0.5]], 1.5)
    assert np.bincount(i)[0] == 18


def test_mixed_pbc_counts(oracle):
    p = [[0.5, 0.5, 0.5]]
    assert len(oracle.oracle_neighbour_list("i", np.eye(3), p, 1.1, False)) == 0
    assert np.bincount(oracle.oracle_neighbour_list(
        "i", np.eye(3), p, 1.1, [True, False, False]))[0] == 2
    assert np.bincount(oracle.oracle_neighbour_list(
        "i", np.eye(3), p, 1.1, [True, False, True]))[0] == 4


def test_per_atom_and_per_type(oracle):
    i, j = oracle.oracle_neighbour_list(
        "ij", 10.0 * np.eye(3), [[0.0, 0, 0], [1.0, 0, 0], [2.5, 0, 0]],
        np.array([0.4, 0.4, 1.2]), False)
    assert sorted(zip(i.tolist(), j.tolist())) == [(1, 2), (2, 1)]
    i, j = oracle.oracle_neighbour_list(
        "ij", 10.0 * np.eye(3), [[0.0, 0, 0], [1.0, 0, 0], [2.0, 0, 0]],
        np.array([[0.5, 1.5], [1.5, 0.5]]), False, types=np.array([0, 1, 0]))
    assert sorted(zip(i.tolist(), j.tolist())) == [(0, 1), (1, 0), (1, 2), (2, 1)]


def test_sc_lattice_shift_consistency(oracle):
    r = np.array([[0.5 + x, 0.5 + y, 0.5 + z] for x in range(2) for y in range(2)
                  for z in range(2)], dtype=float)
    cell = 2.0 * np.eye(3)
    i, j, D, d, S = oracle.oracle_neighbour_list("ijDdS", cell, r, 1.1, True)
    assert len(i) == 48
    assert np.allclose(D, r[j] - r[i] + S @ cell, atol=1e-12)
    assert np.allclose(d, np.linalg.norm(D, axis=1), atol=1e-12)
    assert (np.bincount(i) == 6).all() and (np.bincount(j) == 6).all()


@pytest.mark.parametrize("seed,pbc", [(1234, True), (1234, False),
                                      (1234, (True, False, True)), (7, True),
                                      (7, (True, True, False))])
def test_oracle_vs_brute_force(oracle, seed, pbc):
    rng = np.random.default_rng(seed)
    cell = np.array([[4.0, 0.0, 0.0], [1.3, 3.7, 0.0], [0.8, 0.6, 4.2]])
    pos = rng.uniform(-0.3, 1.3, size=(30, 3)) @ cell
    i, j = oracle.oracle_neighbour_list("ij", cell, pos, 1.6, pbc)
    assert sorted(zip(i.tolist(), j.tolist())) == oracle.brute_force_pairs(cell, pos, pbc, 1.6)


def test_zero_volume_is_an_error(oracle):
    with pytest.raises(oracle.OracleError):
        oracle.oracle_neighbour_list("i", np.array([[1.0, 0, 0], [2.0, 0, 0], [0, 0, 1.0]]),
                                     [[0.0, 0, 0]], 1.0, True,
                                     inv_cell=np.zeros((3, 3)))


def test_oracle_equals_reference_core_when_built(oracle):
    if not oracle.ref_available():
        pytest.skip("reference core not compiled here")
    from matscipy_neighbours import _workloads as W
    for w in (W.plain_small(), W.fcc_bulk(reps=10), W.diff_lattice(shape=(10, 10, 8)),
              W.sparse_slab(n=20000), W.dilute_gas(n=20000)):
        types = w.get("numbers")
        types = None if types is None else np.ascontiguousarray(types, dtype=np.int32)
        a = oracle.oracle_neighbour_list("ijdDS", w["cell"], w["positions"], w["cutoff"],
                                         w["pbc"], types=types)
        b = oracle.ref_neighbour_list("ijdDS", w["cell"], w["positions"], w["cutoff"],
                                      w["pbc"], types=types)
        assert len(a[0]) > 0
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


# --- CSR helpers: the oracle's restatement against the reference's own code
#     (first_neighbours.cc, triplet_list.cc compiled into oracle/_ref) and the
#     reference tests' known answers (tests/test_extension.py:277-336) ---------

def test_csr_oracle_known_answers(oracle):
    f = oracle.oracle_first_neighbours
    assert list(f(5, [1, 1, 1, 1, 3, 3, 3])) == [-1, 0, 4, 4, 7, 7]
    assert list(f(8, [0, 1, 2, 3, 3, 5, 6])) == [0, 1, 2, 3, 5, 5, 6, 7, 7]
    assert list(f(5, [])) == [0] * 6
    first_i = np.array([0, 2, 6, 10], dtype=np.int32)
    ij, ik = oracle.oracle_triplet_list(first_i, np.array([2.2] * 4 + [3.0] * 2 + [2.0] * 4),
                                        2.6)
    assert list(ij) == [0, 1, 2, 3, 6, 6, 6, 7, 7, 7, 8, 8, 8, 9, 9, 9]
    assert list(ik) == [1, 0, 3, 2, 7, 8, 9, 6, 8, 9, 6, 7, 9, 6, 7, 8]


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_csr_oracle_equals_reference_and_host_path(oracle, seed):
    from matscipy_neighbours import _matscipy_neighbours as ext
    rng = np.random.default_rng(seed)
    n = 300
    pos = rng.uniform(0, 9, size=(n, 3))
    i, d = oracle.oracle_neighbour_list("id", 9 * np.eye(3), pos, 2.2, (True, False, True))
    seed_o = oracle.oracle_first_neighbours(n, i)
    assert np.array_equal(seed_o, ext.first_neighbours(n, i))
    if oracle.ref_available():
        assert np.array_equal(seed_o, oracle.ref_first_neighbours(n, i))
    for cut in (None, 1.7):
        dd = None if cut is None else d
        want = oracle.oracle_triplet_list(seed_o, dd, cut)
        got = ext.triplet_list(seed_o) if cut is None else ext.triplet_list(seed_o, dd, cut)
        assert np.array_equal(want[0], got[0]) and np.array_equal(want[1], got[1])
        if oracle.ref_available():
            ref = oracle.ref_triplet_list(seed_o, dd, cut)
            assert np.array_equal(want[0], ref[0]) and np.array_equal(want[1], ref[1])
