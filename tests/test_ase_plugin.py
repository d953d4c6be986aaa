"""The ASE plugin entry point: the adapter forwards an Atoms-like object to
neighbour_list, refuses self_interaction=True, and registers nothing when the
installed ASE has no plugin API (ASE is absent here)."""
import numpy as np
import pytest


class _Atoms:
    """The attributes of ase.Atoms that neighbour_list reads."""

    def __init__(self, positions, cell, pbc, numbers):
        self.positions = positions
        self.cell = cell
        self.pbc = pbc
        self.numbers = numbers


def _atoms(seed=0, n=200, box=9.0):
    rng = np.random.default_rng(seed)
    return _Atoms(rng.uniform(0, box, size=(n, 3)), np.diag([box, box, box]),
                  np.array([True, True, False]), np.ones(n, dtype=np.int64))


def test_plugin_registration_and_self_interaction():
    from matscipy_neighbours import _ase_plugin as plugin
    try:
        import ase  # noqa: F401
        has_ase = True
    except ImportError:
        has_ase = False
    if not has_ase:
        assert plugin.__ase_plugins__ == set()
    with pytest.raises(NotImplementedError):
        plugin.neighbor_list("ij", _atoms(), 2.0, self_interaction=True)


def test_plugin_without_gpu_fails_loudly():
    from matscipy_neighbours import _ase_plugin as plugin
    from matscipy_neighbours import _matscipy_neighbours as ext
    if ext._has_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(RuntimeError):
        plugin.neighbor_list("ij", _atoms(), 2.0)


@pytest.mark.gpu
def test_plugin_matches_neighbour_list():
    from matscipy_neighbours import _ase_plugin as plugin
    from matscipy_neighbours import neighbour_list
    a = _atoms()
    got = plugin.neighbor_list("ijdDS", a, 2.5)
    want = neighbour_list("ijdDS", positions=a.positions, cell=a.cell, pbc=a.pbc,
                          cutoff=2.5)
    assert len(got[0]) > 0
    for g, w in zip(got, want):
        assert np.array_equal(g, w)
