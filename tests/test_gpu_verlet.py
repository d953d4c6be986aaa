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
