"""The fused Lennard-Jones consumer (nbl_lj_forces) against the same potential
evaluated in float64 numpy over the oracle's own pair list (i, D, d): forces
and energy agree to 1e-12 relative (only the summation order differs)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lj_reference(oracle, w, eps, sig):
    i, D, d = oracle.oracle_neighbour_list("iDd", w["cell"], w["positions"], w["cutoff"],
                                           w["pbc"])
    s6 = (sig * sig / (d * d)) ** 3
    coef = -24.0 * eps * s6 * (2.0 * s6 - 1.0) / (d * d)
    f = np.zeros((len(w["positions"]), 3))
    np.add.at(f, i, coef[:, None] * D)
    e = 0.5 * np.sum(4.0 * eps * (s6 * s6 - s6))
    return e, f


def _systems():
    from matscipy_neighbours import _workloads as W
    rng = np.random.default_rng(4)
    a = 1.6  # reduced-unit FCC spacing of the reference's LJ droplet example
    g = np.stack(np.meshgrid(*[np.arange(8)] * 3, indexing="ij"), -1).reshape(-1, 3)
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    fcc = ((g[:, None, :] + basis[None]) * a).reshape(-1, 3) + rng.normal(0, 0.05, (2048, 3))
    return [("fcc_droplet_open", dict(positions=fcc, cell=np.diag([13.0, 13.0, 13.0]),
                                      pbc=(False, False, False), cutoff=2.5), 1.0, 1.0),
            ("fcc_bulk_6_periodic", W.fcc_bulk(reps=6), 0.8, 2.3),
            ("plain_small", W.plain_small(), 1.3, 0.9)]


@pytest.mark.parametrize("k", range(3))
@pytest.mark.parametrize("device_input", [False, True])
def test_lennard_jones_matches_pair_list(oracle, k, device_input):
    import torch
    import matscipy_neighbours as m
    name, w, eps, sig = _systems()[k]
    want_e, want_f = _lj_reference(oracle, w, eps, sig)
    pos = torch.from_numpy(np.ascontiguousarray(w["positions"])).cuda() if device_input \
        else w["positions"]
    e, f = m.lennard_jones(pos, float(w["cutoff"]), cell=w["cell"], pbc=w["pbc"],
                           epsilon=eps, sigma=sig)
    if device_input:
        torch.cuda.synchronize()
        e, f = float(e.item()), f.cpu().numpy()
    scale = np.abs(want_f).max()
    assert np.allclose(f, want_f, rtol=1e-12, atol=1e-12 * scale), name
    assert abs(e - want_e) <= 1e-12 * max(1.0, abs(want_e)), (name, e, want_e)


def test_lennard_jones_twice_and_empty():
    import matscipy_neighbours as m
    rng = np.random.default_rng(0)
    pos = rng.uniform(0, 5, size=(200, 3))
    e1, f1 = m.lennard_jones(pos, 1.5, cell=5 * np.eye(3))
    e2, f2 = m.lennard_jones(pos, 1.5, cell=5 * np.eye(3))
    assert e1 == e2 and np.array_equal(f1, f2)
    e, f = m.lennard_jones(np.zeros((0, 3)), 1.5, cell=5 * np.eye(3))
    assert e == 0.0 and f.shape == (0, 3)
