"""Randomised parity: seeded random systems -- triclinic cells of any size
against the cutoff (many periodic images down to sparse grids), mixed
periodicity, atoms outside the box, scalar / per-atom / per-type cutoffs --
each through a random engine configuration (precision, grid layout, atoms per
work item, runs of cells, the one-launch count phase, the pair-pass form) and compared with the
CPU oracle bit for bit, row order included."""
import ctypes

import numpy as np
import pytest

from conftest import assert_same_lists

pytestmark = pytest.mark.gpu

NCASES = 400


def _case(seed):
    rng = np.random.default_rng(1000 + seed)
    n = int(rng.choice([0, 1, 2, 7, 40, 120, 300, 700]))
    edges = rng.uniform(2.5, 30.0, size=3)
    cell = np.diag(edges)
    cell[1, 0] = rng.uniform(-0.4, 0.4) * edges[1]
    cell[2, 0] = rng.uniform(-0.4, 0.4) * edges[2]
    cell[2, 1] = rng.uniform(-0.4, 0.4) * edges[2]
    pbc = rng.integers(0, 2, size=3).astype(bool)
    frac = rng.uniform(-0.15, 1.15, size=(n, 3))
    frac[:, pbc] = rng.uniform(0.0, 1.0, size=(n, int(pbc.sum())))
    if n > 4 and rng.random() < 0.3:  # a few atoms far outside on periodic axes
        frac[: n // 5] += rng.integers(-3, 4, size=(n // 5, 3)) * pbc
    pos = np.ascontiguousarray(frac @ cell)
    kind = rng.choice(["scalar", "per_atom", "per_type"])
    types = None
    if kind == "scalar":
        cutoff = float(rng.uniform(0.5, 6.0))
    elif kind == "per_atom":
        cutoff = rng.uniform(0.0, 3.0, size=n)
    else:
        nt = int(rng.integers(1, 4))
        m = rng.uniform(0.5, 5.0, size=(nt, nt))
        cutoff = np.ascontiguousarray((m + m.T) / 2)
        types = rng.integers(0, nt, size=n).astype(np.int32)
    cfg = dict(precision=str(rng.choice(["fp32", "fp64"])),
               grid=str(rng.choice(["auto", "dense", "morton", "hashed"])),
               atoms_per_item=int(rng.choice([0, 5, 16])),
               cells_per_item=int(rng.choice([0, 1, 4, 8])),
               one_launch_atoms=int(rng.choice([0, -1, 2048])),
               thread_per_atom=int(rng.choice([0, -1, 1])))
    return dict(positions=pos, cell=cell, pbc=pbc, cutoff=cutoff, types=types), cfg


@pytest.mark.parametrize("seed", range(NCASES))
def test_random_system_and_configuration(oracle, seed):
    import torch

    import matscipy_neighbours as m
    from matscipy_neighbours import _matscipy_neighbours as ext
    w, cfg = _case(seed)
    plan = ext.plan_for(0)
    prev = ext.set_options()
    ext.set_options(precision=cfg["precision"], grid=cfg["grid"])
    lc = ext.LaunchConfig(atoms_per_item=cfg["atoms_per_item"],
                          cells_per_item=cfg["cells_per_item"],
                          one_launch_atoms=cfg["one_launch_atoms"],
                          thread_per_atom=cfg["thread_per_atom"])
    ext.check(ext.lib.nbl_plan_set_launch_config(plan, ctypes.byref(lc)))
    try:
        want = oracle.oracle_neighbour_list("ijdDS", w["cell"], w["positions"], w["cutoff"],
                                            w["pbc"], types=w["types"])
        kw = {} if w["types"] is None else {"numbers": w["types"]}
        # host arrays in and out, then device positions in and out
        got = m.neighbour_list("ijdDS", positions=w["positions"], cell=w["cell"],
                               pbc=w["pbc"], cutoff=w["cutoff"], **kw)
        assert_same_lists(got, want, "ijdDS")
        pos = torch.from_numpy(w["positions"].reshape(-1, 3)).cuda()
        got = m.neighbour_list("ijdDS", positions=pos, cell=w["cell"], pbc=w["pbc"],
                               cutoff=w["cutoff"], array_namespace=torch, **kw)
        torch.cuda.synchronize()
        assert_same_lists(tuple(t.cpu().numpy() for t in got), want, "ijdDS")
    finally:
        ext.check(ext.lib.nbl_plan_set_launch_config(plan, ctypes.byref(ext.LaunchConfig())))
        ext.set_options(precision=prev["precision"], grid=prev["grid"])
