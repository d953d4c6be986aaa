"""GPU engine vs the CPU oracle: bit-identical outputs (same arrays, same
order) for every precision mode and grid layout, on the reference's golden
cases, the five workload shapes at reduced size, and edge cases.  The golden
and edge cases run through three count paths: the one-CTA launch that small
systems take by default, the multi-kernel sequence with warp work items
(single-CTA path off) and the multi-kernel sequence with the thread-per-atom
pair passes."""
import itertools

import numpy as np
import pytest

from _cases import digest, golden_cases
from conftest import assert_same_lists

pytestmark = pytest.mark.gpu

CASES = golden_cases()
MODES = list(itertools.product(["fp32", "fp64"], ["dense", "morton", "hashed"]))


@pytest.fixture(autouse=True)
def _restore_options():
    from matscipy_neighbours import set_options
    prev = set_options()
    yield
    set_options(precision=prev["precision"], grid=prev["grid"])


@pytest.fixture(params=["one_cta", "multi_kernel", "thread_per_atom"])
def count_path(request):
    """The plan's single-CTA threshold: its largest value (every golden and
    edge case that fits takes the one-CTA count phase), or -1 (never); and
    the multi-kernel sequence with the thread-per-atom pair passes forced on."""
    import ctypes
    from matscipy_neighbours import _matscipy_neighbours as ext
    plan = ext.plan_for(0)
    cfg = ext.LaunchConfig(one_launch_atoms=2048 if request.param == "one_cta" else -1,
                           thread_per_atom=1 if request.param == "thread_per_atom" else -1)
    ext.check(ext.lib.nbl_plan_set_launch_config(plan, ctypes.byref(cfg)))
    yield request.param
    ext.check(ext.lib.nbl_plan_set_launch_config(plan, ctypes.byref(ext.LaunchConfig())))


def engine(q, w, precision="fp32", grid="auto"):
    import matscipy_neighbours as m
    from matscipy_neighbours import _matscipy_neighbours as ext
    m.set_options(precision=precision, grid=grid)
    cell = np.asarray(w["cell"], dtype=float)
    pbc = np.broadcast_to(np.asarray(w["pbc"], dtype=bool), (3,))
    args = [q, np.zeros(3), cell, np.linalg.inv(cell.T), pbc,
            np.asarray(w["positions"], dtype=float).reshape(-1, 3), w["cutoff"]]
    if w.get("types") is not None:
        args.append(np.asarray(w["types"], dtype=np.int32))
    return ext.neighbour_list(*args)


def expected(oracle, q, w):
    return oracle.oracle_neighbour_list(q, w["cell"], w["positions"], w["cutoff"],
                                        w["pbc"], types=w.get("types"))


@pytest.mark.parametrize("mode", MODES, ids=["-".join(m) for m in MODES])
@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_golden(case, mode, count_path):
    out = engine(case["quantities"], case, *mode)
    if len(case["quantities"]) == 1:
        out = (out,)
    assert len(out[0]) == case["npairs"]
    for q, a in zip(case["quantities"], out):
        assert digest(a) == case["digest"][q], q


def _workloads():
    from matscipy_neighbours import _workloads as W
    out = [("plain_small", W.plain_small()),
           ("fcc_bulk_16", W.fcc_bulk(reps=16)),
           ("slab_20k", W.sparse_slab(n=20000)),
           ("diff_lattice_16", W.diff_lattice(shape=(16, 16, 8)))]
    for k, s in enumerate(W.batched_systems(nsys=24, seed=5)):
        out.append((f"batched_{k}", s))
    return out


WL = _workloads()


@pytest.mark.parametrize("mode", MODES, ids=["-".join(m) for m in MODES])
@pytest.mark.parametrize("name,w", WL, ids=[n for n, _ in WL])
def test_workloads_vs_oracle(oracle, name, w, mode):
    q = w.get("quantities", "ijdDS")
    wl = dict(w)
    if "numbers" in w:
        wl["types"] = w["numbers"]
    assert_same_lists(engine(q, wl, *mode), expected(oracle, q, wl), q)


# --- edge cases ------------------------------------------------------------

def _edge_cases():
    rng = np.random.default_rng(11)
    out = []
    out.append(("empty", dict(cell=10 * np.eye(3), positions=np.zeros((0, 3)),
                              cutoff=2.0, pbc=True)))
    out.append(("one_atom_periodic", dict(cell=np.eye(3), positions=[[0.2, 0.3, 0.9]],
                                          cutoff=2.3, pbc=True)))
    # every atom in one cell: a 0.5 A cluster, 700 atoms, candidates > tile
    out.append(("one_dense_cell", dict(cell=40 * np.eye(3),
                                       positions=rng.uniform(10, 10.5, size=(1500, 3)),
                                       cutoff=3.0, pbc=True)))
    # box much smaller than the cutoff: many periodic images (nscan > 1)
    out.append(("tiny_box", dict(cell=np.array([[1.5, 0, 0], [0.3, 1.2, 0],
                                                [0.1, 0.2, 1.4]]),
                                 positions=rng.uniform(0, 1.2, size=(3, 3)),
                                 cutoff=4.0, pbc=True)))
    # atoms far outside a non-periodic box (the shift quirk)
    pos = rng.uniform(0, 8, size=(60, 3))
    pos[:10, 2] += 30.0
    pos[10:20, 2] -= 25.0
    out.append(("outside_nonperiodic", dict(cell=8 * np.eye(3), positions=pos,
                                            cutoff=2.5, pbc=(True, True, False))))
    # periodic atoms many images away
    pos = rng.uniform(0, 6, size=(40, 3))
    pos[::3] += 60.0
    pos[1::3] -= 35.0
    out.append(("far_images_periodic", dict(cell=6 * np.eye(3), positions=pos,
                                            cutoff=2.0, pbc=True)))
    # triclinic, strongly sheared
    c = np.array([[6.0, 0, 0], [4.5, 5.0, 0], [-3.0, 2.5, 5.5]])
    out.append(("sheared", dict(cell=c, positions=rng.uniform(0, 1, size=(200, 3)) @ c,
                                cutoff=2.7, pbc=True)))
    # per-type with out-of-range types (fall back to the global test)
    types = rng.integers(-1, 4, size=300).astype(np.int32)
    out.append(("types_out_of_range", dict(cell=12 * np.eye(3),
                                           positions=rng.uniform(0, 12, size=(300, 3)),
                                           cutoff=np.array([[2.0, 2.5, 3.0],
                                                            [2.5, 1.0, 0.0],
                                                            [3.0, 0.0, 3.5]]),
                                           pbc=True, types=types)))
    # per-atom radii including zeros
    r = rng.uniform(0, 1.6, size=250)
    r[::7] = 0.0
    out.append(("per_atom_zeros", dict(cell=10 * np.eye(3),
                                       positions=rng.uniform(0, 10, size=(250, 3)),
                                       cutoff=r, pbc=(False, True, True))))
    # large per-type matrix (119 x 119, as a dict over element numbers gives)
    m = np.zeros((119, 119))
    m[1, 8] = m[8, 1] = 1.2
    m[8, 8] = 3.1
    m[1, 1] = 0.9
    types = rng.choice([1, 8], size=400).astype(np.int32)
    out.append(("big_type_table", dict(cell=14 * np.eye(3),
                                       positions=rng.uniform(0, 14, size=(400, 3)),
                                       cutoff=m, pbc=True, types=types)))
    # cutoff exactly at lattice spacing (ties decided by FP64 ordering)
    g = np.stack(np.meshgrid(*[np.arange(6)] * 3, indexing="ij"), -1).reshape(-1, 3)
    out.append(("lattice_ties", dict(cell=6.0 * np.eye(3), positions=g * 1.0,
                                     cutoff=1.0, pbc=True)))
    out.append(("lattice_ties_sqrt2", dict(cell=6.0 * np.eye(3), positions=g * 1.0,
                                           cutoff=float(np.sqrt(2.0)), pbc=True)))
    return out


EDGE = _edge_cases()


@pytest.mark.parametrize("mode", MODES, ids=["-".join(m) for m in MODES])
@pytest.mark.parametrize("name,w", EDGE, ids=[n for n, _ in EDGE])
def test_edge_cases(oracle, name, w, mode, count_path):
    q = "ijdDS"
    assert_same_lists(engine(q, w, *mode), expected(oracle, q, w), q)


@pytest.mark.parametrize("q", ["i", "j", "D", "d", "S", "Sdj", "ii", "DDd", ""])
def test_quantity_subsets_and_order(oracle, q):
    from matscipy_neighbours import _workloads as W
    w = W.plain_small()
    got = engine(q, w)
    want = expected(oracle, q, w) if q else ()
    if q == "":
        assert got == ()
        return
    assert_same_lists(got, want, q)


def test_non_finite_position_is_an_error():
    w = dict(cell=5 * np.eye(3), positions=np.array([[0.0, 0, 0], [np.nan, 1, 1]]),
             cutoff=1.0, pbc=True)
    with pytest.raises(RuntimeError):
        engine("ij", w)


def test_zero_volume_raises_runtime_error():
    from matscipy_neighbours import _matscipy_neighbours as ext
    with pytest.raises(RuntimeError, match="Zero cell volume"):
        ext.neighbour_list("i", np.zeros(3), np.array([[1.0, 0, 0], [2.0, 0, 0],
                                                       [0, 0, 1.0]]),
                           np.zeros((3, 3)), np.array([True] * 3), np.zeros((1, 3)), 1.0)


def test_single_quantity_is_bare_array():
    import matscipy_neighbours as m
    out = m.neighbour_list("i", positions=[[0.5, 0.5, 0.5]], cell=np.eye(3), pbc=True,
                           cutoff=1.1)
    assert isinstance(out, np.ndarray) and len(out) == 6
