"""Parity at the benchmark's full sizes: the engine's output against the
reference's own CPU core (oracle/_ref; the C restatement where that core was
not built) on the very inputs the benchmark times.

* dense bulk: 1,048,576-atom sheared FCC, rc 5 A, "ijdDS" (47.8 M pairs,
  2.5 GB of output), FP32 filter and plain FP64, dense and hashed grids;
* sparse slab: 200,000 atoms, pbc (T, T, F), per-type cutoffs, "ijdD", every
  precision x grid combination;
* batched: all 4,096 small systems through the batched graph launch, each
  system compared with the checker run on that system alone;
* differentiation lattice: 131,072 atoms, rc 6 A, "ijdDS".

The bar is the one of every parity test here: the same arrays, bit for bit,
in the same order (the reference's own GPU-vs-CPU test,
tests/test_neighbour_list_gpu.cc:57-91, compares canonically sorted lists
with a 1e-12 tolerance).  Large outputs come back to the host one quantity at
a time.
"""
import numpy as np
import pytest

from conftest import assert_same_lists

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def _checker(oracle):
    if oracle.ref_available():
        import os
        oracle.ref_set_threads(len(os.sched_getaffinity(0)))
        return oracle.ref_neighbour_list
    return oracle.oracle_neighbour_list


@pytest.fixture(autouse=True)
def _restore_options():
    from matscipy_neighbours import set_options
    prev = set_options()
    yield
    set_options(precision=prev["precision"], grid=prev["grid"])


def _engine_device(w, q, precision, grid):
    """The public API with device positions: device outputs (torch)."""
    import torch

    import matscipy_neighbours as m
    m.set_options(precision=precision, grid=grid)
    pos = torch.from_numpy(np.ascontiguousarray(w["positions"])).cuda()
    kw = {}
    if w.get("numbers") is not None:
        kw["numbers"] = w["numbers"]
    out = m.neighbour_list(q, positions=pos, cell=w["cell"], pbc=w["pbc"],
                           cutoff=w["cutoff"], array_namespace=torch, **kw)
    torch.cuda.synchronize()
    return out if len(q) > 1 else (out,)


def _compare_device(got, want, q):
    """One quantity at a time: bounded host memory for the 2.5 GB lists."""
    if len(q) == 1:
        want = (want,)
    assert len(got) == len(want)
    for c, g, w in zip(q, got, want):
        assert_same_lists(g.cpu().numpy(), w, c)


# --- dense bulk, 1,048,576 atoms -------------------------------------------

@pytest.fixture(scope="module")
def dense_bulk(oracle):
    from matscipy_neighbours import _workloads as W
    w = W.fcc_bulk()
    want = _checker(oracle)("ijdDS", w["cell"], w["positions"], w["cutoff"], w["pbc"])
    return w, want


@pytest.mark.parametrize("precision,grid", [("fp32", "auto"), ("fp64", "auto"),
                                            ("fp32", "hashed")])
def test_dense_bulk_full_size(dense_bulk, precision, grid):
    w, want = dense_bulk
    assert len(want[0]) == 47812982
    got = _engine_device(w, "ijdDS", precision, grid)
    _compare_device(got, want, "ijdDS")


# --- sparse slab, 200,000 atoms, per-type cutoffs ----------------------------

@pytest.fixture(scope="module")
def slab(oracle):
    from matscipy_neighbours import _workloads as W
    w = W.sparse_slab()
    want = _checker(oracle)("ijdD", w["cell"], w["positions"], w["cutoff"], w["pbc"],
                            types=w["numbers"])
    return w, want


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("grid", ["auto", "dense", "morton", "hashed"])
def test_sparse_slab_full_size(slab, precision, grid):
    w, want = slab
    got = _engine_device(w, "ijdD", precision, grid)
    _compare_device(got, want, "ijdD")


# --- batched, all 4,096 systems ---------------------------------------------

@pytest.fixture(scope="module")
def batch_systems(oracle):
    from matscipy_neighbours import _workloads as W
    systems = W.batched_systems(seed=1)
    fn = _checker(oracle)
    want = [fn("ijdDS", s["cell"], s["positions"], s["cutoff"], s["pbc"]) for s in systems]
    return systems, want


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_batched_4096_systems_each_system(batch_systems, precision):
    from matscipy_neighbours.batch import NeighbourListBatch
    systems, want = batch_systems
    b = NeighbourListBatch(systems, precision=precision, graph=True, autotune=True)
    b.run()
    b.run()  # a replay of the captured graph gives the same lists
    off = b.sys_offsets()
    outs = [t.cpu().numpy() for t in b.results()]
    b.close()
    assert off[-1] == sum(len(w[0]) for w in want)
    for s in range(len(systems)):
        got = tuple(o[off[s]:off[s + 1]] for o in outs)
        assert_same_lists(got, want[s], "ijdDS")


# --- differentiation lattice, 131,072 atoms --------------------------------

def test_diff_lattice_full_size(oracle):
    from matscipy_neighbours import _workloads as W
    w = W.diff_lattice()
    want = _checker(oracle)("ijdDS", w["cell"], w["positions"], w["cutoff"], w["pbc"])
    for precision in ("fp32", "fp64"):
        got = _engine_device(w, "ijdDS", precision, "auto")
        _compare_device(got, want, "ijdDS")
