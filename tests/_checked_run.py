"""The engine's checked build (libnbl_b200_checked.so) over every pair-pass
path, compared with the CPU oracle.  Run as a child process by
test_gpu_checked.py with MATSCIPY_NEIGHBOURS_CHECKED=1, because the library
is chosen once per process when the package is imported.

The checked build tests, inside the pair passes (warp and thread-per-atom),
every cell slice, candidate index, hit-word index and output slot (the slot must lie in its own row
[offsets[i], offsets[i+1])); a failed test would come back as
NBL_ERROR_INTERNAL ("device-side bound exceeded").  So a clean run here shows
that none of those indices leaves its bounds on these inputs, and the oracle
comparison shows the checks changed no result.  Prints "checked ok <n>" at
the end; any failure raises.
"""
import ctypes
import itertools
import pathlib
import sys

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[1]
for p in (ROOT / "tests", ROOT / "matscipy-neighbours_b200", ROOT / "oracle"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

import torch  # noqa: E402

import oracle  # noqa: E402
from _cases import digest, golden_cases  # noqa: E402
from conftest import assert_same_lists  # noqa: E402

import matscipy_neighbours as m  # noqa: E402
from matscipy_neighbours import _matscipy_neighbours as ext  # noqa: E402
from matscipy_neighbours import _workloads as W  # noqa: E402

DONE = [0]


def _loaded_libraries():
    names = set()
    with open("/proc/self/maps") as f:
        for line in f:
            if "libnbl_b200" in line:
                names.add(pathlib.Path(line.split()[-1]).name)
    return names


def _device_list(q, w, precision="fp32", grid="auto"):
    m.set_options(precision=precision, grid=grid)
    pos = torch.from_numpy(np.ascontiguousarray(w["positions"], dtype=float)).cuda()
    kw = {}
    if w.get("types") is not None:
        kw["numbers"] = w["types"]
    out = m.neighbour_list(q, positions=pos, cell=w["cell"], pbc=w["pbc"],
                           cutoff=w["cutoff"], array_namespace=torch, **kw)
    torch.cuda.synchronize()
    out = out if len(q) > 1 else (out,)
    return tuple(t.cpu().numpy() for t in out)


def _want(q, w):
    return oracle.oracle_neighbour_list(q, w["cell"], w["positions"], w["cutoff"],
                                        w["pbc"], types=w.get("types"))


def golden():
    for case in golden_cases():
        if case["npairs"] > 2_000_000:
            continue
        for precision, grid in itertools.product(("fp32", "fp64"),
                                                 ("dense", "morton", "hashed")):
            out = _device_list(case["quantities"], case, precision, grid)
            assert len(out[0]) == case["npairs"], case["name"]
            for q, a in zip(case["quantities"], out):
                assert digest(a) == case["digest"][q], (case["name"], q, precision, grid)
            DONE[0] += 1


def workloads():
    rng = np.random.default_rng(11)
    per_atom = W.plain_small(n=3000, box=15.0)
    per_atom["cutoff"] = rng.uniform(1.0, 2.6, size=3000)
    per_type = W.plain_small(n=3000, box=15.0)
    per_type["types"] = rng.integers(0, 2, size=3000).astype(np.int32)
    per_type["cutoff"] = np.array([[2.0, 2.6], [2.6, 3.1]])
    cases = [W.fcc_bulk(reps=10), W.sparse_slab(n=20000), W.diff_lattice(shape=(12, 12, 6)),
             per_atom, per_type]
    for w in cases:
        want = _want("ijdDS", w)
        for precision in ("fp32", "fp64"):
            assert_same_lists(_device_list("ijdDS", w, precision), want, "ijdDS")
            DONE[0] += 1
        # a subset of the quantities (the non-ALL5 fill)
        assert_same_lists(_device_list("ijd", w, "fp32"), want[:3], "ijd")
        DONE[0] += 1


def launch_shapes():
    rng = np.random.default_rng(17)
    cluster = dict(positions=rng.uniform(0.0, 6.0, size=(900, 3)), cell=18.0 * np.eye(3),
                   pbc=np.array([True, True, True]), cutoff=2.9)
    plan = ext.plan_for(0)
    for w in (cluster, W.fcc_bulk(reps=5, cutoff=4.0)):
        want = _want("ijdDS", w)
        for precision in ("fp32", "fp64"):
            for cw, big, grp, fw, tile, strided in itertools.product(
                    (2, 4, 8), (0, 1), (2, 4), (2, 4, 8), (32, 7), (0, 1)):
                if precision == "fp64" and grp == 2:
                    continue
                cfg = ext.LaunchConfig(0, 0, strided, 1 - strided, cw, fw, grp, big, tile)
                ext.check(ext.lib.nbl_plan_set_launch_config(plan, ctypes.byref(cfg)))
                assert_same_lists(_device_list("ijdDS", w, precision), want, "ijdDS")
                DONE[0] += 1
    ext.check(ext.lib.nbl_plan_set_launch_config(plan, ctypes.byref(ext.LaunchConfig())))


def row_slices():
    from matscipy_neighbours.distributed import neighbour_list_rows
    w = W.fcc_bulk(reps=8)
    want = _want("ijdDS", w)
    pos = torch.from_numpy(np.ascontiguousarray(w["positions"])).cuda()
    n = len(pos)
    for precision in ("fp32", "fp64"):
        m.set_options(precision=precision, grid="auto")
        parts = [neighbour_list_rows("ijdDS", pos, w["cell"], w["pbc"], w["cutoff"], r)
                 for r in ((0, n // 3), (n // 3, n // 3 + 17), (n // 3 + 17, n))]
        torch.cuda.synchronize()
        got = tuple(np.concatenate([p[k].cpu().numpy() for p in parts]) for k in range(5))
        assert_same_lists(got, want, "ijdDS")
        DONE[0] += 1


def batch():
    from matscipy_neighbours.batch import NeighbourListBatch
    systems = W.batched_systems(seed=2, nsys=40)
    want = [_want("ijdDS", s) for s in systems]
    for precision in ("fp32", "fp64"):
        b = NeighbourListBatch(systems, precision=precision, graph=True, autotune=False)
        b.run()
        b.run()
        off = b.sys_offsets()
        outs = [t.cpu().numpy() for t in b.results()]
        b.close()
        for s in range(len(systems)):
            assert_same_lists(tuple(o[off[s]:off[s + 1]] for o in outs), want[s], "ijdDS")
        DONE[0] += 1


def matrix_and_forces():
    w = W.fcc_bulk(reps=6)
    i, j, D = _want("ijD", w)
    idx, dist, count = m.neighbour_matrix(positions=w["positions"], cell=w["cell"],
                                          pbc=w["pbc"], cutoff=w["cutoff"],
                                          max_neighbours=200)
    idx, dist, count = (np.asarray(x) for x in (idx, dist, count))
    deg = np.bincount(i, minlength=len(w["positions"]))
    assert np.array_equal(count, deg)
    start = np.concatenate([[0], np.cumsum(deg)])
    for a in range(len(deg)):
        assert np.array_equal(idx[a, :deg[a]], j[start[a]:start[a + 1]])
        assert np.array_equal(dist[a, :deg[a]].view(np.int64),
                              D[start[a]:start[a + 1]].view(np.int64))
    DONE[0] += 1
    # the fused force sink against numpy over the oracle's pairs
    d = np.sqrt((D * D).sum(axis=1))
    s6 = (1.0 / (d * d)) ** 3
    coef = -24.0 * s6 * (2.0 * s6 - 1.0) / (d * d)
    f = np.zeros((len(w["positions"]), 3))
    np.add.at(f, i, coef[:, None] * D)
    e = 0.5 * np.sum(4.0 * (s6 * s6 - s6))
    ge, gf = m.lennard_jones(w["positions"], float(w["cutoff"]), cell=w["cell"], pbc=w["pbc"])
    scale = np.abs(f).max()
    assert np.allclose(gf, f, rtol=1e-12, atol=1e-12 * scale)
    assert abs(ge - e) <= 1e-12 * max(1.0, abs(e))
    DONE[0] += 1


def thread_per_atom():
    """The thread-per-atom pair passes over the golden cases (every grid) and
    the workload shapes."""
    plan = ext.plan_for(0)
    cfg = ext.LaunchConfig(thread_per_atom=1, one_launch_atoms=-1)
    ext.check(ext.lib.nbl_plan_set_launch_config(plan, ctypes.byref(cfg)))
    try:
        for case in golden_cases():
            if case["npairs"] > 2_000_000:
                continue
            for grid in ("dense", "morton", "hashed"):
                out = _device_list(case["quantities"], case, "fp32", grid)
                for q, a in zip(case["quantities"], out):
                    assert digest(a) == case["digest"][q], (case["name"], q, grid)
                DONE[0] += 1
        for w in (W.sparse_slab(n=20000), W.fcc_bulk(reps=6)):
            want = _want("ijdDS", w)
            assert_same_lists(_device_list("ijdDS", w), want, "ijdDS")
            assert_same_lists(_device_list("ijd", w), want[:3], "ijd")
            DONE[0] += 2
    finally:
        ext.check(ext.lib.nbl_plan_set_launch_config(plan, ctypes.byref(ext.LaunchConfig())))


def main():
    assert ext.CHECKED and ext._LIB_PATH.name == "libnbl_b200_checked.so"
    torch.cuda.set_device(0)
    golden()
    workloads()
    launch_shapes()
    row_slices()
    batch()
    matrix_and_forces()
    thread_per_atom()
    libs = _loaded_libraries()
    assert libs == {"libnbl_b200_checked.so"}, libs
    print(f"checked ok {DONE[0]}")


if __name__ == "__main__":
    main()
