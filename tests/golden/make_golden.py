"""Generate the golden fixtures in this directory from the reference itself.

    python tests/golden/make_golden.py

Runs the reference's own CPU core (oracle/_ref/libref_neighbours.so, built
from the reference sources by `make -C oracle ref`) on small seeded inputs and
stores, per case, the inputs and a SHA-256 digest of every output array
(plus the full outputs for the smallest cases).  The tests pin the C oracle
and the GPU engine to these files; they never need the reference at run time.
"""
import hashlib
import json
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT / "matscipy-neighbours_b200"))

import oracle as O  # noqa: E402
from matscipy_neighbours import _workloads as W  # noqa: E402


def digest(a):
    a = np.ascontiguousarray(a)
    return hashlib.sha256(a.tobytes()).hexdigest()


def cases():
    rng = np.random.default_rng(1234)
    yield "cube_1atom_1.1", dict(cell=np.eye(3), positions=[[0.5, 0.5, 0.5]],
                                 cutoff=1.1, pbc=True)
    yield "cube_1atom_1.5", dict(cell=np.eye(3), positions=[[0.5, 0.5, 0.5]],
                                 cutoff=1.5, pbc=True)
    yield "cube_1atom_TFT", dict(cell=np.eye(3), positions=[[0.5, 0.5, 0.5]],
                                 cutoff=1.1, pbc=[True, False, True])
    for k, pbc in enumerate([True, False, (True, False, True), (False, True, False)]):
        yield f"cubic40_{k}", dict(cell=5.0 * np.eye(3),
                                   positions=rng.uniform(0, 5.0, size=(40, 3)),
                                   cutoff=1.7, pbc=pbc)
    rng = np.random.default_rng(7)
    tri = np.array([[4.0, 0.0, 0.0], [1.3, 3.7, 0.0], [0.8, 0.6, 4.2]])
    frac = rng.uniform(-0.3, 1.3, size=(30, 3))
    for k, pbc in enumerate([True, False, (True, True, False)]):
        yield f"triclinic30_{k}", dict(cell=tri, positions=frac @ tri, cutoff=1.6,
                                       pbc=pbc)
    rng = np.random.default_rng(3)
    pos = rng.uniform(0, 6.0, size=(250, 3))
    for k, pbc in enumerate([True, False, (True, False, True)]):
        yield f"vacuum250_{k}", dict(cell=120.0 * np.eye(3), positions=pos, cutoff=1.5,
                                     pbc=pbc)
    rng = np.random.default_rng(99)
    pos = rng.uniform(0, 6.0, size=(25, 3))
    pos[3] += 6.0 * np.eye(3)[0]
    pos[7] -= 2 * 6.0 * np.eye(3)[1]
    pos[11] += 3 * 6.0 * np.eye(3)[2]
    for k, pbc in enumerate([True, False, (True, False, True)]):
        yield f"outside25_{k}", dict(cell=6.0 * np.eye(3), positions=pos, cutoff=1.5,
                                     pbc=pbc)
    rng = np.random.default_rng(2024)
    c = np.array([[5.0, 0.0, 0.0], [0.5, 4.5, 0.0], [0.2, 0.3, 5.5]])
    yield "invariant35", dict(cell=c, positions=rng.uniform(-1, 6, size=(35, 3)),
                              cutoff=1.9, pbc=True)
    yield "per_atom3", dict(cell=10.0 * np.eye(3),
                            positions=[[0.0, 0, 0], [1.0, 0, 0], [2.5, 0, 0]],
                            cutoff=np.array([0.4, 0.4, 1.2]), pbc=False)
    yield "per_type3", dict(cell=10.0 * np.eye(3),
                            positions=[[0.0, 0, 0], [1.0, 0, 0], [2.0, 0, 0]],
                            cutoff=np.array([[0.5, 1.5], [1.5, 0.5]]), pbc=False,
                            types=np.array([0, 1, 0], dtype=np.int32))
    w = W.plain_small()
    yield "plain_small_1000", dict(cell=w["cell"], positions=w["positions"],
                                   cutoff=w["cutoff"], pbc=w["pbc"])
    w = W.fcc_bulk(reps=8)
    yield "fcc_bulk_8", dict(cell=w["cell"], positions=w["positions"],
                             cutoff=w["cutoff"], pbc=w["pbc"])
    w = W.sparse_slab(n=4000, box=80.0, z0=36.0, z1=44.0)
    yield "slab_4000", dict(cell=w["cell"], positions=w["positions"],
                            cutoff=w["cutoff"], pbc=w["pbc"], types=w["numbers"],
                            quantities="ijdD")
    for k, s in enumerate(W.batched_systems(nsys=12)):
        yield f"batched_{k}", dict(cell=s["cell"], positions=s["positions"],
                                   cutoff=s["cutoff"], pbc=s["pbc"])
    w = W.diff_lattice(shape=(8, 8, 6))
    yield "diff_lattice_384", dict(cell=w["cell"], positions=w["positions"],
                                   cutoff=w["cutoff"], pbc=w["pbc"])


def main():
    if not O.ref_available():
        O.build()
    manifest = {}
    arrays = {}
    for name, c in cases():
        q = c.get("quantities", "ijdDS")
        pos = np.ascontiguousarray(c["positions"], dtype=float).reshape(-1, 3)
        cell = np.ascontiguousarray(c["cell"], dtype=float)
        pbc = np.broadcast_to(np.asarray(c["pbc"], dtype=bool), (3,)).copy()
        cut = c["cutoff"]
        types = c.get("types")
        out = O.ref_neighbour_list(q, cell, pos, cut, pbc, types=types)
        entry = {"quantities": q, "npairs": int(len(out[0])),
                 "digest": {k: digest(v) for k, v in zip(q, out)}}
        arrays[f"{name}/positions"] = pos
        arrays[f"{name}/cell"] = cell
        arrays[f"{name}/pbc"] = pbc
        arrays[f"{name}/cutoff"] = np.asarray(cut, dtype=float)
        entry["cutoff_is_scalar"] = isinstance(cut, float)
        if types is not None:
            arrays[f"{name}/types"] = np.asarray(types, dtype=np.int32)
        if entry["npairs"] <= 2000:
            for k, v in zip(q, out):
                arrays[f"{name}/out_{k}"] = v
        manifest[name] = entry
    np.savez_compressed(HERE / "golden_inputs.npz", **arrays)
    (HERE / "golden_manifest.json").write_text(json.dumps(manifest, indent=1,
                                                          sort_keys=True))
    print(f"{len(manifest)} cases written")


if __name__ == "__main__":
    main()
