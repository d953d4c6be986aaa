"""Shared test inputs: the golden fixtures and the reference's known answers."""
import json
import pathlib

import numpy as np

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"


def golden_cases():
    manifest = json.loads((GOLDEN / "golden_manifest.json").read_text())
    data = np.load(GOLDEN / "golden_inputs.npz")
    out = []
    for name, e in sorted(manifest.items()):
        cut = data[f"{name}/cutoff"]
        cut = float(cut) if e["cutoff_is_scalar"] else np.array(cut)
        types = data[f"{name}/types"] if f"{name}/types" in data.files else None
        full = {q: data[f"{name}/out_{q}"] for q in e["quantities"]
                if f"{name}/out_{q}" in data.files}
        out.append(dict(name=name, quantities=e["quantities"], npairs=e["npairs"],
                        digest=e["digest"], positions=data[f"{name}/positions"],
                        cell=data[f"{name}/cell"], pbc=data[f"{name}/pbc"],
                        cutoff=cut, types=types, full=full))
    return out


def digest(a):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()
