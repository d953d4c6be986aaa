"""Public neighbour-list API, a drop-in for ``matscipy_neighbours.neighbours``.

Same functions, arguments, defaults, return conventions and exception classes
as the reference's pure-Python layer
(``language_bindings/python/matscipy_neighbours/neighbours.py``), on top of the
B200 engine binding ``_matscipy_neighbours`` instead of the reference's
C-extension.  Every pair list is computed on the GPU:

* host (numpy) positions -> the engine copies them in and the results back
  (the reference's "host fast path", ``neighbours.py:249-257``);
* device positions (torch, cupy, anything with ``__dlpack__``) -> results stay
  on the device as DLPack tensors (``neighbours.py:259-288``).
"""

import numpy as np

from . import _matscipy_neighbours as _ext

try:  # pragma: no cover - ase is optional
    from ase.data import atomic_numbers as _atomic_numbers
except ImportError:  # pragma: no cover
    _atomic_numbers = {}

__all__ = [
    "neighbour_list",
    "neighbour_matrix",
    "first_neighbours",
    "get_jump_indicies",
    "triplet_list",
    "mic",
    "coordination",
    "DLPackTensor",
]

_DLPACK_CPU = 1
_DLPACK_CUDA = 2


def mic(dr, cell, pbc=None):
    """Minimum image convention for distance vectors ``dr`` (n, 3) in a cell
    whose rows are the lattice vectors (``neighbours.py:39-62``)."""
    dr = np.asarray(dr, dtype=float)
    cell = np.asarray(cell, dtype=float)
    rec = np.linalg.inv(cell)
    if pbc is not None:
        rec = rec * np.asarray(pbc, dtype=int).reshape(3, 1)
    return dr - np.round(dr @ rec) @ cell


class DLPackTensor:
    """A zero-copy DLPack tensor produced by the neighbour list; consume it with
    any framework's ``from_dlpack`` (``neighbours.py:65-81``)."""

    __slots__ = ("_capsule", "_device")

    def __init__(self, capsule, device):
        self._capsule = capsule
        self._device = device

    def __dlpack__(self, *args, **kwargs):
        return self._capsule

    def __dlpack_device__(self):
        return self._device


_DLPackArray = DLPackTensor


def _dlpack_device(x):
    fn = getattr(x, "__dlpack_device__", None)
    if fn is None:
        return None
    try:
        dt, did = fn()
        return (int(dt), int(did))
    except Exception:  # pragma: no cover - defensive
        return None


def _is_on_device(x):
    dev = _dlpack_device(x)
    return dev is not None and dev[0] != _DLPACK_CPU


def _resolve_device(device, on_device_input):
    """``device``: None (follow the input), "cpu", "cuda"/"gpu", an int id or
    ("cuda", id) -> (use_gpu, device_id) (``neighbours.py:111-128``)."""
    if device is None:
        return (on_device_input, -1)
    if isinstance(device, str):
        d = device.lower()
        if d == "cpu":
            return (False, -1)
        if d in ("cuda", "gpu", "rocm", "hip"):
            return (True, -1)
        raise ValueError(f"Unknown device {device!r}.")
    if isinstance(device, int):
        return (True, device)
    if isinstance(device, (tuple, list)) and len(device) == 2:
        return (True, int(device[1]))
    raise ValueError(f"Unknown device {device!r}.")


def _consume(wrappers, array_namespace, use_gpu):
    """None -> cupy on the device, numpy on the host; "dlpack" -> the
    DLPackTensors; a module -> its from_dlpack (``neighbours.py:131-142``)."""
    if array_namespace == "dlpack":
        return wrappers
    if array_namespace is None:
        if use_gpu:
            import cupy as array_namespace
        else:
            array_namespace = np
    return [array_namespace.from_dlpack(w) for w in wrappers]


def _host_metadata(cell, pbc, numbers, cell_origin, nat, *, positions=None):
    """Normalise the host-side geometry (``neighbours.py:145-164``): cell
    shrink-wrapped around host positions when None, origin 0, pbc False,
    numbers 1, inv_cell = inv(cell.T)."""
    if cell is None:
        r = np.asarray(positions, dtype=float)
        rmin, rmax = r.min(axis=0), r.max(axis=0)
        cell_origin = rmin if cell_origin is None else cell_origin
        cell = np.diag(rmax - rmin)
    if cell_origin is None:
        cell_origin = np.zeros(3)
    if pbc is None:
        pbc = np.zeros(3, dtype=bool)
    if numbers is None:
        numbers = np.ones(nat, dtype=np.int32)
    cell = np.ascontiguousarray(np.asarray(cell, dtype=float))
    cell_origin = np.ascontiguousarray(np.asarray(cell_origin, dtype=float))
    pbc = np.ascontiguousarray(np.broadcast_to(pbc, (3,)), dtype=bool)
    numbers = np.ascontiguousarray(np.asarray(numbers), dtype=np.int32)
    inv_cell = np.ascontiguousarray(np.linalg.inv(cell.T))
    return cell_origin, cell, inv_cell, pbc, numbers


def _resolve_cutoff(cutoff, numbers):
    """Element-pair dict -> (Zmax+1)^2 matrix with 0 for unspecified pairs;
    scalars and per-atom arrays pass through (``neighbours.py:167-181``)."""
    if isinstance(cutoff, dict):
        maxnum = int(np.max(numbers))
        matrix = np.zeros((maxnum + 1, maxnum + 1), dtype=float)
        for (el1, el2), c in cutoff.items():
            el1 = _atomic_numbers.get(el1, el1)
            el2 = _atomic_numbers.get(el2, el2)
            if el1 <= maxnum and el2 <= maxnum:
                matrix[el1, el2] = c
                matrix[el2, el1] = c
        return matrix, numbers
    return cutoff, numbers


def _gather(atoms, positions, cell, pbc, numbers, cell_origin):
    if atoms is not None:
        if any(x is not None for x in (positions, cell, pbc, numbers, cell_origin)):
            raise ValueError("Cannot combine an ASE Atoms object with explicit "
                             "positions/cell/pbc/numbers/cell_origin.")
        return (atoms.positions, np.asarray(atoms.cell), atoms.pbc,
                atoms.numbers.astype(np.int32), np.zeros(3))
    if positions is None:
        raise ValueError("Provide either an ASE Atoms object or a positions array.")
    return positions, cell, pbc, numbers, cell_origin


def _route(positions, device, cell):
    on_device = _is_on_device(positions)
    use_gpu, device_id = _resolve_device(device, on_device)
    if on_device and not use_gpu:
        raise ValueError("device='cpu' with device-resident positions is not "
                         "supported; move the array to the host first.")
    if use_gpu and not getattr(_ext, "_has_gpu", 0):
        raise RuntimeError("GPU requested but no CUDA device is available.")
    if use_gpu and on_device and cell is None:
        raise ValueError("cell must be given for device-resident positions.")
    return on_device, use_gpu, device_id


def neighbour_list(quantities, atoms=None, cutoff=None, *, positions=None,
                   cell=None, pbc=None, numbers=None, cell_origin=None,
                   device=None, array_namespace=None):
    """Neighbour list of an atomic configuration (``neighbours.py:200-288``).

    quantities: any string over ``i`` (first index), ``j`` (second index),
    ``d`` (distance), ``D`` (distance vector), ``S`` (cell shift); one output
    per character in that order, a bare array for one character.  ``cutoff``:
    a float, a per-atom radius array (pair cutoff = r_i + r_j) or a
    ``{(el1, el2): c}`` dict / square matrix used with ``numbers``.  Outputs
    satisfy ``D == r[j] - r[i] + S @ cell`` and are sorted by ``i``.
    ``device`` and ``array_namespace`` as in the reference: device positions
    give device outputs (cupy by default; pass ``array_namespace=torch`` or
    ``"dlpack"`` for others)."""
    if cutoff is None:
        raise ValueError("Please provide a value for the cutoff radius.")
    positions, cell, pbc, numbers, cell_origin = _gather(
        atoms, positions, cell, pbc, numbers, cell_origin)
    on_device, use_gpu, device_id = _route(positions, device, cell)

    if not use_gpu and array_namespace is None:
        positions = np.ascontiguousarray(positions, dtype=float)
        co, ce, inv, pb, nums = _host_metadata(cell, pbc, numbers, cell_origin,
                                               len(positions), positions=positions)
        rc, nums = _resolve_cutoff(cutoff, nums)
        return _ext.neighbour_list(quantities, co, ce, inv, pb, positions, rc, nums)

    nat = int(positions.shape[0])
    if on_device:
        py_in, host_pos = positions, np.empty((0, 3), dtype=float)
    else:
        py_in, host_pos = None, np.ascontiguousarray(positions, dtype=float)
        if use_gpu and device_id < 0:
            device_id = 0
    co, ce, inv, pb, nums = _host_metadata(
        cell, pbc, numbers, cell_origin, nat,
        positions=None if on_device else host_pos)
    rc, nums = _resolve_cutoff(cutoff, nums)
    capsules = _ext.neighbour_list_dlpack(quantities, co, ce, inv, pb, host_pos, rc,
                                          nums, 1 if use_gpu else 0, py_in, device_id)
    if use_gpu:
        out_id = _dlpack_device(positions)[1] if on_device else device_id
        out_dev = (_ext._device_type, out_id)
    else:
        out_dev = (_DLPACK_CPU, 0)
    wrappers = [DLPackTensor(c, out_dev) for c in capsules]
    arrays = _consume(wrappers, array_namespace, use_gpu)
    return arrays[0] if len(quantities) == 1 else tuple(arrays)


def neighbour_matrix(atoms=None, cutoff=None, max_neighbours=None, *,
                     positions=None, cell=None, pbc=None, numbers=None,
                     cell_origin=None, device=None, array_namespace=None):
    """Dense fixed-capacity neighbour list ``(idx, dist, count)``
    (``neighbours.py:291-357``): row a holds atom a's neighbours (``j`` and
    ``D``), unused slots are 0, ``count`` is the true degree; ``ValueError`` if
    any atom has more than ``max_neighbours`` neighbours."""
    if cutoff is None:
        raise ValueError("Please provide a value for the cutoff radius.")
    if max_neighbours is None:
        raise ValueError("Please provide max_neighbours (the row capacity).")
    positions, cell, pbc, numbers, cell_origin = _gather(
        atoms, positions, cell, pbc, numbers, cell_origin)
    on_device, use_gpu, device_id = _route(positions, device, cell)
    nat = int(positions.shape[0])
    if on_device:
        py_in, host_pos = positions, np.empty((0, 3), dtype=float)
    else:
        py_in, host_pos = None, np.ascontiguousarray(positions, dtype=float)
        if use_gpu and device_id < 0:
            device_id = 0
    co, ce, inv, pb, nums = _host_metadata(
        cell, pbc, numbers, cell_origin, nat,
        positions=None if on_device else host_pos)
    rc, nums = _resolve_cutoff(cutoff, nums)
    idx_cap, dist_cap, count_cap, overflow = _ext.neighbour_matrix_dlpack(
        co, ce, inv, pb, host_pos, rc, int(max_neighbours), nums,
        1 if use_gpu else 0, py_in, device_id)
    if overflow:
        raise ValueError(
            f"max_neighbours={max_neighbours} is too small: some atom has more "
            "neighbours than that. Retry with a larger max_neighbours.")
    if use_gpu:
        out_id = _dlpack_device(positions)[1] if on_device else device_id
        out_dev = (_ext._device_type, out_id)
    else:
        out_dev = (_DLPACK_CPU, 0)
    wrappers = [DLPackTensor(c, out_dev) for c in (idx_cap, dist_cap, count_cap)]
    return tuple(_consume(wrappers, array_namespace, use_gpu))


# Pure extension functions, re-exported unchanged (neighbours.py:34-36).
first_neighbours = _ext.first_neighbours
get_jump_indicies = _ext.get_jump_indicies


def triplet_list(first_neighbours, abs_dr_p=None, cutoff=None):
    """Triplet list from a first-neighbour (row-start) array
    (``neighbours.py:360-370``): distances are used only with a cutoff.  A
    device array (torch CUDA tensor or CUDA __dlpack__) is handled on its GPU
    and gives torch CUDA tensors."""
    if _is_on_device(first_neighbours):
        if abs_dr_p is not None and cutoff is not None:
            return _ext.triplet_list(first_neighbours, abs_dr_p, float(cutoff))
        return _ext.triplet_list(first_neighbours)
    first_neighbours = np.ascontiguousarray(first_neighbours, dtype=np.int32)
    if abs_dr_p is not None and cutoff is not None:
        abs_dr_p = np.ascontiguousarray(abs_dr_p, dtype=float)
        return _ext.triplet_list(first_neighbours, abs_dr_p, float(cutoff))
    return _ext.triplet_list(first_neighbours)


def coordination(atoms=None, cutoff=None, *, positions=None, cell=None, pbc=None,
                 numbers=None, cell_origin=None, device=None, array_namespace=None):
    """Number of neighbours of each atom (``neighbours.py:373-422``), from the
    count pass alone (the pairs are never materialised)."""
    positions, cell, pbc, numbers, cell_origin = _gather(
        atoms, positions, cell, pbc, numbers, cell_origin)
    on_device, use_gpu, device_id = _route(positions, device, cell)
    nat = int(positions.shape[0])
    host_pos = None if on_device else np.ascontiguousarray(positions, dtype=float)
    co, ce, inv, pb, nums = _host_metadata(cell, pbc, numbers, cell_origin, nat,
                                           positions=host_pos)
    rc, nums = _resolve_cutoff(cutoff, nums)
    counts = _ext.coordination(co, ce, inv, pb, host_pos, rc, nums,
                               device_id=max(device_id, 0),
                               py_in=positions if on_device else None)
    if use_gpu:
        out_id = _dlpack_device(positions)[1] if on_device else max(device_id, 0)
        return _consume([DLPackTensor(counts.__dlpack__(), (_ext._device_type, out_id))],
                        array_namespace, True)[0]
    host = counts.cpu().numpy().astype(np.int64)
    if array_namespace is None:
        return host
    if array_namespace == "dlpack":
        return DLPackTensor(host.__dlpack__(), host.__dlpack_device__())
    return array_namespace.from_dlpack(host)
