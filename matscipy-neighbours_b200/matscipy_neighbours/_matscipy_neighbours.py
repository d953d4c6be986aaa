"""Binding of the B200 engine (``libnbl_b200.so``) under the names of the
reference's C-extension ``_matscipy_neighbours``.

Mirrors ``language_bindings/python/module.c:45-113`` (method table and the
``_has_gpu`` / ``_device_type`` constants), ``bind_py_neighbours.cc:88-268``
(``neighbour_list``: argument coercion, cutoff resolution, quantity parsing,
error classes, bare array for one quantity) and ``bind_py_dlpack.cc:231-408``
(``neighbour_list_dlpack``: DLPack capsules out, device positions in through
``__dlpack__``).

Every pair list is computed by the CUDA engine; there is no CPU path.  Host
(numpy) positions are copied to the GPU and the results copied back.  The
binding calls the engine through ctypes, which releases the GIL for the
duration of each call.  PyTorch is used here, and only here, for device
buffers, streams and DLPack interop.
"""

import ctypes
import os
import pathlib
import threading

import numpy as np

# MATSCIPY_NEIGHBOURS_CHECKED=1 selects the checked build of the engine (the
# same kernels with every device-side index tested; built by
# ``build.py --checked``).
CHECKED = os.environ.get("MATSCIPY_NEIGHBOURS_CHECKED", "0") not in ("", "0")
_LIB_PATH = pathlib.Path(__file__).resolve().with_name(
    "libnbl_b200_checked.so" if CHECKED else "libnbl_b200.so")

QUANTITY_FIRST = 1
QUANTITY_SECOND = 2
QUANTITY_DISTVEC = 4
QUANTITY_ABSDIST = 8
QUANTITY_SHIFT = 16
_QBITS = {"i": QUANTITY_FIRST, "j": QUANTITY_SECOND, "D": QUANTITY_DISTVEC,
          "d": QUANTITY_ABSDIST, "S": QUANTITY_SHIFT}

GRID_AUTO, GRID_DENSE, GRID_MORTON, GRID_HASHED = 0, 1, 2, 3
PRECISION_FP32_FILTER, PRECISION_FP64 = 0, 1

(NBL_SUCCESS, NBL_ERROR_INVALID_ARGUMENT, NBL_ERROR_ZERO_VOLUME, NBL_ERROR_RANGE,
 NBL_ERROR_OUT_OF_MEMORY, NBL_ERROR_CUDA, NBL_ERROR_CAPACITY, NBL_ERROR_NO_DEVICE,
 NBL_ERROR_INTERNAL) = range(9)


class Request(ctypes.Structure):
    """``nbl_request`` (include/nbl_b200.h)."""
    _fields_ = [("quantities", ctypes.c_int),
                ("cell_origin", ctypes.c_void_p),
                ("cell", ctypes.c_void_p),
                ("inv_cell", ctypes.c_void_p),
                ("pbc", ctypes.c_void_p),
                ("nat", ctypes.c_int64),
                ("positions", ctypes.c_void_p),
                ("positions_on_device", ctypes.c_int),
                ("cutoff", ctypes.c_double),
                ("per_atom_cutoff", ctypes.c_void_p),
                ("per_type_cutoff_sq", ctypes.c_void_p),
                ("ncutoffs", ctypes.c_int32),
                ("types", ctypes.c_void_p),
                ("aux_on_device", ctypes.c_int),
                ("grid", ctypes.c_int),
                ("precision", ctypes.c_int),
                ("device_id", ctypes.c_int)]


class Outputs(ctypes.Structure):
    """``nbl_outputs`` (include/nbl_b200.h)."""
    _fields_ = [("first", ctypes.c_void_p),
                ("second", ctypes.c_void_p),
                ("distvec", ctypes.c_void_p),
                ("absdist", ctypes.c_void_p),
                ("shift", ctypes.c_void_p)]


class LaunchConfig(ctypes.Structure):
    """``nbl_launch_config`` (include/nbl_b200.h): the pair passes' launch
    configuration (zero fields: defaults)."""
    _fields_ = [(n, ctypes.c_int) for n in (
        "count_ctas_per_sm", "fill_ctas_per_sm", "count_strided", "fill_strided",
        "count_warps", "fill_warps", "count_group", "count_large_staging",
        "atoms_per_item", "cells_per_item", "one_launch_atoms", "thread_per_atom")]

    def as_dict(self):
        return {n: int(getattr(self, n)) for n, _ in self._fields_}


def _load():
    if not _LIB_PATH.exists():
        raise ImportError(
            f"{_LIB_PATH.name} is not built; run "
            "`python matscipy-neighbours_b200/build.py"
            f"{' --checked' if CHECKED else ''}` (needs nvcc)")
    lib = ctypes.CDLL(str(_LIB_PATH))
    P = ctypes.c_void_p
    sigs = {
        "nbl_plan_create": ([ctypes.c_int, ctypes.POINTER(P)], ctypes.c_int),
        "nbl_plan_destroy": ([P], ctypes.c_int),
        "nbl_plan_trim": ([P], ctypes.c_int),
        "nbl_set_atom_range": ([P, ctypes.c_int64, ctypes.c_int64], ctypes.c_int),
        "nbl_plan_set_launch": ([P, ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "nbl_plan_set_launch_config": ([P, ctypes.POINTER(LaunchConfig)], ctypes.c_int),
        "nbl_plan_get_launch_config": ([P, ctypes.POINTER(LaunchConfig)], ctypes.c_int),
        "nbl_debug_inject": ([ctypes.c_int, ctypes.c_int64], ctypes.c_int),
        "nbl_count": ([P, ctypes.POINTER(Request), P, ctypes.POINTER(ctypes.c_int64)],
                      ctypes.c_int),
        "nbl_fill": ([P, ctypes.POINTER(Outputs), P], ctypes.c_int),
        "nbl_fill_host": ([P, ctypes.POINTER(Outputs), P], ctypes.c_int),
        "nbl_check": ([P, P], ctypes.c_int),
        "nbl_counts": ([P, P, P], ctypes.c_int),
        "nbl_row_offsets": ([P, P, P], ctypes.c_int),
        "nbl_fill_matrix": ([P, ctypes.c_int32, P, P, P, ctypes.POINTER(ctypes.c_int), P],
                            ctypes.c_int),
        "nbl_last_error": ([], ctypes.c_char_p),
        "nbl_has_gpu": ([], ctypes.c_int),
        "nbl_device_type": ([], ctypes.c_int),
        "nbl_version": ([], ctypes.c_char_p),
        "nbl_launch_count": ([ctypes.c_int], ctypes.c_longlong),
        "nbl_first_neighbours": ([ctypes.c_int64, ctypes.c_int64, P, P, P], ctypes.c_int),
        "nbl_lj_forces": ([P, ctypes.POINTER(Request), ctypes.c_double, ctypes.c_double, P, P,
                           P], ctypes.c_int),
        "nbl_triplet_list": ([ctypes.c_int64, P, P, ctypes.c_double, P, P, ctypes.c_int64,
                              ctypes.POINTER(ctypes.c_int64), P], ctypes.c_int),
    }
    for name, (args, res) in sigs.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return lib


lib = _load()

_has_gpu = int(lib.nbl_has_gpu())
_device_type = int(lib.nbl_device_type())


class EngineError(RuntimeError):
    pass


def check(status):
    """Raise the Python exception matching an nbl_status."""
    if status == NBL_SUCCESS:
        return
    msg = lib.nbl_last_error().decode(errors="replace")
    if status == NBL_ERROR_OUT_OF_MEMORY:
        raise MemoryError(msg)
    if status == NBL_ERROR_INVALID_ARGUMENT:
        raise ValueError(msg)
    raise RuntimeError(msg)


# ---------------------------------------------------------------------------
# options (not part of the reference's interface; defaults reproduce it)
# ---------------------------------------------------------------------------
_options = {"precision": PRECISION_FP32_FILTER, "grid": GRID_AUTO}


def set_options(precision=None, grid=None):
    """Set the engine's candidate precision ("fp32" filter with FP64 recheck,
    or "fp64") and cell-grid layout ("auto", "dense", "morton", "hashed").
    Every combination returns the same pairs; returns the previous options."""
    prev = dict(_options)
    if precision is not None:
        _options["precision"] = {"fp32": PRECISION_FP32_FILTER,
                                 "fp64": PRECISION_FP64}.get(precision, precision)
    if grid is not None:
        _options["grid"] = {"auto": GRID_AUTO, "dense": GRID_DENSE,
                            "morton": GRID_MORTON, "hashed": GRID_HASHED}.get(grid, grid)
    return prev


# ---------------------------------------------------------------------------
# plans (one per host thread and device)
# ---------------------------------------------------------------------------
_tls = threading.local()


def plan_for(device_id):
    plans = getattr(_tls, "plans", None)
    if plans is None:
        plans = _tls.plans = {}
    p = plans.get(device_id)
    if p is None:
        if not _has_gpu:
            raise RuntimeError("no CUDA device: the neighbour-list engine runs on "
                               "the GPU only")
        h = ctypes.c_void_p()
        check(lib.nbl_plan_create(int(device_id), ctypes.byref(h)))
        p = plans[device_id] = h
    return p


# ---------------------------------------------------------------------------
# argument handling (bind_py_neighbours.cc:97-195)
# ---------------------------------------------------------------------------

def _fromany(obj, dtype, nmin, nmax):
    a = np.asarray(obj, dtype=dtype)
    if a.ndim < nmin:
        raise ValueError("object of too small depth for desired array")
    if a.ndim > nmax:
        raise ValueError("object too deep for desired array")
    return np.ascontiguousarray(a)


def coerce_geometry(cell_origin, cell, inv_cell, pbc):
    origin = _fromany(cell_origin, np.float64, 1, 1)
    cell = _fromany(cell, np.float64, 2, 2)
    inv = _fromany(inv_cell, np.float64, 2, 2)
    pbc = _fromany(pbc, np.bool_, 1, 1)
    if origin.shape != (3,) or cell.shape != (3, 3) or inv.shape != (3, 3) or \
            pbc.shape != (3,):
        raise ValueError("cell_origin, cell, inv_cell and pbc must have shapes "
                         "(3,), (3, 3), (3, 3) and (3,)")
    return origin, cell, inv, np.ascontiguousarray(pbc.astype(np.uint8))


def resolve_cutoff(py_cut, nat):
    """bind_py_neighbours.cc:128-173.  Returns (cutoff, per_atom,
    per_type_sq, ncutoffs): a Python float is the global cutoff; a 1-D array
    holds per-atom radii (binning cutoff = max 2r); a square 2-D array holds
    per-type cutoffs (squared here; binning cutoff = max entry)."""
    if isinstance(py_cut, float):
        return float(py_cut), None, None, 0
    a = _fromany(py_cut, np.float64, 1, 2)
    cutoff = 0.0
    if a.ndim == 1:
        if a.shape[0] != nat:
            raise TypeError("One-dimensional cutoff array must have length that "
                            "corresponds to position array.")
        # std::max(cutoff, 2 r) from 0 (NaN entries never win)
        cutoff = float(np.fmax.reduce(2.0 * a, initial=0.0))
        return cutoff, a, None, 0
    if a.shape[1] != a.shape[0]:
        raise TypeError("Two-dimensional cutoff array must be square.")
    cutoff = float(np.fmax.reduce(a.ravel(), initial=0.0))
    return cutoff, None, np.ascontiguousarray(a * a), int(a.shape[0])


def quantity_flags(quantities):
    try:
        q = quantities.encode("ascii")
    except UnicodeEncodeError:
        raise TypeError("Conversion to ASCII string failed.") from None
    flags = 0
    for ch in q.decode():
        if ch not in _QBITS:
            raise ValueError("Unsupported quantity specified.")
        flags |= _QBITS[ch]
    return flags


def _ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def make_request(flags, origin, cell, inv, pbc, nat, pos_ptr, on_device, cutoff,
                 per_atom, per_type_sq, ncutoffs, types, device_id=-1,
                 aux_on_device=False):
    r = Request()
    r.quantities = flags
    r.cell_origin = origin.ctypes.data
    r.cell = cell.ctypes.data
    r.inv_cell = inv.ctypes.data
    r.pbc = pbc.ctypes.data
    r.nat = int(nat)
    r.positions = pos_ptr
    r.positions_on_device = 1 if on_device else 0
    r.cutoff = float(cutoff)
    if aux_on_device:
        r.per_atom_cutoff = per_atom
        r.types = types
    else:
        r.per_atom_cutoff = None if per_atom is None else per_atom.ctypes.data
        r.types = None if types is None else types.ctypes.data
    r.per_type_cutoff_sq = None if per_type_sq is None else per_type_sq.ctypes.data
    r.ncutoffs = int(ncutoffs)
    r.aux_on_device = 1 if aux_on_device else 0
    r.grid = int(_options["grid"])
    r.precision = int(_options["precision"])
    r.device_id = int(device_id)
    return r


# ---------------------------------------------------------------------------
# host buffers
# ---------------------------------------------------------------------------

def _torch():
    import torch
    return torch


def host_empty(shape, dtype):
    """A host array for device->host copies: page-locked when torch can
    provide it (faster copies), plain numpy memory otherwise."""
    try:
        torch = _torch()
        tdt = {np.dtype(np.int32): torch.int32,
               np.dtype(np.float64): torch.float64}[np.dtype(dtype)]
        return torch.empty(shape, dtype=tdt, pin_memory=True).numpy()
    except Exception:
        return np.empty(shape, dtype=dtype)


_SHAPES = {"i": ((), np.int32), "j": ((), np.int32), "D": ((3,), np.float64),
           "d": ((), np.float64), "S": ((3,), np.int32)}


# Below this many output bytes nbl_fill_host lands the whole list in the
# plan's own pinned buffer with one copy and copies it on into the caller's
# arrays, so plain numpy arrays are as fast as page-locked ones (and cheaper
# to allocate).
_ONE_COPY_BYTES = 256 << 10


_PAIR_BYTES = {"i": 4, "j": 4, "D": 24, "d": 8, "S": 12}


def _host_outputs(quantities, npairs):
    kinds = set(quantities)
    total = npairs * sum(_PAIR_BYTES[ch] for ch in kinds)
    alloc = np.empty if total <= _ONE_COPY_BYTES else host_empty
    bufs = {}
    for ch in kinds:
        extra, dt = _SHAPES[ch]
        bufs[ch] = alloc((npairs,) + extra, dt)
    return bufs


def _outputs_struct(bufs, ptr_of):
    o = Outputs()
    o.first = ptr_of(bufs["i"]) if "i" in bufs else None
    o.second = ptr_of(bufs["j"]) if "j" in bufs else None
    o.distvec = ptr_of(bufs["D"]) if "D" in bufs else None
    o.absdist = ptr_of(bufs["d"]) if "d" in bufs else None
    o.shift = ptr_of(bufs["S"]) if "S" in bufs else None
    return o


def _ordered(quantities, bufs):
    seen = set()
    out = []
    for ch in quantities:
        a = bufs[ch]
        out.append(a.copy() if ch in seen else a)
        seen.add(ch)
    return out


# ---------------------------------------------------------------------------
# engine calls
# ---------------------------------------------------------------------------

def _parse(quantities, cell_origin, cell, inv_cell, pbc, positions, cutoffs, types):
    if not isinstance(quantities, str):
        raise TypeError("argument 1 must be str")
    origin, cell, inv, pbc8 = coerce_geometry(cell_origin, cell, inv_cell, pbc)
    ty = None
    if types is not None:
        ty = _fromany(types, np.int32, 1, 1)
    return origin, cell, inv, pbc8, ty


def run_host(quantities, origin, cell, inv, pbc8, pos, rc, per_atom, per_type_sq,
             ncut, types, flags, device_id=0):
    """Host positions in, host arrays out (the reference's
    neighbour_list_gpu(), neighbour_list_gpu.hh:28-34)."""
    nat = pos.shape[0]
    plan = plan_for(device_id)
    req = make_request(flags, origin, cell, inv, pbc8, nat,
                       ctypes.c_void_p(pos.ctypes.data) if nat else None, False, rc,
                       per_atom, per_type_sq, ncut, types, device_id)
    npairs = ctypes.c_int64()
    check(lib.nbl_count(plan, ctypes.byref(req), None, ctypes.byref(npairs)))
    n = int(npairs.value)
    bufs = _host_outputs(quantities, n)
    if n:
        o = _outputs_struct(bufs, lambda a: a.ctypes.data)
        check(lib.nbl_fill_host(plan, ctypes.byref(o), None))
    return bufs


def neighbour_list(quantities, cell_origin, cell, inv_cell, pbc, positions, cutoffs,
                   types=None):
    """Host entry of the reference's extension (bind_py_neighbours.cc:88):
    numpy in, numpy out, one array per quantity character (a bare array for a
    single character)."""
    origin, cell, inv, pbc8, ty = _parse(quantities, cell_origin, cell, inv_cell, pbc,
                                         positions, cutoffs, types)
    pos = _fromany(positions, np.float64, 2, 2)
    nat = pos.shape[0]
    if pos.ndim == 2 and nat and pos.shape[1] != 3:
        raise ValueError("positions must have shape (n, 3)")
    if ty is not None and ty.shape[0] != nat:
        raise TypeError("Position and type arrays must have identical first "
                        "dimension.")
    rc, per_atom, per_type_sq, ncut = resolve_cutoff(cutoffs, nat)
    flags = quantity_flags(quantities)
    bufs = run_host(quantities, origin, cell, inv, pbc8, pos, rc, per_atom,
                    per_type_sq, ncut, ty, flags)
    out = _ordered(quantities, bufs)
    return out[0] if len(quantities) == 1 else tuple(out)


def import_device_positions(py_in):
    """bind_py_dlpack.cc:133-175: a C-contiguous float64 (n, 3) device array
    through its __dlpack__ (torch, cupy, ...).  Returns a torch tensor viewing
    the same memory."""
    torch = _torch()
    if isinstance(py_in, torch.Tensor):
        t = py_in
    else:
        t = torch.from_dlpack(py_in)
    if t.dtype != torch.float64 or t.dim() != 2 or t.shape[1] != 3 or \
            not t.is_contiguous() or not t.is_cuda:
        raise TypeError("device positions must be a C-contiguous float64 array "
                        "of shape (n, 3)")
    return t


def run_device(quantities, origin, cell, inv, pbc8, pos_t, host_pos, rc, per_atom,
               per_type_sq, ncut, types, flags, device_id, atom_range=None):
    """Device (or host-uploaded) positions in, torch CUDA tensors out on the
    device's current stream (neighbour_list_gpu_device,
    neighbour_list_gpu.hh:95-96).  atom_range=(lo, hi) keeps only the rows
    lo <= i < hi: the slice of the full list that those rows occupy."""
    torch = _torch()
    dev = torch.device("cuda", device_id)
    stream = torch.cuda.current_stream(dev)
    plan = plan_for(device_id)
    if pos_t is not None:
        nat = pos_t.shape[0]
        ptr = ctypes.c_void_p(pos_t.data_ptr()) if nat else None
        on_dev = True
    else:
        nat = host_pos.shape[0]
        ptr = ctypes.c_void_p(host_pos.ctypes.data) if nat else None
        on_dev = False
    req = make_request(flags, origin, cell, inv, pbc8, nat, ptr, on_dev, rc, per_atom,
                       per_type_sq, ncut, types, device_id)
    npairs = ctypes.c_int64()
    ctx = torch.cuda.device(dev) if torch.cuda.current_device() != device_id else _NO_CONTEXT
    with ctx:
        if atom_range is not None:
            check(lib.nbl_set_atom_range(plan, int(atom_range[0]), int(atom_range[1])))
        try:
            check(lib.nbl_count(plan, ctypes.byref(req),
                                ctypes.c_void_p(stream.cuda_stream), ctypes.byref(npairs)))
        finally:
            if atom_range is not None:
                # The range applies to the count just made (and its fill);
                # later calls on this thread's plan build full lists again.
                lib.nbl_set_atom_range(plan, 0, -1)
        n = int(npairs.value)
        bufs = _device_outputs(torch, quantities, n, dev)
        if n:
            o = _outputs_struct(bufs, lambda t: t.data_ptr())
            check(lib.nbl_fill(plan, ctypes.byref(o), ctypes.c_void_p(stream.cuda_stream)))
    return bufs


class _NoContext:
    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


_NO_CONTEXT = _NoContext()


def _device_outputs(torch, quantities, n, dev):
    """The requested outputs as views of one device allocation (each starting
    on a 256-byte boundary): one allocator call instead of one per quantity.
    The views keep the allocation alive together."""
    chars = [ch for ch in "ijDdS" if ch in quantities]
    offs, total = {}, 0
    for ch in chars:
        extra, dt = _SHAPES[ch]
        offs[ch] = total
        total += (n * (3 if extra else 1) * np.dtype(dt).itemsize + 255) & ~255
    raw = torch.empty(max(total, 1), dtype=torch.uint8, device=dev)
    bufs = {}
    for ch in chars:
        extra, dt = _SHAPES[ch]
        tdt = torch.int32 if dt == np.int32 else torch.float64
        nbytes = n * (3 if extra else 1) * np.dtype(dt).itemsize
        bufs[ch] = raw[offs[ch]:offs[ch] + nbytes].view(tdt).view((n,) + extra)
    return bufs


def neighbour_list_dlpack(quantities, cell_origin, cell, inv_cell, pbc, host_pos,
                          cutoffs, types=None, backend=0, py_in=None, device_id=-1):
    """DLPack entry of the reference's extension (bind_py_dlpack.cc:231): a
    tuple of "dltensor" capsules, one per quantity character.  backend 0
    returns host capsules (the pairs are still computed on the GPU), backend 1
    device capsules; `py_in` (anything with __dlpack__) supplies device
    positions in place of `host_pos`."""
    origin, cell, inv, pbc8, ty = _parse(quantities, cell_origin, cell, inv_cell, pbc,
                                         host_pos, cutoffs, types)
    hpos = _fromany(host_pos, np.float64, 2, 2)
    device_in = py_in is not None
    pos_t = import_device_positions(py_in) if device_in else None
    nat = pos_t.shape[0] if device_in else hpos.shape[0]
    if ty is not None and ty.shape[0] != nat:
        raise TypeError("Position and type arrays must have identical first "
                        "dimension.")
    rc, per_atom, per_type_sq, ncut = resolve_cutoff(cutoffs, nat)
    flags = quantity_flags(quantities)
    if backend == 0 and not device_in:
        bufs = run_host(quantities, origin, cell, inv, pbc8, hpos, rc, per_atom,
                        per_type_sq, ncut, ty, flags, max(device_id, 0))
        return tuple(a.__dlpack__() for a in _ordered(quantities, bufs))
    dev_id = pos_t.device.index if device_in else max(device_id, 0)
    bufs = run_device(quantities, origin, cell, inv, pbc8, pos_t, hpos, rc, per_atom,
                      per_type_sq, ncut, ty, flags, dev_id)
    out = []
    seen = set()
    for ch in quantities:
        t = bufs[ch]
        out.append((t.clone() if ch in seen else t).__dlpack__())
        seen.add(ch)
    return tuple(out)


def coordination(cell_origin, cell, inv_cell, pbc, positions, cutoffs, types=None,
                 device_id=0, py_in=None):
    """Per-atom neighbour counts without materialising the pairs (the count
    pass only; bind_py_dlpack.cc:410 coordination_dlpack).  Returns a torch
    int32 CUDA tensor."""
    torch = _torch()
    origin, cell, inv, pbc8, ty = _parse("i", cell_origin, cell, inv_cell, pbc,
                                         positions, cutoffs, types)
    device_in = py_in is not None
    pos_t = import_device_positions(py_in) if device_in else None
    hpos = None if device_in else _fromany(positions, np.float64, 2, 2)
    nat = pos_t.shape[0] if device_in else hpos.shape[0]
    rc, per_atom, per_type_sq, ncut = resolve_cutoff(cutoffs, nat)
    dev_id = pos_t.device.index if device_in else max(device_id, 0)
    dev = torch.device("cuda", dev_id)
    stream = torch.cuda.current_stream(dev)
    plan = plan_for(dev_id)
    ptr = (ctypes.c_void_p(pos_t.data_ptr()) if device_in else
           ctypes.c_void_p(hpos.ctypes.data)) if nat else None
    req = make_request(QUANTITY_FIRST, origin, cell, inv, pbc8, nat, ptr, device_in, rc,
                       per_atom, per_type_sq, ncut, ty, dev_id)
    npairs = ctypes.c_int64()
    with torch.cuda.device(dev):
        check(lib.nbl_count(plan, ctypes.byref(req), ctypes.c_void_p(stream.cuda_stream),
                            ctypes.byref(npairs)))
        counts = torch.empty((nat,), dtype=torch.int32, device=dev)
        if nat:
            check(lib.nbl_counts(plan, ctypes.c_void_p(counts.data_ptr()),
                                 ctypes.c_void_p(stream.cuda_stream)))
    return counts


def neighbour_matrix_dlpack(cell_origin, cell, inv_cell, pbc, host_pos, cutoffs,
                            max_neighbours, types=None, backend=0, py_in=None,
                            device_id=-1):
    """Dense (n x K) neighbour matrix (bind_py_dlpack.cc:500-658
    neighbour_matrix_dlpack): returns (idx, dist, count) capsules and the
    overflow flag.  Rows hold each atom's neighbours in the reference's row
    order, filled straight from the fill pass (no pair list in between)."""
    torch = _torch()
    origin, cell, inv, pbc8, ty = _parse("", cell_origin, cell, inv_cell, pbc,
                                         host_pos, cutoffs, types)
    K = int(max_neighbours)
    if K <= 0:
        raise ValueError("max_neighbours must be positive")
    device_in = py_in is not None
    pos_t = import_device_positions(py_in) if device_in else None
    hpos = _fromany(host_pos, np.float64, 2, 2)
    nat = pos_t.shape[0] if device_in else hpos.shape[0]
    if ty is not None and ty.shape[0] != nat:
        raise TypeError("Position and type arrays must have identical first "
                        "dimension.")
    rc, per_atom, per_type_sq, ncut = resolve_cutoff(cutoffs, nat)
    dev_id = pos_t.device.index if device_in else max(device_id, 0)
    dev = torch.device("cuda", dev_id)
    stream = torch.cuda.current_stream(dev)
    plan = plan_for(dev_id)
    ptr = (ctypes.c_void_p(pos_t.data_ptr()) if device_in else
           ctypes.c_void_p(hpos.ctypes.data)) if nat else None
    req = make_request(0, origin, cell, inv, pbc8, nat, ptr, device_in, rc, per_atom,
                       per_type_sq, ncut, ty, dev_id)
    npairs = ctypes.c_int64()
    overflow = ctypes.c_int(0)
    with torch.cuda.device(dev):
        check(lib.nbl_count(plan, ctypes.byref(req), ctypes.c_void_p(stream.cuda_stream),
                            ctypes.byref(npairs)))
        idx = torch.zeros((nat, K), dtype=torch.int32, device=dev)
        dist = torch.zeros((nat, K, 3), dtype=torch.float64, device=dev)
        count = torch.zeros((nat,), dtype=torch.int32, device=dev)
        if nat:
            check(lib.nbl_fill_matrix(plan, K, ctypes.c_void_p(idx.data_ptr()),
                                      ctypes.c_void_p(dist.data_ptr()),
                                      ctypes.c_void_p(count.data_ptr()),
                                      ctypes.byref(overflow),
                                      ctypes.c_void_p(stream.cuda_stream)))
    outs = (idx, dist, count)
    if backend == 0 and not device_in:
        outs = tuple(t.cpu().numpy() for t in outs)
    return tuple(t.__dlpack__() for t in outs) + (bool(overflow.value),)


# ---------------------------------------------------------------------------
# post-processing helpers with the reference extension's names
# (first_neighbours.cc:15-57, triplet_list.cc:15-34); host numpy code, outside
# the GPU hot path.
# ---------------------------------------------------------------------------

def _device_array(x, dtype):
    """A torch CUDA tensor of `dtype` viewing (or, for another dtype, copying)
    a device array `x` (torch tensor or anything with a CUDA __dlpack__);
    None for host arrays."""
    dev = getattr(x, "__dlpack_device__", None)
    if dev is None:
        return None
    try:
        if int(dev()[0]) == 1:  # kDLCPU
            return None
    except Exception:
        return None
    torch = _torch()
    t = x if isinstance(x, torch.Tensor) else torch.from_dlpack(x)
    if not t.is_cuda:
        return None
    return t.to(dtype).contiguous()


def first_neighbours(n, i):
    """seed[k] = index of the first pair of atom k in the i-sorted list,
    seed[n] = len(i); -1 for atoms before the first one with pairs.  A device
    `i` (torch CUDA tensor or CUDA __dlpack__) is handled on its GPU and
    gives a torch CUDA tensor."""
    n = int(n)
    it = _device_array(i, _torch().int32) if hasattr(i, "__dlpack_device__") else None
    if it is not None:
        torch = _torch()
        if it.dim() != 1:
            raise ValueError("object too deep for desired array")
        seed = torch.empty(n + 1, dtype=torch.int32, device=it.device)
        stream = torch.cuda.current_stream(it.device)
        with torch.cuda.device(it.device):
            check(lib.nbl_first_neighbours(n, int(it.shape[0]),
                                           ctypes.c_void_p(it.data_ptr()) if it.numel() else None,
                                           ctypes.c_void_p(seed.data_ptr()),
                                           ctypes.c_void_p(stream.cuda_stream)))
        return seed
    i = _fromany(i, np.int32, 1, 1)
    nn = i.shape[0]
    if nn == 0:
        return np.zeros(n + 1, dtype=np.int32)
    seed = np.full(n + 1, -1, dtype=np.int32)
    first = int(i[0])
    starts = np.searchsorted(i, np.arange(n + 1), side="left").astype(np.int32)
    seed[first:] = starts[first:]
    seed[int(i[-1]) + 1:] = nn
    return seed


def get_jump_indicies(sorted_array):
    """Indices where a sorted array changes value, with both ends."""
    s = _fromany(sorted_array, np.int32, 1, 1)
    n = int(np.count_nonzero(s[1:] != s[:-1])) + 1 if s.shape[0] > 0 else 1
    return first_neighbours(n, s)


def triplet_list(first_i, absdist=None, cutoff=None):
    """(ij, ik) pair-index triplets sharing a first atom, ij != ik, ij-major;
    with distances, both below `cutoff`."""
    ft = (_device_array(first_i, _torch().int32)
          if hasattr(first_i, "__dlpack_device__") else None)
    if ft is not None:
        return _triplet_list_device(ft, absdist, cutoff)
    fn = _fromany(first_i, np.int32, 1, 1)
    if absdist is not None and cutoff is None:
        raise TypeError("triplet_list: distances given without a cutoff")
    d = None if absdist is None else _fromany(absdist, np.float64, 1, 1)
    ij_all, ik_all = [], []
    for r in range(fn.shape[0] - 1):
        b, e = int(fn[r]), int(fn[r + 1])
        if e - b < 2:
            continue
        idx = np.arange(b, e, dtype=np.int32)
        ij = np.repeat(idx, e - b)
        ik = np.tile(idx, e - b)
        keep = ij != ik
        if d is not None:
            keep &= (d[ij] < cutoff) & (d[ik] < cutoff)
        ij_all.append(ij[keep])
        ik_all.append(ik[keep])
    if not ij_all:
        return np.zeros(0, dtype=np.int32), np.zeros(0, dtype=np.int32)
    return np.concatenate(ij_all), np.concatenate(ik_all)


def _triplet_list_device(ft, absdist, cutoff):
    """triplet_list on the GPU of `ft` (nbl_triplet_list): torch CUDA tensors."""
    torch = _torch()
    if absdist is not None and cutoff is None:
        raise TypeError("triplet_list: distances given without a cutoff")
    dt = None
    if absdist is not None:
        dt = _device_array(absdist, torch.float64) if hasattr(absdist, "__dlpack_device__") \
            else None
        if dt is None:
            dt = torch.as_tensor(np.ascontiguousarray(absdist, dtype=np.float64),
                                 device=ft.device)
    stream = torch.cuda.current_stream(ft.device)
    sp = ctypes.c_void_p(stream.cuda_stream)
    fp = ctypes.c_void_p(ft.data_ptr()) if ft.numel() else None
    dp = ctypes.c_void_p(dt.data_ptr()) if dt is not None and dt.numel() else None
    c = float(cutoff) if cutoff is not None else 0.0
    n = ctypes.c_int64()
    with torch.cuda.device(ft.device):
        check(lib.nbl_triplet_list(int(ft.shape[0]), fp, dp, c, None, None, 0,
                                   ctypes.byref(n), sp))
        ij = torch.empty(int(n.value), dtype=torch.int32, device=ft.device)
        ik = torch.empty(int(n.value), dtype=torch.int32, device=ft.device)
        if n.value:
            check(lib.nbl_triplet_list(int(ft.shape[0]), fp, dp, c,
                                       ctypes.c_void_p(ij.data_ptr()),
                                       ctypes.c_void_p(ik.data_ptr()), int(n.value),
                                       ctypes.byref(n), sp))
    return ij, ik
