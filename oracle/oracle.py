"""TEST INFRASTRUCTURE ONLY: Python access to the CPU parity oracle.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module, and only as the checker.

Three independent CPU implementations of the matscipy-neighbours pair list:

``oracle_neighbour_list``
    The plain-C restatement in ``nbl_oracle.c`` (built by ``oracle/Makefile``
    into ``liboracle.so``).
``ref_neighbour_list``
    The reference's own C++ core (``src/libneighbours/neighbour_list.cc:99``)
    compiled from its sources into ``oracle/_ref/libref_neighbours.so`` by
    ``make -C oracle ref``; absent where the reference sources are absent.
``brute_force_pairs``
    An O(N^2) explicit-image numpy enumeration, the same idea as the
    reference's test helper (``tests/test_extension.py:50-92``).

The argument conventions are those of the reference's C-extension
``_matscipy_neighbours.neighbour_list(quantities, cell_origin, cell, inv_cell,
pbc, positions, cutoff[, types])`` (``bind_py_neighbours.cc:88-268``): the
cutoff is a float, a per-atom radius array (pair cutoff = sum; binning cutoff
= max 2r) or a square per-type matrix (squared before the core sees it;
binning cutoff = max entry).
"""

import ctypes
import os
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libref_neighbours.so"
REF_GPU_SO = HERE / "_ref" / "libref_gpu.so"

_QBITS = {"i": 1, "j": 2, "D": 4, "d": 8, "S": 16}


class _OracleResult(ctypes.Structure):
    _fields_ = [("npairs", ctypes.c_int64),
                ("i", ctypes.POINTER(ctypes.c_int32)),
                ("j", ctypes.POINTER(ctypes.c_int32)),
                ("D", ctypes.POINTER(ctypes.c_double)),
                ("d", ctypes.POINTER(ctypes.c_double)),
                ("S", ctypes.POINTER(ctypes.c_int32)),
                ("counts", ctypes.POINTER(ctypes.c_int64))]


class _RefResult(ctypes.Structure):
    _fields_ = [("npairs", ctypes.c_int64),
                ("i", ctypes.POINTER(ctypes.c_int32)),
                ("j", ctypes.POINTER(ctypes.c_int32)),
                ("D", ctypes.POINTER(ctypes.c_double)),
                ("d", ctypes.POINTER(ctypes.c_double)),
                ("S", ctypes.POINTER(ctypes.c_int32))]


class OracleError(RuntimeError):
    pass


_lib = None
_ref = None


def reference_src():
    """The reference's src/libneighbours directory: NBL_REFERENCE_SRC, else that
    of a checkout of the reference beside this repository (../reference)."""
    return pathlib.Path(os.environ.get(
        "NBL_REFERENCE_SRC", HERE.parent.parent / "reference" / "src" / "libneighbours"))


def build():
    """Compile the C restatement (and the reference core when its sources are
    present).  Cheap and idempotent."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    src = reference_src()
    if src.is_dir():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF_SRC={src}"], check=True)
        subprocess.run(["make", "-s", "-C", str(HERE), "ref_gpu", f"REF_SRC={src}"],
                       check=True)


def _load():
    global _lib
    if _lib is None:
        if not ORACLE_SO.exists():
            build()
        lib = ctypes.CDLL(str(ORACLE_SO))
        lib.oracle_neighbour_list.restype = ctypes.c_int
        lib.oracle_result_free.argtypes = [ctypes.POINTER(_OracleResult)]
        P = ctypes.c_void_p
        lib.oracle_first_neighbours.argtypes = [ctypes.c_int32, ctypes.c_int64, P, P]
        lib.oracle_first_neighbours.restype = None
        lib.oracle_triplet_list.argtypes = [ctypes.c_int32, P, P, ctypes.c_double, P, P,
                                            ctypes.c_int64]
        lib.oracle_triplet_list.restype = ctypes.c_int64
        _lib = lib
    return _lib


def ref_available():
    return REF_SO.exists()


def _load_ref():
    global _ref
    if _ref is None:
        if not REF_SO.exists():
            raise OracleError("reference core not built (make -C oracle ref)")
        lib = ctypes.CDLL(str(REF_SO))
        lib.ref_neighbour_list.restype = ctypes.c_int
        lib.ref_result_free.argtypes = [ctypes.POINTER(_RefResult)]
        lib.ref_set_threads.restype = ctypes.c_int
        lib.ref_set_threads.argtypes = [ctypes.c_int]
        lib.ref_last_error.restype = ctypes.c_char_p
        P = ctypes.c_void_p
        lib.ref_first_neighbours.argtypes = [ctypes.c_int, ctypes.c_int, P, P]
        lib.ref_first_neighbours.restype = None
        lib.ref_triplet_list.argtypes = [ctypes.c_int, P, P, ctypes.c_double, P, P,
                                         ctypes.c_int64]
        lib.ref_triplet_list.restype = ctypes.c_int64
        _ref = lib
    return _ref


def ref_set_threads(n):
    """Set the reference core's OpenMP thread count; returns the count used."""
    return _load_ref().ref_set_threads(int(n))


def _dptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def resolve_cutoff(cutoff, nat):
    """bind_py_neighbours.cc:136-173: returns (binning cutoff, per_atom,
    per_type_sq, ncutoffs)."""
    if isinstance(cutoff, float):
        return float(cutoff), None, None, 0
    a = np.ascontiguousarray(cutoff, dtype=np.float64)
    if a.ndim == 0:
        return float(a), None, None, 0
    if a.ndim == 1:
        if a.shape[0] != nat:
            raise TypeError("One-dimensional cutoff array must have length that "
                            "corresponds to position array.")
        rc = 0.0
        for v in a:
            rc = max(rc, 2 * float(v))
        return rc, a, None, 0
    if a.ndim != 2 or a.shape[0] != a.shape[1]:
        raise TypeError("Two-dimensional cutoff array must be square.")
    rc = 0.0
    for v in a.ravel():
        rc = max(rc, float(v))
    return rc, None, np.ascontiguousarray(a * a), a.shape[0]


def _args(cell, positions, pbc, origin, inv_cell=None):
    cell = np.ascontiguousarray(cell, dtype=np.float64).reshape(3, 3)
    pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
    origin = (np.zeros(3) if origin is None
              else np.ascontiguousarray(origin, dtype=np.float64))
    inv = (np.ascontiguousarray(np.linalg.inv(cell.T)) if inv_cell is None
           else np.ascontiguousarray(inv_cell, dtype=np.float64))
    pbc = np.ascontiguousarray(np.broadcast_to(pbc, (3,)), dtype=np.int32)
    return cell, pos, origin, inv, pbc


def _unpack(res, quantities, nat=None):
    n = int(res.npairs)
    out = {}

    def take(ptr, shape, dtype):
        if not ptr or n == 0:
            return np.zeros(shape, dtype=dtype)
        return np.ctypeslib.as_array(ptr, shape=shape).astype(dtype, copy=True)

    out["i"] = take(res.i, (n,), np.int32)
    out["j"] = take(res.j, (n,), np.int32)
    out["D"] = take(res.D, (n, 3), np.float64)
    out["d"] = take(res.d, (n,), np.float64)
    out["S"] = take(res.S, (n, 3), np.int32)
    vals = tuple(out[q] for q in quantities)
    return vals[0] if len(quantities) == 1 else vals


def _flags(quantities):
    f = 0
    for q in quantities:
        if q not in _QBITS:
            raise ValueError("Unsupported quantity specified.")
        f |= _QBITS[q]
    return f


def oracle_neighbour_list(quantities, cell, positions, cutoff, pbc=True,
                          types=None, origin=None, inv_cell=None):
    """The C restatement with reference-extension argument semantics."""
    lib = _load()
    cell, pos, origin, inv, pbc = _args(cell, positions, pbc, origin, inv_cell)
    nat = pos.shape[0]
    rc, pa, pt, nc = resolve_cutoff(cutoff, nat)
    ty = None if types is None else np.ascontiguousarray(types, dtype=np.int32)
    flags = _flags(quantities)
    res = _OracleResult()
    st = lib.oracle_neighbour_list(
        ctypes.c_int(flags), _dptr(origin), _dptr(cell), _dptr(inv), _dptr(pbc),
        ctypes.c_int32(nat), _dptr(pos), ctypes.c_double(rc), _dptr(pa),
        _dptr(pt), ctypes.c_int32(nc), _dptr(ty), ctypes.byref(res))
    try:
        if st == 1:
            raise OracleError("Zero cell volume.")
        if st == 2:
            raise OracleError("atom coordinate out of range")
        return _unpack(res, quantities)
    finally:
        lib.oracle_result_free(ctypes.byref(res))


def oracle_counts(cell, positions, cutoff, pbc=True, types=None, origin=None):
    """Per-atom neighbour counts from the C restatement (coordination)."""
    i = oracle_neighbour_list("i", cell, positions, cutoff, pbc, types, origin)
    return np.bincount(i, minlength=np.asarray(positions).reshape(-1, 3).shape[0])


def ref_neighbour_list(quantities, cell, positions, cutoff, pbc=True,
                       types=None, origin=None, morton=False, inv_cell=None):
    """The reference's own C++ core (oracle/_ref), same conventions."""
    lib = _load_ref()
    cell, pos, origin, inv, pbc = _args(cell, positions, pbc, origin, inv_cell)
    nat = pos.shape[0]
    rc, pa, pt, nc = resolve_cutoff(cutoff, nat)
    ty = None if types is None else np.ascontiguousarray(types, dtype=np.int32)
    flags = _flags(quantities)
    res = _RefResult()
    st = lib.ref_neighbour_list(
        ctypes.c_int(flags), _dptr(origin), _dptr(cell), _dptr(inv), _dptr(pbc),
        ctypes.c_int(nat), _dptr(pos), ctypes.c_double(rc), _dptr(pa),
        _dptr(pt), ctypes.c_int(nc), _dptr(ty), ctypes.c_int(1 if morton else 0),
        ctypes.byref(res))
    try:
        if st != 0:
            raise OracleError(lib.ref_last_error().decode())
        return _unpack(res, quantities)
    finally:
        lib.ref_result_free(ctypes.byref(res))


def brute_force_pairs(cell, positions, pbc, cutoff):
    """O(N^2) explicit-image enumeration of (i, j, S) with |D| < cutoff, for
    small cases.  Periodic atoms are first wrapped into the cell (as the
    binning does), so S is reported relative to the wrapped images and only the
    (i, j) multiset is comparable with the cell-list result."""
    cell = np.asarray(cell, dtype=np.float64)
    pos = np.asarray(positions, dtype=np.float64)
    pbc = np.broadcast_to(pbc, (3,))
    frac = pos @ np.linalg.inv(cell)
    for k in range(3):
        if pbc[k]:
            frac[:, k] -= np.floor(frac[:, k])
    pos = frac @ cell
    vol = abs(np.linalg.det(cell))
    rng = []
    for k in range(3):
        if pbc[k]:
            a, b = cell[(k + 1) % 3], cell[(k + 2) % 3]
            rng.append(int(np.ceil(cutoff / (vol / np.linalg.norm(np.cross(a, b))))))
        else:
            rng.append(0)
    shifts = np.array(np.meshgrid(*[np.arange(-r, r + 1) for r in rng],
                                  indexing="ij")).reshape(3, -1).T
    n = len(pos)
    pairs = []
    for s in shifts:
        off = s @ cell
        d = pos[None, :, :] + off[None, None, :] - pos[:, None, :]
        r = np.sqrt((d * d).sum(-1))
        mask = r < cutoff
        if not s.any():
            np.fill_diagonal(mask, False)
        ii, jj = np.nonzero(mask)
        pairs.extend(zip(ii.tolist(), jj.tolist()))
    return sorted(pairs)


def canonical(i, j, S):
    """Rows (i, j, S) sorted lexicographically: an order-free comparison key
    (the same idea as the reference's tests/test_dlpack.py:32-36)."""
    rows = np.column_stack([np.asarray(i), np.asarray(j), np.asarray(S)])
    rows = rows.astype(np.int64)
    return rows[np.lexsort(rows.T[::-1])]


# ---- CSR helpers -------------------------------------------------------------

def _csr_first(fn, n, i):
    i = np.ascontiguousarray(i, dtype=np.int32)
    seed = np.empty(int(n) + 1, dtype=np.int32)
    fn(int(n), int(i.shape[0]), i.ctypes.data if i.size else None, seed.ctypes.data)
    return seed


def _csr_triplets(fn, first_i, absdist, cutoff):
    f = np.ascontiguousarray(first_i, dtype=np.int32)
    d = None if absdist is None else np.ascontiguousarray(absdist, dtype=np.float64)
    dp = None if d is None else d.ctypes.data
    c = float(cutoff) if cutoff is not None else 0.0
    n = int(fn(int(f.shape[0]), f.ctypes.data, dp, c, None, None, 0))
    ij = np.empty(n, dtype=np.int32)
    ik = np.empty(n, dtype=np.int32)
    if n:
        fn(int(f.shape[0]), f.ctypes.data, dp, c, ij.ctypes.data, ik.ctypes.data, n)
    return ij, ik


def oracle_first_neighbours(n, i):
    """first_neighbours.cc:15-38 restated in C (nbl_oracle.c)."""
    return _csr_first(_load().oracle_first_neighbours, n, i)


def oracle_triplet_list(first_i, absdist=None, cutoff=None):
    """triplet_list.cc:15-34 restated in C (nbl_oracle.c)."""
    return _csr_triplets(_load().oracle_triplet_list, first_i, absdist, cutoff)


def ref_first_neighbours(n, i):
    """The reference's own first_neighbours (oracle/_ref)."""
    return _csr_first(_load_ref().ref_first_neighbours, n, i)


def ref_triplet_list(first_i, absdist=None, cutoff=None):
    """The reference's own triplet_list (oracle/_ref)."""
    return _csr_triplets(_load_ref().ref_triplet_list, first_i, absdist, cutoff)


# ---- the reference's CUDA backend (a timing comparator) ---------------------

def refgpu_available():
    return REF_GPU_SO.exists()


def refgpu_neighbour_list(quantities, cell, positions_ptr, nat, cutoff, pbc=True, origin=None,
                          outputs=None, capacity=0):
    """One build by the reference's own CUDA backend (oracle/_ref/libref_gpu.so,
    neighbour_list_gpu_device, src/libneighbours/neighbour_list_gpu.cc:518) of
    device positions at `positions_ptr` (an integer device address, `nat`
    atoms); scalar cutoff.  Returns (npairs, device milliseconds of the call).
    `outputs` (five integer device addresses, in "ijDdS" order, or None)
    receive the pairs when `capacity` holds them."""
    lib = ctypes.CDLL(str(REF_GPU_SO))
    fn = lib.refgpu_neighbour_list
    P = ctypes.c_void_p
    fn.argtypes = [ctypes.c_int, P, P, P, P, ctypes.c_int, P, ctypes.c_double,
                   ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_float),
                   P, P, P, P, P, ctypes.c_int64]
    fn.restype = ctypes.c_int
    cell = np.ascontiguousarray(cell, dtype=np.float64).reshape(3, 3)
    inv = np.ascontiguousarray(np.linalg.inv(cell.T))
    origin = (np.zeros(3) if origin is None
              else np.ascontiguousarray(origin, dtype=np.float64))
    pb = np.ascontiguousarray(np.broadcast_to(pbc, (3,)), dtype=np.int32)
    n = ctypes.c_int64()
    ms = ctypes.c_float()
    outs = outputs if outputs is not None else (None,) * 5
    st = fn(_flags(quantities), _dptr(origin), _dptr(cell), _dptr(inv), _dptr(pb), int(nat),
            ctypes.c_void_p(int(positions_ptr)), float(cutoff), ctypes.byref(n),
            ctypes.byref(ms), *[None if o is None else ctypes.c_void_p(int(o)) for o in outs],
            int(capacity))
    if st != 0:
        raise OracleError("reference GPU backend returned an error")
    return int(n.value), float(ms.value)
