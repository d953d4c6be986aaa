"""Pair lists reused across molecular-dynamics steps (a Verlet list).

``VerletList(cutoff, skin, cell, pbc)`` builds the list of one system with
cutoff + skin (the engine's ``neighbour_list``) and keeps it.  At each step,
``update(positions)`` measures the largest displacement since that build
(``nbl_max_displacement``); while it is below skin / 2 no pair can have
entered the cutoff sphere unseen, so the stored list is refreshed instead of
rebuilt (``nbl_verlet_refresh``: D and d recomputed from the positions, the
pairs with d < cutoff kept in the stored order).  Past skin / 2 the list is
rebuilt.  Either way the result holds the pair set ``neighbour_list`` returns
at ``cutoff`` for the current positions, rows ascending in i.  After a
refresh, D = r_j - r_i + S @ cell (periodic axes) differs from the rebuild's
arithmetic in the last bits, and a pair whose distance is within that
rounding of the cutoff can fall on the other side.

The reference rebuilds its list every step in its MD example
(examples/lj_langevin/lj_langevin_gpu.cu:171-179); this class is an addition.
Positions are torch CUDA float64 (n, 3) tensors; results are torch tensors.
"""

import ctypes

import numpy as np

from . import _matscipy_neighbours as _ext
from .neighbours import _host_metadata


def _lib():
    lib = _ext.lib
    P = ctypes.c_void_p
    lib.nbl_max_displacement.argtypes = [ctypes.c_int64, P, P, P, P]
    lib.nbl_max_displacement.restype = ctypes.c_int
    lib.nbl_verlet_refresh.argtypes = [ctypes.c_int64, P, P, P, P, P, P, ctypes.c_double,
                                       ctypes.POINTER(_ext.Outputs), ctypes.c_int64,
                                       ctypes.POINTER(ctypes.c_int64), P]
    lib.nbl_verlet_refresh.restype = ctypes.c_int
    return lib


class VerletList:
    """A reused pair list of one system; see the module docstring.

    cutoff, skin: floats (the list is built with cutoff + skin).  cell (3, 3,
    rows are lattice vectors) and pbc are fixed for the object's lifetime.
    quantities: the arrays ``update`` returns, any string over "ijdDS".
    """

    def __init__(self, cutoff, skin, cell, pbc=True, quantities="ijdDS", cell_origin=None):
        if not (skin >= 0.0 and cutoff > 0.0):
            raise ValueError("cutoff must be > 0 and skin >= 0")
        self.cutoff = float(cutoff)
        self.skin = float(skin)
        self.quantities = quantities
        _ext.quantity_flags(quantities)  # validates
        self._cell_origin = cell_origin
        co, ce, inv, pb, _ = _host_metadata(cell, pbc, None, cell_origin, 0)
        self._cell = np.ascontiguousarray(ce, dtype=np.float64)
        self._pbc = np.ascontiguousarray(np.asarray(pb, dtype=np.uint8))
        self._pbc_bool = np.asarray(pb, dtype=bool)
        self._lib = _lib()
        self._stored = None   # (i, j, S) of the skin list
        self._ref = None      # positions at the last build
        self.builds = 0
        self.refreshes = 0

    def _build(self, pos):
        from .neighbours import neighbour_list
        torch = _ext._torch()
        i, j, S = neighbour_list("ijS", positions=pos, cell=self._cell, pbc=self._pbc_bool,
                                 cell_origin=self._cell_origin,
                                 cutoff=self.cutoff + self.skin, array_namespace=torch)
        self._stored = (i.contiguous(), j.contiguous(), S.contiguous())
        self._ref = pos.detach().clone()
        self.builds += 1

    def max_displacement(self, positions):
        """Largest |r - r_build| over the atoms (a 0-d CUDA tensor; async)."""
        torch = _ext._torch()
        pos = _ext.import_device_positions(positions)
        out = torch.empty((), dtype=torch.float64, device=pos.device)
        stream = torch.cuda.current_stream(pos.device)
        with torch.cuda.device(pos.device):
            _ext.check(self._lib.nbl_max_displacement(
                int(pos.shape[0]), ctypes.c_void_p(pos.data_ptr()) if pos.numel() else None,
                ctypes.c_void_p(self._ref.data_ptr()) if pos.numel() else None,
                ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream.cuda_stream)))
        return out

    def update(self, positions):
        """The pairs within `cutoff` at `positions`, as a tuple in the order of
        `quantities` (a bare tensor for one character).  The tensors are views
        of the first rows of buffers sized for the stored (cutoff + skin)
        pairs, so that one device call writes them and reads the count."""
        torch = _ext._torch()
        pos = _ext.import_device_positions(positions)
        if self._stored is None or pos.shape[0] != self._ref.shape[0]:
            self._build(pos)
        elif float(self.max_displacement(pos).item()) * 2.0 >= self.skin:
            self._build(pos)
        else:
            self.refreshes += 1
        i, j, S = self._stored
        np_ = int(i.shape[0])
        stream = torch.cuda.current_stream(pos.device)
        sp = ctypes.c_void_p(stream.cuda_stream)
        n = ctypes.c_int64()
        dev = pos.device
        # room for every stored pair: one call writes the kept ones and
        # returns their number; the results are views of the first n rows
        want = set(self.quantities)
        bufs = {"i": torch.empty(np_ if "i" in want else 0, dtype=torch.int32, device=dev),
                "j": torch.empty(np_ if "j" in want else 0, dtype=torch.int32, device=dev),
                "D": torch.empty((np_ if "D" in want else 0, 3), dtype=torch.float64, device=dev),
                "d": torch.empty(np_ if "d" in want else 0, dtype=torch.float64, device=dev),
                "S": torch.empty((np_ if "S" in want else 0, 3), dtype=torch.int32, device=dev)}
        o = _ext.Outputs()
        o.first = bufs["i"].data_ptr() if "i" in want and np_ else None
        o.second = bufs["j"].data_ptr() if "j" in want and np_ else None
        o.distvec = bufs["D"].data_ptr() if "D" in want and np_ else None
        o.absdist = bufs["d"].data_ptr() if "d" in want and np_ else None
        o.shift = bufs["S"].data_ptr() if "S" in want and np_ else None
        with torch.cuda.device(dev):
            _ext.check(self._lib.nbl_verlet_refresh(
                np_, ctypes.c_void_p(i.data_ptr()) if np_ else None,
                ctypes.c_void_p(j.data_ptr()) if np_ else None,
                ctypes.c_void_p(S.data_ptr()) if np_ else None,
                ctypes.c_void_p(pos.data_ptr()) if pos.numel() else None,
                ctypes.c_void_p(self._cell.ctypes.data), ctypes.c_void_p(self._pbc.ctypes.data),
                self.cutoff, ctypes.byref(o), np_, ctypes.byref(n), sp))
        m = int(n.value)
        bufs = {k: v[:m] for k, v in bufs.items()}
        out = [bufs[c] for c in self.quantities]
        return out[0] if len(out) == 1 else tuple(out)
