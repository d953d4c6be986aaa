"""Neighbour lists of many independent systems in one launch.

``NeighbourListBatch`` plans a list of systems once (each with its own cell,
pbc and cutoff), then builds all their pair lists with one launch sequence --
by default a captured CUDA graph that is replayed on every ``run()`` -- while
positions change in place.  Each system's pairs are exactly what
``neighbour_list`` returns for that system alone (same order, same bits).

This is an addition to the reference's API (which handles one system per
call); it is built on the C-ABI ``nbl_batch_*`` entry points.
"""

import ctypes

import numpy as np

from . import _matscipy_neighbours as _ext
from .neighbours import _resolve_cutoff


class _System(ctypes.Structure):
    _fields_ = [("cell_origin", ctypes.c_void_p), ("cell", ctypes.c_void_p),
                ("inv_cell", ctypes.c_void_p), ("pbc", ctypes.c_void_p),
                ("nat", ctypes.c_int64), ("cutoff", ctypes.c_double)]


class _BatchRequest(ctypes.Structure):
    _fields_ = [("quantities", ctypes.c_int), ("nsys", ctypes.c_int32),
                ("systems", ctypes.c_void_p), ("positions", ctypes.c_void_p),
                ("positions_on_device", ctypes.c_int),
                ("per_atom_cutoff", ctypes.c_void_p), ("types", ctypes.c_void_p),
                ("per_type_cutoff_sq", ctypes.c_void_p), ("ncutoffs", ctypes.c_int32),
                ("aux_on_device", ctypes.c_int), ("grid", ctypes.c_int),
                ("precision", ctypes.c_int), ("autotune", ctypes.c_int)]


class _BatchOutputs(ctypes.Structure):
    _fields_ = [("first", ctypes.c_void_p), ("second", ctypes.c_void_p),
                ("distvec", ctypes.c_void_p), ("absdist", ctypes.c_void_p),
                ("shift", ctypes.c_void_p), ("sys_offsets", ctypes.c_void_p),
                ("capacity", ctypes.c_int64), ("positions", ctypes.c_void_p)]


def _sigs():
    lib = _ext.lib
    P = ctypes.c_void_p
    table = {
        "nbl_batch_create": ([ctypes.c_int, ctypes.POINTER(P)], ctypes.c_int),
        "nbl_batch_destroy": ([P], ctypes.c_int),
        "nbl_batch_setup": ([P, ctypes.POINTER(_BatchRequest), ctypes.c_int64], ctypes.c_int),
        "nbl_batch_run": ([P, P], ctypes.c_int),
        "nbl_batch_capture": ([P, P], ctypes.c_int),
        "nbl_batch_launch": ([P, P], ctypes.c_int),
        "nbl_batch_finish": ([P, P, ctypes.POINTER(ctypes.c_int64)], ctypes.c_int),
        "nbl_batch_get_outputs": ([P, ctypes.POINTER(_BatchOutputs)], ctypes.c_int),
        "nbl_batch_get_config": ([P, ctypes.POINTER(ctypes.c_int),
                                  ctypes.POINTER(ctypes.c_int),
                                  ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
        "nbl_batch_get_tickets": ([P, ctypes.POINTER(ctypes.c_int),
                                   ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
        "nbl_batch_get_launch_config": ([P, ctypes.POINTER(_ext.LaunchConfig),
                                         ctypes.POINTER(ctypes.c_float),
                                         ctypes.POINTER(ctypes.c_float)], ctypes.c_int),
    }
    for name, (args, res) in table.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return lib


_SHAPES = {"i": ((), np.int32), "j": ((), np.int32), "D": ((3,), np.float64),
           "d": ((), np.float64), "S": ((3,), np.int32)}


class NeighbourListBatch:
    """Pair lists of many systems, built together on one GPU.

    systems: a list of dicts with ``positions`` (n, 3), ``cell`` (3, 3, rows
    are lattice vectors), ``pbc``, ``cutoff`` and optionally ``numbers`` and
    ``cell_origin`` -- the arguments of ``neighbour_list``.  All systems must
    use the same kind of cutoff: all scalars, all per-atom radius arrays, or
    one shared per-type matrix / element-pair dict (with ``numbers``).

    precision: "fp32" (FP32 filter with the exact FP64 guard-band recheck) or
    "fp64"; both give the reference's pairs bit for bit.  graph: capture the
    build in a CUDA graph and replay it on ``run()``.  capacity: output pairs
    to reserve (None: the current count plus 25 %); ``run()`` grows it and
    rebuilds when a step needs more.  autotune: time the launch configuration
    at set-up.
    """

    def __init__(self, systems, quantities="ijdDS", *, precision="fp32", grid="auto",
                 capacity=None, graph=True, autotune=True, device=0):
        import torch
        self._torch = torch
        self._lib = _sigs()
        self.quantities = quantities
        self.flags = _ext.quantity_flags(quantities)
        self.device = torch.device("cuda", device)
        self.graph = graph
        self._precision = {"fp32": _ext.PRECISION_FP32_FILTER,
                           "fp64": _ext.PRECISION_FP64}[precision]
        self._grid = {"auto": _ext.GRID_AUTO, "dense": _ext.GRID_DENSE,
                      "morton": _ext.GRID_MORTON, "hashed": _ext.GRID_HASHED}[grid]
        self._autotune = 1 if autotune else 0
        self._keep = []
        # All work of the batch runs on this stream (a graph cannot be captured
        # on the legacy default stream); order other work against it with
        # torch.cuda.current_stream().wait_stream(batch.stream).
        self.stream = torch.cuda.Stream(self.device)
        self._sp = ctypes.c_void_p(self.stream.cuda_stream)
        self._prepare(systems)
        h = ctypes.c_void_p()
        _ext.check(self._lib.nbl_batch_create(device, ctypes.byref(h)))
        self._h = h
        self._setup(0 if capacity is None else int(capacity))

    # -- planning ----------------------------------------------------------
    def _prepare(self, systems):
        torch = self._torch
        self.nsys = len(systems)
        self.natoms = []
        sys_arr = (_System * max(self.nsys, 1))()
        pos_chunks, radius_chunks, type_chunks = [], [], []
        kinds = set()
        per_type = None
        for k, sd in enumerate(systems):
            pos = sd["positions"]
            if isinstance(pos, torch.Tensor):
                pos_np = None
                nat = int(pos.shape[0])
                pos_chunks.append(pos.to(self.device, torch.float64).reshape(-1, 3))
            else:
                pos_np = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
                nat = pos_np.shape[0]
                pos_chunks.append(torch.from_numpy(pos_np))
            numbers = sd.get("numbers")
            cell = sd.get("cell")
            if cell is None:
                raise ValueError(f"system {k}: a cell is required in a batch")
            from .neighbours import _host_metadata
            co, ce, inv, pb, nums = _host_metadata(cell, sd.get("pbc"), numbers,
                                                   sd.get("cell_origin"), nat,
                                                   positions=pos_np)
            rc, nums = _resolve_cutoff(sd["cutoff"], nums)
            rc_bin, per_atom, pt_sq, nc = _ext.resolve_cutoff(rc, nat)
            if per_atom is not None:
                kinds.add("atom")
                radius_chunks.append(torch.from_numpy(np.ascontiguousarray(per_atom)))
            elif pt_sq is not None:
                kinds.add("type")
                if per_type is not None and not np.array_equal(per_type[0], pt_sq):
                    raise ValueError("all systems of a batch must share one per-type "
                                     "cutoff table")
                per_type = (pt_sq, nc)
                type_chunks.append(torch.from_numpy(np.ascontiguousarray(nums,
                                                                         dtype=np.int32)))
            else:
                kinds.add("scalar")
            pbc8 = np.ascontiguousarray(pb.astype(np.uint8))
            self._keep.extend([co, ce, inv, pbc8])
            sys_arr[k].cell_origin = co.ctypes.data
            sys_arr[k].cell = ce.ctypes.data
            sys_arr[k].inv_cell = inv.ctypes.data
            sys_arr[k].pbc = pbc8.ctypes.data
            sys_arr[k].nat = nat
            sys_arr[k].cutoff = rc_bin
            self.natoms.append(nat)
        if len(kinds) > 1:
            raise ValueError("all systems of a batch must use the same kind of cutoff")
        self._systems = sys_arr
        dev = self.device
        self.positions = (torch.cat([c.to(dev) for c in pos_chunks]).contiguous()
                          if pos_chunks else torch.zeros((0, 3), dtype=torch.float64,
                                                         device=dev))
        self._radii = (torch.cat(radius_chunks).to(dev).contiguous()
                       if radius_chunks else None)
        self._types = (torch.cat(type_chunks).to(dev).contiguous()
                       if type_chunks else None)
        self._per_type = per_type
        self.atom_offsets = np.concatenate([[0], np.cumsum(self.natoms)]).astype(np.int64)

    def _request(self):
        r = _BatchRequest()
        r.quantities = self.flags
        r.nsys = self.nsys
        r.systems = ctypes.addressof(self._systems)
        r.positions = self.positions.data_ptr() if self.positions.numel() else None
        r.positions_on_device = 1
        r.per_atom_cutoff = self._radii.data_ptr() if self._radii is not None else None
        r.types = self._types.data_ptr() if self._types is not None else None
        if self._per_type is not None:
            pt, nc = self._per_type
            self._keep.append(pt)
            r.per_type_cutoff_sq = pt.ctypes.data
            r.ncutoffs = nc
        r.aux_on_device = 1
        r.grid = self._grid
        r.precision = self._precision
        r.autotune = self._autotune
        return r

    def _setup(self, capacity):
        req = self._request()
        _ext.check(self._lib.nbl_batch_setup(self._h, ctypes.byref(req), capacity))
        out = _BatchOutputs()
        _ext.check(self._lib.nbl_batch_get_outputs(self._h, ctypes.byref(out)))
        self._out = out
        self.capacity = int(out.capacity)
        self._captured = False
        if self.graph:
            _ext.check(self._lib.nbl_batch_capture(self._h, self._sp))
            self._captured = True

    # -- running -----------------------------------------------------------
    def launch(self):
        """Enqueue one build on ``self.stream`` (no synchronisation).  Work that
        changed the positions on another stream must be ordered before it."""
        self.stream.wait_stream(self._torch.cuda.current_stream(self.device))
        if self._captured:
            _ext.check(self._lib.nbl_batch_launch(self._h, self._sp))
        else:
            _ext.check(self._lib.nbl_batch_run(self._h, self._sp))

    def finish(self):
        """Wait for the last launch; returns the total pair count.  Grows the
        output capacity and rebuilds when the pairs did not fit."""
        n = ctypes.c_int64()
        st = self._lib.nbl_batch_finish(self._h, self._sp, ctypes.byref(n))
        if st == _ext.NBL_ERROR_CAPACITY:
            self._setup(int(n.value * 1.25) + 4096)
            self.launch()
            st = self._lib.nbl_batch_finish(self._h, self._sp, ctypes.byref(n))
        _ext.check(st)
        self.npairs = int(n.value)
        return self.npairs

    def run(self):
        """Build all pair lists; returns the total pair count."""
        self.launch()
        return self.finish()

    def config(self):
        """(count CTAs per SM, atoms per count sweep, fill CTAs per SM)."""
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _ext.check(self._lib.nbl_batch_get_config(self._h, ctypes.byref(a), ctypes.byref(b),
                                                  ctypes.byref(c)))
        return a.value, b.value, c.value

    def launch_config(self):
        """Everything the autotuner chose (``nbl_launch_config`` as a dict:
        grids, work-item striding, warps per CTA of each pass, atoms per FP32
        sweep, candidate staging, atoms per work item) plus the median
        count-phase and fill times it measured for that choice (ms; 0 without
        tuning)."""
        cfg = _ext.LaunchConfig()
        cms, fms = ctypes.c_float(), ctypes.c_float()
        _ext.check(self._lib.nbl_batch_get_launch_config(self._h, ctypes.byref(cfg),
                                                         ctypes.byref(cms), ctypes.byref(fms)))
        out = cfg.as_dict()
        fp32 = self._precision == _ext.PRECISION_FP32_FILTER
        out["count_candidates_per_warp"] = (384 if fp32 else 192) * (
            2 if out["count_large_staging"] else 1)
        out["tuned_count_ms"] = float(cms.value)
        out["tuned_fill_ms"] = float(fms.value)
        return out

    def tickets(self):
        """(count pass, fill pass) hand out work items by atomic ticket."""
        a, b = ctypes.c_int(), ctypes.c_int()
        _ext.check(self._lib.nbl_batch_get_tickets(self._h, ctypes.byref(a), ctypes.byref(b)))
        return bool(a.value), bool(b.value)

    # -- results -----------------------------------------------------------
    def _tensor(self, ch):
        torch = self._torch
        ptr = {"i": self._out.first, "j": self._out.second, "D": self._out.distvec,
               "d": self._out.absdist, "S": self._out.shift}[ch]
        extra, dt = _SHAPES[ch]
        tdt = torch.int32 if dt == np.int32 else torch.float64
        n = self.npairs
        if n == 0:
            return torch.zeros((0,) + extra, dtype=tdt, device=self.device)
        # A view of the batch's device buffer (valid until the next run).
        return _device_view(torch, ptr, (n,) + extra, tdt, self.device)

    def sys_offsets(self):
        """Pair offset of every system, int64 [nsys+1] (host)."""
        t = _device_view(self._torch, self._out.sys_offsets, (self.nsys + 1,),
                         self._torch.int64, self.device)
        return t.cpu().numpy()

    def results(self):
        """The concatenated outputs (torch CUDA tensors, in quantity order)."""
        return tuple(self._tensor(ch) for ch in self.quantities)

    def system(self, s):
        """Outputs of system s alone (views of the concatenated outputs)."""
        off = self.sys_offsets()
        out = self.results()
        return tuple(t[off[s]:off[s + 1]] for t in out)

    def close(self):
        if getattr(self, "_h", None):
            self.stream.synchronize()
            self._lib.nbl_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _device_view(torch, ptr, shape, dtype, device):
    """A torch tensor over device memory owned by the batch (no copy)."""
    elem = torch.empty((), dtype=dtype).element_size()
    n = int(np.prod(shape)) if len(shape) else 1
    typestr = {torch.int32: "<i4", torch.int64: "<i8", torch.float64: "<f8"}[dtype]

    class _CAI:
        pass

    holder = _CAI()
    holder.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr,
                                       "data": (int(ptr), False), "version": 3,
                                       "strides": None}
    t = torch.as_tensor(holder, device=device)
    assert t.element_size() == elem and t.numel() == n
    return t
