"""Differentiable pair lists: ``neighbour_list_autograd``.

Returns the reference's ``i, j, D, d, S`` for one system, with ``D`` and ``d``
attached to the autograd graph of ``positions`` and ``cell``.  The backward
pass is a hand-written CUDA kernel (``nbl_backward``): for the fixed pair
list, ``D = r_j - r_i + S @ cell`` (shift terms only on periodic axes) and
``d = |D|``, so with ``g = dL/dD + dL/dd * D / d`` it accumulates ``-g`` on
atom i, ``+g`` on atom j and ``S^T g`` on the cell -- a segmented reduction
over the i-sorted rows (no atomics) plus the j-side scatter.
"""

import ctypes

import numpy as np

from . import _matscipy_neighbours as _ext
from .neighbours import _host_metadata, _resolve_cutoff


class BackwardArgs(ctypes.Structure):
    """``nbl_backward_args`` (include/nbl_b200.h)."""
    _fields_ = [("npairs", ctypes.c_int64), ("nat", ctypes.c_int64),
                ("first", ctypes.c_void_p), ("second", ctypes.c_void_p),
                ("shift", ctypes.c_void_p), ("distvec", ctypes.c_void_p),
                ("absdist", ctypes.c_void_p), ("grad_distvec", ctypes.c_void_p),
                ("grad_absdist", ctypes.c_void_p), ("row_offsets", ctypes.c_void_p),
                ("pbc", ctypes.c_void_p), ("grad_positions", ctypes.c_void_p),
                ("grad_cell", ctypes.c_void_p), ("deterministic", ctypes.c_int)]


def _lib():
    lib = _ext.lib
    lib.nbl_backward.argtypes = [ctypes.POINTER(BackwardArgs), ctypes.c_void_p]
    lib.nbl_backward.restype = ctypes.c_int
    return lib


def _function():
    import torch

    class _PairList(torch.autograd.Function):
        @staticmethod
        def forward(ctx, positions, cell, pbc, cutoff, numbers, cell_origin, deterministic):
            dev = positions.device
            pos = positions.detach().to(torch.float64).contiguous()
            cell_np = cell.detach().cpu().numpy().astype(np.float64)
            nat = pos.shape[0]
            co, ce, inv, pb, nums = _host_metadata(cell_np, pbc, numbers, cell_origin, nat)
            rc, nums = _resolve_cutoff(cutoff, nums)
            rc, per_atom, per_type_sq, ncut = _ext.resolve_cutoff(rc, nat)
            pbc8 = np.ascontiguousarray(pb.astype(np.uint8))
            types = nums if per_type_sq is not None else None
            stream = torch.cuda.current_stream(dev)
            sp = ctypes.c_void_p(stream.cuda_stream)
            plan = _ext.plan_for(dev.index)
            req = _ext.make_request(31, co, ce, inv, pbc8, nat,
                                    ctypes.c_void_p(pos.data_ptr()) if nat else None, True,
                                    rc, per_atom, per_type_sq, ncut, types, dev.index)
            n = ctypes.c_int64()
            with torch.cuda.device(dev):
                _ext.check(_ext.lib.nbl_count(plan, ctypes.byref(req), sp, ctypes.byref(n)))
                P = int(n.value)
                i = torch.empty(P, dtype=torch.int32, device=dev)
                j = torch.empty(P, dtype=torch.int32, device=dev)
                D = torch.empty((P, 3), dtype=torch.float64, device=dev)
                d = torch.empty(P, dtype=torch.float64, device=dev)
                S = torch.empty((P, 3), dtype=torch.int32, device=dev)
                off = torch.empty(nat + 1, dtype=torch.int64, device=dev)
                _ext.check(_ext.lib.nbl_row_offsets(plan, ctypes.c_void_p(off.data_ptr()), sp))
                if P:
                    o = _ext._outputs_struct({"i": i, "j": j, "D": D, "d": d, "S": S},
                                             lambda t: t.data_ptr())
                    _ext.check(_ext.lib.nbl_fill(plan, ctypes.byref(o), sp))
            ctx.save_for_backward(i, j, S, D, d, off)
            ctx.pbc8 = pbc8
            ctx.nat = nat
            ctx.deterministic = bool(deterministic)
            ctx.cell_device = cell.device
            ctx.mark_non_differentiable(i, j, S)
            return i, j, D, d, S

        @staticmethod
        def backward(ctx, g_i, g_j, g_D, g_d, g_S):
            i, j, S, D, d, off = ctx.saved_tensors
            dev = D.device
            nat = ctx.nat
            grad_pos = torch.empty((nat, 3), dtype=torch.float64, device=dev)
            grad_cell = torch.empty(9, dtype=torch.float64, device=dev)
            gD = g_D.contiguous() if g_D is not None else None
            gd = g_d.contiguous() if g_d is not None else None
            a = BackwardArgs()
            a.npairs = D.shape[0]
            a.nat = nat
            a.first, a.second, a.shift = i.data_ptr(), j.data_ptr(), S.data_ptr()
            a.distvec, a.absdist = D.data_ptr(), d.data_ptr()
            a.grad_distvec = gD.data_ptr() if gD is not None else None
            a.grad_absdist = gd.data_ptr() if gd is not None else None
            a.row_offsets = off.data_ptr()
            a.pbc = ctx.pbc8.ctypes.data
            a.grad_positions = grad_pos.data_ptr()
            a.grad_cell = grad_cell.data_ptr()
            a.deterministic = 1 if ctx.deterministic else 0
            if gD is None and gd is None:
                grad_pos.zero_()
                grad_cell.zero_()
            else:
                stream = torch.cuda.current_stream(dev)
                with torch.cuda.device(dev):
                    _ext.check(_lib().nbl_backward(ctypes.byref(a),
                                                   ctypes.c_void_p(stream.cuda_stream)))
            return (grad_pos, grad_cell.reshape(3, 3).to(ctx.cell_device), None, None, None,
                    None, None)

    return _PairList


_FN = None


def neighbour_list_autograd(positions, cell, pbc, cutoff, numbers=None, cell_origin=None,
                            *, deterministic=False):
    """``(i, j, D, d, S)`` of one system on the GPU with ``D`` and ``d``
    differentiable with respect to ``positions`` ((n, 3) float64 CUDA tensor)
    and ``cell`` ((3, 3) float64 tensor, rows are lattice vectors).  The pair
    list itself is computed from the detached values, exactly as
    ``neighbour_list`` computes it.  ``deterministic=True`` makes the gradients
    bit-reproducible (the j-side reduction is ordered instead of atomic)."""
    global _FN
    if _FN is None:
        _FN = _function()
    return _FN.apply(positions, cell, pbc, cutoff, numbers, cell_origin, deterministic)
