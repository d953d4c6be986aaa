"""Consumers fused into the pair pass: results of a pair potential without
materialising the neighbour list.

``lennard_jones`` evaluates a truncated Lennard-Jones potential over exactly
the pairs ``neighbour_list`` would return, inside the engine's fill pass
(``nbl_lj_forces``): each atom's force is summed over its row, the energy over
all pairs, and no pair is ever written to memory.  The reference computes the
same forces in its GPU example from a materialised "ij" list with one thread
and three atomics per pair (examples/lj_langevin/lj_langevin_gpu.cu:59-74);
this is an addition to its API.
"""

import ctypes

import numpy as np

from . import _matscipy_neighbours as _ext
from .neighbours import _host_metadata, _is_on_device


def lennard_jones(positions, cutoff, *, cell, pbc=True, epsilon=1.0, sigma=1.0,
                  cell_origin=None):
    """Energy and forces of U(r) = 4 eps ((sigma/r)^12 - (sigma/r)^6) over all
    pairs closer than `cutoff` (a float), truncated there without a shift.

    positions: (n, 3) float64, host (numpy) or device (torch CUDA tensor or a
    CUDA __dlpack__ array).  Returns (energy, forces): a Python float and an
    (n, 3) numpy array for host input; a 0-d and an (n, 3) torch CUDA tensor,
    computed asynchronously on the current stream, for device input.
    """
    torch = _ext._torch()
    on_device = _is_on_device(positions)
    if on_device:
        pos_t = _ext.import_device_positions(positions)
        dev = pos_t.device
        host_pos = None
    else:
        host_pos = np.ascontiguousarray(positions, dtype=np.float64)
        if host_pos.ndim != 2 or (host_pos.shape[0] and host_pos.shape[1] != 3):
            raise ValueError("positions must have shape (n, 3)")
        dev = torch.device("cuda", 0)
        pos_t = torch.from_numpy(host_pos).to(dev)
    nat = int(pos_t.shape[0])
    if not isinstance(cutoff, (int, float)):
        raise TypeError("lennard_jones takes one scalar cutoff")
    co, ce, inv, pb, _ = _host_metadata(cell, pbc, None, cell_origin, nat)
    origin, ce, inv, pbc8 = _ext.coerce_geometry(co, ce, inv, pb)
    forces = torch.empty((nat, 3), dtype=torch.float64, device=dev)
    energy = torch.empty((), dtype=torch.float64, device=dev)
    plan = _ext.plan_for(dev.index)
    req = _ext.make_request(_ext.QUANTITY_FIRST, origin, ce, inv, pbc8, nat,
                            ctypes.c_void_p(pos_t.data_ptr()) if nat else None, True,
                            float(cutoff), None, None, 0, None, dev.index)
    stream = torch.cuda.current_stream(dev)
    with torch.cuda.device(dev):
        _ext.check(_ext.lib.nbl_lj_forces(plan, ctypes.byref(req), float(epsilon),
                                          float(sigma), ctypes.c_void_p(forces.data_ptr()),
                                          ctypes.c_void_p(energy.data_ptr()),
                                          ctypes.c_void_p(stream.cuda_stream)))
    if on_device:
        return energy, forces
    _ext.check(_ext.lib.nbl_check(plan, ctypes.c_void_p(stream.cuda_stream)))
    return float(energy.item()), forces.cpu().numpy()
