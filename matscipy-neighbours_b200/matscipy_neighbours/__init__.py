"""matscipy_neighbours (B200 engine) -- neighbour lists for particle simulations.

A drop-in for the reference package of the same name: the same public
functions, computed by hand-written sm_100a CUDA kernels behind a C-ABI
(``include/nbl_b200.h``).  The output of ``neighbour_list`` is bit-identical to
the reference's CPU path, including the order of pairs.
"""

from .neighbours import (
    DLPackTensor,
    coordination,
    first_neighbours,
    get_jump_indicies,
    mic,
    neighbour_list,
    neighbour_matrix,
    triplet_list,
)
from ._matscipy_neighbours import set_options
from .consumers import lennard_jones

__all__ = [
    "neighbour_list",
    "neighbour_matrix",
    "first_neighbours",
    "get_jump_indicies",
    "triplet_list",
    "mic",
    "coordination",
    "DLPackTensor",
    "set_options",
    "lennard_jones",
]
