"""ASE neighbour-list adapter (the reference's ``matscipy_neighbours._ase_plugin``,
which its packaging registers under the ``ase.plugins`` entry point,
pyproject.toml:22-23).  This tree ships no packaging metadata, so ASE does not
discover the module by itself: import it, or declare the entry point in the
package that installs it.

``neighbor_list`` follows ASE's neighbour-list protocol: ``(quantities,
atoms, cutoff, *, self_interaction=False)`` returning the flat ``i, j, d, D,
S`` arrays of ``matscipy_neighbours.neighbour_list``.  That list never holds
an atom paired with itself in the same image, so ``self_interaction=True`` is
refused rather than answered differently.  ``__ase_plugins__`` holds the
plugin record when the installed ASE has the plugin API and is empty
otherwise, so discovery of other plugins never breaks.  The engine is
imported only when the adapter is called.
"""
from __future__ import annotations

PLUGIN_NAME = "matscipy-neighbours"


def neighbor_list(quantities, atoms, cutoff, *, self_interaction=False):
    """Neighbour list of an ASE ``Atoms`` object through the B200 engine."""
    if self_interaction:
        raise NotImplementedError(
            "the matscipy-neighbours backend has no self_interaction=True mode")
    from .neighbours import neighbour_list as _engine_list

    return _engine_list(quantities, atoms, cutoff)


def _plugins():
    try:
        from ase._4.plugins.neighborlist import NeighborListPlugin
    except ImportError:
        return set()
    return {NeighborListPlugin(
        PLUGIN_NAME,
        long_name="matscipy-neighbours neighbour list on the B200 engine",
        citation="https://github.com/libAtoms/matscipy-neighbours",
        implementation="matscipy_neighbours._ase_plugin.neighbor_list",
    )}


__ase_plugins__ = _plugins()
