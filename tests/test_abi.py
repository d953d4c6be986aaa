"""The C-ABI library: it loads without a GPU, exports every entry point
include/nbl_b200.h declares, and reports errors instead of aborting."""
import ctypes
import pathlib
import re

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "nbl_b200.h").read_text()
    return sorted(set(re.findall(r"NBL_API\s+[\w\s\*]*?\b(nbl_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("nbl_count", "nbl_fill", "nbl_fill_host", "nbl_neighbour_list_device",
              "nbl_last_error", "nbl_has_gpu", "nbl_device_type"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    from matscipy_neighbours import _matscipy_neighbours as ext
    lib = ctypes.CDLL(str(ext._LIB_PATH))
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_checked_build_exports_the_same_entry_points():
    """The checked build (build.py --checked) is a drop-in for the release
    library: same symbols, its version string says which it is."""
    from matscipy_neighbours import _matscipy_neighbours as ext
    path = ext._LIB_PATH.with_name("libnbl_b200_checked.so")
    if not path.exists():
        pytest.skip("checked build not built")
    lib = ctypes.CDLL(str(path))
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    lib.nbl_version.restype = ctypes.c_char_p
    assert b"checked" in lib.nbl_version()
    assert b"checked" not in ext.lib.nbl_version()


def test_library_is_sm100a_build():
    from matscipy_neighbours import _matscipy_neighbours as ext
    assert b"sm_100a" in ext.lib.nbl_version()
    assert ext._device_type == 2


def test_plan_without_gpu_reports_error():
    from matscipy_neighbours import _matscipy_neighbours as ext
    if ext._has_gpu:
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    st = ext.lib.nbl_plan_create(0, ctypes.byref(h))
    assert st == ext.NBL_ERROR_NO_DEVICE
    assert b"no CUDA device" in ext.lib.nbl_last_error()


def test_null_arguments_are_rejected():
    from matscipy_neighbours import _matscipy_neighbours as ext
    n = ctypes.c_int64()
    assert ext.lib.nbl_count(None, None, None, ctypes.byref(n)) == \
        ext.NBL_ERROR_INVALID_ARGUMENT
    assert ext.lib.nbl_fill(None, None, None) == ext.NBL_ERROR_INVALID_ARGUMENT


def test_api_fails_loudly_without_gpu():
    from matscipy_neighbours import _matscipy_neighbours as ext
    import matscipy_neighbours as m
    if ext._has_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(RuntimeError):
        m.neighbour_list("ij", positions=np.zeros((2, 3)), cell=np.eye(3), cutoff=1.0)


def _header_struct_fields(name):
    text = (ROOT / "include" / "nbl_b200.h").read_text()
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), text, re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    return re.findall(r"\b(\w+)\s*;", body)


def test_launch_config_layout_matches_the_header():
    """The binding's nbl_launch_config mirror has the header's fields, in
    order, all int (a field added on one side only would shift the others)."""
    from matscipy_neighbours import _matscipy_neighbours as ext
    fields = _header_struct_fields("nbl_launch_config")
    assert [n for n, _ in ext.LaunchConfig._fields_] == fields
    assert all(t is ctypes.c_int for _, t in ext.LaunchConfig._fields_)
    assert "thread_per_atom" in fields and "atoms_per_item" in fields


def test_launch_config_needs_a_plan():
    from matscipy_neighbours import _matscipy_neighbours as ext
    cfg = ext.LaunchConfig(thread_per_atom=1)
    assert ext.lib.nbl_plan_set_launch_config(None, ctypes.byref(cfg)) == \
        ext.NBL_ERROR_INVALID_ARGUMENT
    assert ext.lib.nbl_plan_get_launch_config(None, ctypes.byref(cfg)) == \
        ext.NBL_ERROR_INVALID_ARGUMENT
