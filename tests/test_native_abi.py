"""The C-ABI library loads on a machine without a GPU and exports every entry
point declared in include/pamtra_b200.h with matching struct layouts."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "pamtra_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pamtra_b200_\w+)\s*\(", src)))


def test_exports_every_declared_symbol(native):
    lib = native.load()
    names = declared_functions()
    assert len(names) >= 12
    for nm in names:
        assert hasattr(lib, nm), nm
    assert set(names) == set(native.EXPORTS)


def test_struct_layouts(native):
    from pamtra_b200 import packing
    sizes = native.abi_sizes()
    assert sizes == (ctypes.sizeof(packing.Settings), ctypes.sizeof(packing.Species),
                     ctypes.sizeof(native.Columns), ctypes.sizeof(native.Outputs),
                     ctypes.sizeof(native.TmatrixIn), ctypes.sizeof(native.TmatrixOut))


def test_no_device_fails_loudly(native):
    import torch
    if torch.cuda.is_available():
        return
    import pytest
    with pytest.raises(RuntimeError):
        native.Engine(0)
