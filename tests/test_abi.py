"""The C-ABI library loads and exports every entry point its header declares.
No compute calls: this runs without a GPU."""
import ctypes
import os
import re

import pytest

import amber_b200
from amber_b200 import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if h.endswith(".h"):
            src = open(os.path.join(ROOT, "include", h)).read()
            names += re.findall(r"AMBER_API\s+[\w\s\*]*?\b(amber_cuda_\w+)\s*\(", src)
    return names


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(amber_b200.LIB_PATH):
        build.build()
    return ctypes.CDLL(amber_b200.LIB_PATH)


def test_header_declares_entry_points():
    names = declared()
    assert len(names) >= 18
    assert set(amber_b200.EXPORTS) <= set(names)


def test_library_exports_every_declared_symbol(lib):
    for name in declared():
        assert hasattr(lib, name), f"{name} declared in include/ but not exported"


def test_create_without_sm100_fails_loudly():
    """No CPU fallback: without an sm_100 device the context cannot be made."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(amber_b200.AmberError) as e:
        amber_b200.Estimator()
    assert e.value.code == -7


def test_library_is_sm100a_only():
    """The build targets sm_100a only (no PTX for other architectures)."""
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
