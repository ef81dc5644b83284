"""CPU tests of the C ABI library: it builds, loads and exports every
symbol include/radtran_b200.h declares; without a GPU it refuses to create a
context (no CPU fallback)."""
import ctypes as C
import os
import re

import pytest

from radtrancode_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "radtran_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rtb_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_python_export_list():
    assert sorted(_lib.EXPORTED) == declared_symbols()


def test_library_exports_every_declared_symbol():
    path = _lib.build()
    L = C.CDLL(path)
    for name in declared_symbols():
        assert hasattr(L, name), name


def test_version_string():
    assert b"sm_100a" in _lib.lib().rtb_version()


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU refusal")
def test_no_gpu_means_error_not_fallback():
    from radtrancode_b200 import cirsradg
    with pytest.raises(cirsradg.RtbError, match="RTB_ERR_CUDA"):
        cirsradg.Context(0)
