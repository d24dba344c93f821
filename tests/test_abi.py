"""The C-ABI library loads on a machine without a GPU, exports every entry
point declared in include/scarl.h, and its GPU entry points fail cleanly
(status code, no crash) when no device is visible."""
import ctypes as C
import os
import re

import pytest

import scarl_b200 as S
from scarl_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    txt = open(os.path.join(ROOT, "include", "scarl.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|double|const char\*)\s+(scarl_\w+)\s*\(", txt, re.M)))


def test_every_declared_symbol_is_exported():
    names = _declared()
    assert len(names) >= 30
    lib = _lib.lib()
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)


def test_version():
    assert b"sm_100a" in _lib.lib().scarl_version()


def test_no_gpu_is_a_status_not_a_crash():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    h = C.c_void_p()
    rc = _lib.lib().scarl_ctx_create(0, 0, C.byref(h))
    assert rc == _lib.EDEVICE and not h.value
    with pytest.raises(S.ScarlError):
        S.Context(0)


def test_null_context_is_rejected():
    assert _lib.lib().scarl_sync(None) == _lib.EINVAL
    assert _lib.lib().scarl_gen_padded(None, None, 4, None, None, None, None, 1, 0.5, 1, 0, 0,
                                       None) == _lib.EINVAL
