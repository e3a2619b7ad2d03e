"""The C-ABI library: it loads without a GPU and exports every entry point
include/tpm_engine.h declares; without a device, creation fails with the
documented status instead of falling back to anything."""
import ctypes
import os
import re

import pytest

from lageunha_b200 import engine as E

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(ROOT, "include", "tpm_engine.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tpm_[a-z_0-9]+)\s*\(", text)))


def test_library_loads_and_exports_header():
    lib = E.load_library()
    names = _declared()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(E._SIGS), set(names) ^ set(E._SIGS)


def test_version_and_defaults():
    lib = E.load_library()
    assert b"sm_100a" in lib.tpm_version()
    p = E.default_params(64)
    assert p.n_mesh == 64 and abs(p.theta - 0.3) < 1e-7 and p.rsphere == 4.0
    assert abs(p.efold - 0.9) < 1e-7 and abs(p.epsilon - 0.1) < 1e-7


def test_bad_arguments_fail_loudly_without_gpu():
    lib = E.load_library()
    p = E.default_params(8)  # below the minimum mesh
    ctx = ctypes.c_void_p()
    rc = lib.tpm_create(ctypes.byref(p), 0, ctypes.byref(ctx))
    assert rc == -1 and b"n_mesh" in lib.tpm_last_error()
    p = E.default_params(64)
    p.theta = 1.5
    assert lib.tpm_create(ctypes.byref(p), 0, ctypes.byref(ctx)) == -1


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="checks the no-device path")
def test_no_device_is_an_error():
    with pytest.raises(E.EngineError) as ei:
        E.Engine(32)
    assert ei.value.code == -6
