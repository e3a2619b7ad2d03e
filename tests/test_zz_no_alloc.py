"""The allocation-free Morton ordering (tpm_morton_order_noalloc).

Some callers cannot allocate device memory: codes that run all of the GPU's
memory through their own pool, and loops that cannot take the device-wide
synchronisation of cudaMalloc. For them the library offers the engine's
particle sort with its scratch in a fixed device array. These tests call it
through the C ABI and check it against the ordering the engine itself
computes (tpm_compute_forces + tpm_read_order), which is integer work and
must agree bit for bit, on two calls in a row with different particle sets
(the second call reuses the scratch the first one left).

This file is named to be collected last; it passes on its own in a fresh
process and after the other tests.
"""
import ctypes

import numpy as np
import pytest

from lageunha_b200 import engine as E
from lageunha_b200 import ic
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MAX_PARTICLES = 262144  # TPM_NOALLOC_MAX_PARTICLES in include/tpm_engine.h


def _engine_order(n, pu):
    with E.Engine(n, epsilon=0.05) as eng:
        eng.load_fixed(pu)
        eng.compute(E.PART_PM)
        return eng.order()


def _noalloc_order(n, pu):
    import torch

    lib = E.load_library()
    dev = torch.device("cuda:0")
    pos = torch.from_numpy(pu.view(np.int32)).to(dev)
    keys = torch.empty(pu.shape[0], dtype=torch.int64, device=dev)
    perm = torch.empty(pu.shape[0], dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = lib.tpm_morton_order_noalloc(pos.data_ptr(), pu.shape[0], n, keys.data_ptr(), perm.data_ptr(),
                                      ctypes.c_void_p(stream))
    assert rc == 0, lib.tpm_last_error()
    torch.cuda.synchronize(dev)
    return keys.cpu().numpy().view(np.uint64), perm.cpu().numpy().view(np.uint32)


def test_noalloc_order_matches_engine_twice():
    cases = [("clustered256", 48), ("plain64", 64)]  # 110592 and 262144 particles
    for name, n in cases:
        pu = ic.workload(name, scale=n).positions_u32()
        assert pu.shape[0] <= MAX_PARTICLES
        k_eng, p_eng = _engine_order(n, pu)
        k_na, p_na = _noalloc_order(n, pu)
        assert np.array_equal(k_na, k_eng), name
        assert np.array_equal(p_na, p_eng), name
        # and both are the CPU recomputation (stable argsort of the keys)
        order = O.sort_order(O.morton_keys(pu, n))
        assert np.array_equal(p_na.astype(np.int64), order), name


def test_noalloc_ragged_and_single_particle():
    """Counts that are not a multiple of the sort's 2048-particle tile (the
    partial last tile), a single particle (the sort returns at once and the
    keys and indices reach the caller's buffers by a copy), and a mesh that
    is not a power of two."""
    rng = np.random.default_rng(17)
    for np_, n in [(100003, 64), (1, 32), (54321, 48)]:
        pu = rng.integers(0, 2 ** 32, size=(np_, 3), dtype=np.uint64).astype(np.uint32)
        for _ in range(2):
            k_na, p_na = _noalloc_order(n, pu)
            k_ref = O.morton_keys(pu, n)
            order = O.sort_order(k_ref)
            assert np.array_equal(p_na.astype(np.int64), order), (np_, n)
            assert np.array_equal(k_na, k_ref[order]), (np_, n)


def test_noalloc_rejects_oversize_and_bad_arguments():
    import torch

    lib = E.load_library()
    dev = torch.device("cuda:0")
    buf = torch.empty(16, dtype=torch.int64, device=dev)
    rc = lib.tpm_morton_order_noalloc(buf.data_ptr(), MAX_PARTICLES + 1, 64, buf.data_ptr(), buf.data_ptr(), None)
    assert rc == -1 and b"TPM_NOALLOC_MAX_PARTICLES" in lib.tpm_last_error()
    rc = lib.tpm_morton_order_noalloc(None, 10, 64, buf.data_ptr(), buf.data_ptr(), None)
    assert rc == -1
