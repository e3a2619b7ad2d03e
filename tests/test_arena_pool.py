"""The request loop's device arena: its range bookkeeping (RangePool,
lageunha_b200/csrc/arena_core.h) on the host.

The arena hands contexts sub-ranges of large HBM blocks: best fit, the rest
of a range kept free, a released range merged with its free neighbours in
the same block (never across blocks, which the driver returns separately).
The pool is host C++ with no CUDA in it, so this test compiles it with the
host compiler (tests/arena_pool_harness.cpp) and drives it with fake
addresses against a model of the live ranges.
"""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "lageunha_b200", "csrc")
ALIGN = 256


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    out = str(tmp_path_factory.mktemp("arena") / "libarena_pool.so")
    subprocess.run([cxx, "-O1", "-std=c++17", "-shared", "-fPIC", "-I", CSRC,
                    os.path.join(HERE, "arena_pool_harness.cpp"), "-o", out], check=True)
    lib = ctypes.CDLL(out)
    lib.pool_new.restype = ctypes.c_void_p
    lib.pool_delete.argtypes = [ctypes.c_void_p]
    lib.pool_add_block.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64]
    lib.pool_alloc.argtypes = [ctypes.c_void_p, ctypes.c_uint64]
    lib.pool_alloc.restype = ctypes.c_uint64
    lib.pool_release.argtypes = [ctypes.c_void_p, ctypes.c_uint64]
    lib.pool_release.restype = ctypes.c_int
    lib.pool_stats.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    return lib


class Pool:
    def __init__(self, lib):
        self.lib, self.p = lib, lib.pool_new()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.lib.pool_delete(self.p)

    def add(self, base, size):
        self.lib.pool_add_block(self.p, base, size)

    def alloc(self, n):
        return int(self.lib.pool_alloc(self.p, n))

    def release(self, a):
        return bool(self.lib.pool_release(self.p, a))

    def stats(self):
        out = np.zeros(4, np.int64)
        self.lib.pool_stats(self.p, out.ctypes.data)
        return {"reserved": int(out[0]), "in_use": int(out[1]), "free_ranges": int(out[2]),
                "largest_free": int(out[3])}


def _round(n):
    return max(ALIGN, (n + ALIGN - 1) // ALIGN * ALIGN)


def test_random_alloc_release_against_a_model(lib):
    """20000 seeded operations on two adjacent 4 MiB blocks: every range lies
    inside one block, is aligned and rounded, overlaps no live range, and the
    bytes in use match the model; at the end the free space is exactly the
    two whole blocks (merged within each, not across them)."""
    rng = np.random.default_rng(11)
    blk = 4 << 20
    bases = [0x10000000, 0x10000000 + blk]  # the second block starts where the first ends
    live = {}
    with Pool(lib) as pool:
        for b in bases:
            pool.add(b, blk)
        for _ in range(20000):
            if live and (rng.random() < 0.45 or len(live) > 200):
                a = list(live)[rng.integers(len(live))]
                assert pool.release(a)
                del live[a]
            else:
                n = int(rng.integers(1, 96 << 10))
                a = pool.alloc(n)
                if a == 0:
                    # no free range holds it: the model must agree that none could
                    assert _round(n) > pool.stats()["largest_free"]
                    continue
                size = _round(n)
                assert a % ALIGN == 0
                assert any(b <= a and a + size <= b + blk for b in bases)
                for o, s in live.items():
                    assert a + size <= o or o + s <= a
                live[a] = size
            assert pool.stats()["in_use"] == sum(live.values())
        for a in list(live):
            assert pool.release(a)
        st = pool.stats()
    assert st == {"reserved": 2 * blk, "in_use": 0, "free_ranges": 2, "largest_free": blk}


def test_best_fit_takes_the_smallest_hole(lib):
    """Holes of 4, 1 and 2 units between live ranges: a request of 2 units
    takes the 2-unit hole, not the first or the largest one."""
    with Pool(lib) as pool:
        pool.add(0x20000000, 64 * ALIGN)
        sizes = [4, 1, 1, 1, 2, 1]
        addrs = [pool.alloc(k * ALIGN) for k in sizes]
        for i in (0, 2, 4):  # free the 4-, 1- and 2-unit ranges, each between live ones
            assert pool.release(addrs[i])
        assert pool.alloc(2 * ALIGN) == addrs[4]
        assert pool.alloc(1 * ALIGN) == addrs[2]
        assert pool.alloc(3 * ALIGN) == addrs[0]  # the rest of the 4-unit hole stays free
        assert pool.stats()["in_use"] == (4 + 1 + 1 + 1 + 2 + 1 - 1) * ALIGN


def test_release_merges_neighbours_and_ignores_strangers(lib):
    with Pool(lib) as pool:
        pool.add(0x30000000, 8 * ALIGN)
        a, b, c = (pool.alloc(2 * ALIGN) for _ in range(3))
        assert pool.stats()["free_ranges"] == 1  # the tail
        assert pool.release(a) and pool.release(c)
        assert pool.stats()["free_ranges"] == 2  # a alone; c merged with the tail
        assert pool.release(b)  # joins both neighbours
        assert pool.stats() == {"reserved": 8 * ALIGN, "in_use": 0, "free_ranges": 1, "largest_free": 8 * ALIGN}
        assert not pool.release(b)  # already free
        assert not pool.release(0x30000000 + ALIGN)  # not a range start
        assert pool.alloc(9 * ALIGN) == 0  # larger than any free range
        assert pool.alloc(0) == 0x30000000  # empty requests take one unit
