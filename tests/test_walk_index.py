"""Index arithmetic of the tree walk (lageunha_b200/csrc/tree.cu), checked on
the CPU.

Each traversal iteration scans two per-lane counts across the warp: the
children a lane pushes (at most 8) and the particles it appends (its leaf's
count). When every count is below 2^18 the kernel scans them as one packed
word push | cnt << 9: the push sum (at most 256) stays in the low 9 bits and
the count sum (below 2^23) fits the upper 23. This restates the packed scan
in uint32 arithmetic and checks it against the two separate scans, at the
bounds and on random lanes.
"""
import numpy as np


def _inclusive(v):
    return np.cumsum(v.astype(np.uint64)).astype(np.uint64)


def _packed_scan(push, cnt):
    pk = (push.astype(np.uint32) | (cnt.astype(np.uint32) << np.uint32(9))).astype(np.uint32)
    incl = np.cumsum(pk, dtype=np.uint32)  # wraps like the device's 32-bit adds
    total = incl[-1]
    return incl & np.uint32(511), incl >> np.uint32(9), total & np.uint32(511), total >> np.uint32(9)


def _check(push, cnt):
    incl, pincl, total, ptotal = _packed_scan(push, cnt)
    assert np.array_equal(incl.astype(np.uint64), _inclusive(push))
    assert np.array_equal(pincl.astype(np.uint64), _inclusive(cnt))
    assert int(total) == int(push.sum()) and int(ptotal) == int(cnt.sum())


def test_packed_scan_at_its_bounds():
    _check(np.full(32, 8, np.uint32), np.full(32, (1 << 18) - 1, np.uint32))
    _check(np.zeros(32, np.uint32), np.zeros(32, np.uint32))
    # a lane either pushes children or appends particles
    push = np.where(np.arange(32) % 2 == 0, 8, 0).astype(np.uint32)
    cnt = np.where(np.arange(32) % 2 == 1, (1 << 18) - 1, 0).astype(np.uint32)
    _check(push, cnt)


def test_packed_scan_random_lanes():
    rng = np.random.default_rng(11)
    for _ in range(2000):
        kind = rng.integers(0, 4, size=32)
        push = np.where(kind == 2, rng.integers(1, 9, size=32), 0).astype(np.uint32)
        cnt = np.where(kind == 3, rng.integers(1, 1 << 18, size=32), 0).astype(np.uint32)
        _check(push, cnt)
