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


# ------------------------------------------------------------ start cubes
# The walk starts at the 4-cell cubes that meet a group's reach: per axis the
# interval [lo, hi] (cells, unwrapped) becomes at most two runs of wrapped
# cube coordinates (axis_runs in tree.cu, restated here in float32 the way
# the device computes it). The runs must list every cube whose cells meet the
# interval modulo n, each once, for meshes that are and are not multiples of
# four (the last cube of an n = 45 mesh holds one cell).
def _axis_runs(lo, hi, n):
    f32 = np.float32
    lo, hi = f32(lo), f32(hi)
    ncube = (n + 3) >> 2
    fn = f32(n)
    if f32(hi - lo) >= fn:
        return [(0, ncube)]
    lw = f32(lo - fn * np.floor(f32(lo / fn)))
    if lw >= fn or lw < 0:
        lw = f32(0)
    hw = f32(lw + f32(hi - lo))
    a = min(int(lw * f32(0.25)), ncube - 1)
    if hw < fn:
        b = min(int(hw * f32(0.25)), ncube - 1)
        return [(a, b - a + 1)]
    b = min(int(f32(hw - fn) * f32(0.25)), ncube - 1)
    if b >= a:
        return [(0, ncube)]
    return [(a, ncube - a), (0, b + 1)]


def _cubes_meeting(lo, hi, n):
    ncube = (n + 3) >> 2
    out = set()
    for c in range(ncube):
        c_lo, c_hi = 4 * c, min(4 * c + 4, n)
        for k in range(int(np.floor(lo / n)) - 1, int(np.floor(hi / n)) + 2):
            if c_lo + k * n <= hi and c_hi + k * n > lo:
                out.add(c)
    return out


def test_start_cube_runs_cover_the_reach_once():
    rng = np.random.default_rng(23)
    for n in (16, 32, 45, 48, 81, 125, 128, 512):
        for _ in range(400):
            centre = rng.uniform(-1.0, n + 1.0)
            half = rng.uniform(0.0, 4.0) + 3.51
            lo, hi = centre - half, centre + half
            runs = _axis_runs(lo, hi, n)
            listed = [r0 + j for r0, cnt in runs for j in range(cnt)]
            assert len(listed) == len(set(listed)), (n, lo, hi, runs)
            assert set(listed) >= _cubes_meeting(lo, hi, n), (n, lo, hi, runs)
            assert all(0 <= c < (n + 3) >> 2 for c in listed)


def test_start_cube_index_split_by_float_reciprocal():
    """The walk splits its start-cube index j = jx + nx (jy + ny jz) with float
    reciprocals: q = int((j + 0.5) * rcp(d)). The product lies 0.5 / d from the
    nearest integer and the float error is far below that, so q = j // d for
    every j below 2^20 (the walk falls back to integer division above): here
    every divisor up to 96 cubes per axis, IEEE float32 as the device rounds."""
    j = np.arange(0, 1 << 20, dtype=np.int64)
    jf = j.astype(np.float32) + np.float32(0.5)
    for d in range(1, 97):
        q = (jf * (np.float32(1) / np.float32(d))).astype(np.int64)
        assert np.array_equal(q, j // d), d
