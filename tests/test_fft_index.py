"""Index arithmetic of the FFT passes, checked on the CPU.

The x and column passes of lageunha_b200/csrc/pm.cu take per-element
quotients e / d by divisors known only at run time (pencil length L, row
length n/2 + 1, batch width P, ghosted row width n + 16) through `Div`: a
shift when d is a power of two, else p = trunc(float(e) * RN(1/d)) corrected
by one step towards the exact quotient. This restates that arithmetic in
IEEE float32 (numpy rounds float32 products and quotients to nearest, as the
device does) and checks it against integer division at every quotient
boundary e = k d - 1, k d, k d + 1 below the largest e any pass forms, for
every divisor the passes use on meshes from 16 to 4096. The c2r pass's
write phase, threads over (pencil, x) pairs, makes the same stores from the
same transform outputs as one loop per pencil over x.
"""
import numpy as np

# the largest e a pass forms: 64 pencils of a ghosted row of 4096 + 16
# (the c2r write; the column passes form at most 32 * 4096)
E_MAX = 64 * (4096 + 16)


def _div_q(e, d):
    """The device Div::q for 0 <= e < 2^24."""
    if d & (d - 1) == 0:
        return e >> (d.bit_length() - 1)
    inv = np.float32(1.0) / np.float32(d)
    p = (e.astype(np.float32) * inv).astype(np.int64)  # truncation, e >= 0
    r = e - p * d
    return np.where(r < 0, p - 1, np.where(r >= d, p + 1, p))


def _divisors():
    out = set()
    for n in range(16, 4097):
        half = n // 2
        L = half if n % 2 == 0 else n
        out.update({L, n // 2 + 1, n, n + 16})
    for P in range(1, 65):
        out.add(P)
    return sorted(out)


def test_quotient_matches_integer_division_at_every_boundary():
    for d in _divisors():
        k = np.arange(0, E_MAX // d + 2, dtype=np.int64)
        e = np.concatenate([k * d - 1, k * d, k * d + 1])
        e = e[(e >= 0) & (e < E_MAX)]
        got = _div_q(e, d)
        assert np.array_equal(got, e // d), d


def test_quotient_on_random_elements():
    rng = np.random.default_rng(3)
    for d in (17, 45, 75, 81, 129, 135, 272, 2049, 4112):
        e = rng.integers(0, E_MAX, size=200000, dtype=np.int64)
        assert np.array_equal(_div_q(e, d), e // d), d


KGHOST = 8  # ghost layers of the padded potential


def _c2r_writes_serial(n, P, row0, nrows, px, py):
    """(offset, pencil, element) of every store of the x c2r pass's write
    phase as one loop per pencil over x in [-KGHOST, n + KGHOST)."""
    out = set()
    for p in range(P):
        row = row0 + p
        if row >= nrows:
            break
        y, z = row % n, row // n
        ys = [y, y + n if y < KGHOST else (y - n if y >= n - KGHOST else None)]
        zs = [z, z + n if z < KGHOST else (z - n if z >= n - KGHOST else None)]
        for e in range(n + 2 * KGHOST):
            x = e - KGHOST
            xs = (x % n + n) % n
            for zz in zs:
                for yy in ys:
                    if zz is None or yy is None:
                        continue
                    out.add((x + KGHOST + px * ((yy + KGHOST) + py * (zz + KGHOST)), p, xs))
    return out


def _c2r_writes_flat(n, P, row0, nrows, px, py):
    """The same stores as the kernel makes them: threads over (pencil, x)
    pairs, p from the corrected float reciprocal, (y, z) by stepping from the
    block's first row."""
    W = n + 2 * KGHOST
    inv_w = np.float32(1.0) / np.float32(W)
    nrow = min(P, nrows - row0)
    y0, z0 = row0 % n, row0 // n
    out = set()
    for e in range(nrow * W):
        p = int(np.float32(e) * inv_w)
        r = e - p * W
        if r < 0:
            p, r = p - 1, r + W
        elif r >= W:
            p, r = p + 1, r - W
        y, z = y0 + p, z0
        while y >= n:
            y, z = y - n, z + 1
        ys = [y, y + n if y < KGHOST else (y - n if y >= n - KGHOST else None)]
        zs = [z, z + n if z < KGHOST else (z - n if z >= n - KGHOST else None)]
        x = r - KGHOST
        xs = x + n if x < 0 else (x - n if x >= n else x)
        for zz in zs:
            for yy in ys:
                if zz is None or yy is None:
                    continue
                out.add((x + KGHOST + px * ((yy + KGHOST) + py * (zz + KGHOST)), p, xs))
    return out


def test_c2r_flat_write_covers_the_serial_loop():
    for n, P in ((16, 8), (16, 64), (20, 32), (32, 16), (45, 64), (64, 64)):
        px = ((n + 2 * KGHOST) + 3) // 4 * 4
        py = n + 2 * KGHOST
        nrows = n * n
        for row0 in range(0, nrows, P):
            a = _c2r_writes_serial(n, P, row0, nrows, px, py)
            b = _c2r_writes_flat(n, P, row0, nrows, px, py)
            assert a == b, (n, P, row0)


# ------------------------------------------------------- padded pencil slots
# Element m of a pencil lives at shared-memory slot fslot(m) = m + m // 16
# (one spare slot after every 16 elements, so the first Stockham stage's
# stride-R writes fall on distinct bank pairs). This restates the Stockham
# stages of pm.cu (stockham_stage / fft_pencils) over those slots and checks
# the transform against numpy's FFT for the radix sequences the passes use.
def _fslot(m):
    return m + (m >> 4)


def _factorize(L, rmax=16):
    r = []
    while rmax >= 16 and L % 16 == 0:
        r.append(16); L //= 16
    if rmax >= 8 and L % 8 == 0:
        r.append(8); L //= 8
    while L % 4 == 0:
        r.append(4); L //= 4
    while L % 2 == 0:
        r.append(2); L //= 2
    while L % 3 == 0:
        r.append(3); L //= 3
    while L % 5 == 0:
        r.append(5); L //= 5
    assert L == 1
    return r


def _stockham_padded(x, ld, direction):
    """x: [P, L] complex; returns the [P, L] transform through buffers of
    P * ld slots addressed by fslot, stage by stage as the kernel does."""
    P, L = x.shape
    tw = np.exp(-2j * np.pi * np.arange(L) / L)
    a = np.zeros(P * ld, np.complex128)
    b = np.zeros(P * ld, np.complex128)
    for p in range(P):
        a[p * ld + _fslot(np.arange(L))] = x[p]
    src, dst = a, b
    Ns = 1
    for R in _factorize(L):
        jobs = L // R
        step = L // (Ns * R)
        j = np.arange(jobs)
        jn, k = j // Ns, j % Ns
        for p in range(P):
            v = np.stack([src[p * ld + _fslot(j + r * jobs)] for r in range(R)])
            w = np.stack([tw[(r * k * step) % L] for r in range(R)])
            if direction > 0:
                w = np.conj(w)
            v = v * w
            # size-R DFT with the pass's sign
            F = np.exp(direction * 2j * np.pi * np.outer(np.arange(R), np.arange(R)) / R)
            out = F @ v
            d0 = jn * Ns * R + k
            for r in range(R):
                dst[p * ld + _fslot(d0 + r * Ns)] = out[r]
        src, dst = dst, src
        Ns *= R
    return np.stack([src[p * ld + _fslot(np.arange(L))] for p in range(P)])


def test_padded_stockham_matches_numpy():
    rng = np.random.default_rng(5)
    for L, P in [(16, 3), (32, 2), (64, 2), (128, 1), (256, 1), (512, 1), (48, 2), (60, 2), (75, 1), (81, 1)]:
        x = rng.standard_normal((P, L)) + 1j * rng.standard_normal((P, L))
        for direction in (-1, 1):
            ld = _fslot(L - 1) + 1 + 3  # any stride at least the slots a pencil spans
            got = _stockham_padded(x, ld, direction)
            want = np.fft.fft(x, axis=1) if direction < 0 else np.fft.ifft(x, axis=1) * L
            assert np.allclose(got, want, atol=1e-9 * L), (L, P, direction)


def test_padded_slots_spread_the_first_stage_writes():
    """In the first stage (Ns = 1) job j writes elements R j + r; for the 16
    consecutive jobs of a half-warp and each r, the slots fall on 16
    distinct bank pairs (slot mod 16) for every radix the passes use."""
    for R in (2, 4, 8, 16):
        for j0 in range(0, 512 // R, 16):
            for r in range(R):
                pairs = {_fslot(R * j + r) % 16 for j in range(j0, j0 + 16)}
                assert len(pairs) == 16, (R, j0, r)
