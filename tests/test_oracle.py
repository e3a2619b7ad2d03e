"""CPU tests of the oracle (no GPU): the C restatement of the reference's
force path against the golden outputs of the reference itself
(tests/golden/, made by tests/golden/make_golden.py from oracle/_ref), against
the live reference build when it is present, and known-answer checks."""
import numpy as np
import pytest

from lageunha_b200 import ic
from oracle import oracle as O


def _g(golden_dir, name):
    return np.load(f"{golden_dir}/{name}")


def test_spline_table_bit_exact(golden_dir):
    g = _g(golden_dir, "plain16.npz")
    d, s = O.spline_table(int(g["n"]), 0.05)
    assert np.array_equal(d, g["spline_diff"])
    assert np.array_equal(s, g["spline_slope"])


def test_tsc_potential_pm_vs_reference(golden_dir):
    g = _g(golden_dir, "plain16.npz")
    n = int(g["n"])
    pos = O.decode(n, g["indx"], g["offset"])
    rho = O.tsc_density(n, pos)
    assert np.max(np.abs(rho - g["density"])) <= 2e-6
    phi = O.potential(n, pos)
    assert np.max(np.abs(phi - g["potential"])) <= 1e-6 * np.max(np.abs(g["potential"]))
    f = O.pm_force(n, pos)
    assert np.max(O.rel_err(f, g["pm_force"])) <= 1e-4


@pytest.mark.parametrize("variant", [O.VARIANT_A, O.VARIANT_B])
def test_tree_force_bit_exact_vs_reference(golden_dir, variant):
    key = "tree_force_A" if variant == O.VARIANT_A else "tree_force_B"
    for name in ("plain16.npz", "clustered32.npz", "sparse32.npz"):
        g = _g(golden_dir, name)
        n = int(g["n"])
        pos = O.decode(n, g["indx"], g["offset"])
        f = O.tree_force(n, pos, variant=variant, eps=0.05)
        sub = g["sub"] if "sub" in g else np.arange(pos.shape[0])
        assert np.array_equal(f[sub], g[key]), (name, variant)


def test_variants_differ_where_the_bugs_bite(golden_dir):
    # sparse buckets take DirectSummation, clustered ones accept nodes
    for name in ("clustered32.npz", "sparse32.npz"):
        g = _g(golden_dir, name)
        assert not np.array_equal(g["tree_force_A"], g["tree_force_B"])


def test_ewald_golden(golden_dir):
    g = _g(golden_dir, "plain16.npz")
    n = int(g["n"])
    pos = O.decode(n, g["indx"], g["offset"])
    few = O.ewald_force(n, pos, g["ewald_targets"], eps=0.05)
    assert np.max(O.rel_err(few, g["ewald_force"])) <= 1e-10


@pytest.mark.skipif(not O.ref_available(O.VARIANT_B), reason="oracle/_ref not built (reference tree absent)")
def test_live_reference_matches_restatement():
    n = 24
    ps = ic.workload("clustered256", scale=n)
    pos = O.decode(n, ps.indx, ps.offset)
    for v in (O.VARIANT_A, O.VARIANT_B):
        assert np.array_equal(O.tree_force(n, pos, variant=v, eps=0.05),
                              O.ref_tree_force(n, ps.indx, ps.offset, variant=v, eps=0.05))
    assert np.max(O.rel_err(O.pm_force(n, pos), O.ref_pm_force(n, ps.indx, ps.offset))) <= 1e-4


def test_pair_law_kat():
    """Two particles: the tree correction is the tabulated law at their
    separation (GetPointGrav, OST/Model4TreeForce.c:34-38)."""
    n = 32
    d, s = O.spline_table(n, 0.05)
    delta = np.float32(6.0 / 4096)
    for sep in (0.01, 0.3, 1.7, 3.9):
        pos = np.array([[10.0, 10.0, 10.0], [10.0 + sep, 10.0, 10.0]])
        f = O.tree_force(n, pos, eps=0.05).astype(np.float64)
        r = np.float32(sep)
        k = int(r * np.float32(1.0 / delta))
        law = d[k, 0] + s[k, 0] * float(r - np.float32(k) * delta)
        # target 0 minus source 1 is -sep along x
        assert abs(f[0, 0] - (-sep) * law) <= 1e-5 * abs(sep * law)
        assert np.allclose(f[0], -f[1], rtol=1e-6, atol=0)


def test_uniform_lattice_has_no_force():
    n = 16
    idx = np.arange(n ** 3, dtype=np.uint64)
    pos = O.decode(n, idx, np.zeros((n ** 3, 3), np.float32))
    # a single neighbour at one cell pulls with about 1/N^2 = 4e-3; the
    # lattice sums cancel to float rounding
    assert np.max(np.abs(O.tree_force(n, pos, eps=0.05))) < 1e-7
    assert np.max(np.abs(O.pm_force(n, pos))) < 1e-7


def test_morton_keys_match_a_slow_interleave():
    n = 48
    rng = np.random.default_rng(1)
    pu = rng.integers(0, 2 ** 32, size=(200, 3), dtype=np.uint64).astype(np.uint32)
    keys = O.morton_keys(pu, n)
    sub = 13 - O.cell_bits(n)
    for p, k in zip(pu, keys):
        q = [(int(c) * n) >> (32 - sub) for c in p]
        want = 0
        for b in range(13):
            for a in range(3):
                want |= ((q[a] >> b) & 1) << (3 * b + a)
        assert int(k) == want


def test_fixed_point_round_trip():
    ps = ic.workload("plain64", scale=16)
    pos = ps.positions_f64()
    back = ic.from_fixed_point(ps.positions_u32(), 16)
    d = np.abs(back - pos)
    d = np.minimum(d, 16 - d)
    assert np.max(d) <= 16 / 2 ** 32
