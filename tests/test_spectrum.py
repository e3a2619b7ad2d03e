"""Power spectrum of the mass assignment (tpm_set_power_spectrum /
tpm_power_spectrum) against the reference's CorrMeasure
(Cosmos/Correlation.c:13-117) on the same particles.

The golden fixture tests/golden/pk32.npz holds the reference's own output
(pmevol.map, 7 significant digits). Tolerances: P(k) per bin within 1e-4
relative (float TSC sums and FFT against the reference's, plus the 7 printed
digits); sigma_8 within 1e-4 relative; xi within 1e-4 of its largest value;
the log slope within 1e-3 absolute.
"""
import numpy as np
import pytest

from lageunha_b200 import engine as E
from lageunha_b200 import ic
from oracle import oracle as O

CASES = (("plain64", 32, 100.0), ("clustered256", 32, 25.0))


@pytest.mark.skipif(not O.ref_available(O.VARIANT_A), reason="oracle/_ref not built (reference tree absent)")
def test_golden_is_the_reference_output(golden_dir):
    g = np.load(f"{golden_dir}/pk32.npz")
    for name, n, box in CASES:
        ps = ic.workload(name, scale=n)
        r = O.ref_power_spectrum(n, ps.indx, ps.offset, box)
        for k in ("pk", "cor"):
            assert np.array_equal(r[k], g[f"{name}_{k}"]), (name, k)
        assert r["sigma8"] == g[f"{name}_sigma8"] and r["slope"] == g[f"{name}_slope"]


@pytest.mark.gpu
@pytest.mark.parametrize("name,n,box", CASES)
def test_engine_power_spectrum_matches_the_reference(golden_dir, name, n, box):
    g = np.load(f"{golden_dir}/pk32.npz")
    ps = ic.workload(name, scale=n)
    with E.Engine(n, epsilon=0.05) as eng:
        eng.load_fixed(ps.positions_u32())
        eng.measure_power_spectrum(True)
        eng.compute(E.PART_PM)
        r = eng.power_spectrum(box)
        # the measurement does not change the forces
        f_with = eng.forces()
        eng.measure_power_spectrum(False)
        eng.compute(E.PART_PM)
        f_without = eng.forces()
    ngh = n // 2
    want = g[f"{name}_pk"]
    assert want.shape[0] == ngh
    got = r["pk"][:ngh]
    assert np.all(np.abs(got[1:] - want[1:]) <= 1e-4 * np.abs(want[1:])), np.max(np.abs(got[1:] / want[1:] - 1))
    assert r["sigma8"] == pytest.approx(float(g[f"{name}_sigma8"]), rel=1e-4)
    cw = g[f"{name}_cor"]
    assert np.max(np.abs(r["cor"][:ngh] - cw)) <= 1e-4 * np.max(np.abs(cw))
    assert r["slope"] == pytest.approx(float(g[f"{name}_slope"]), abs=1e-3)
    assert np.max(np.abs(f_with - f_without)) <= 1e-5 * np.max(np.abs(f_without))


@pytest.mark.gpu
def test_power_spectrum_on_the_interlaced_path():
    """With the Gaussian law the first of the two interlaced grids is binned,
    the same mass assignment the reference measures."""
    n = 32
    ps = ic.workload("clustered256", scale=n)
    with E.Engine(n, epsilon=0.05) as ref_law, E.Engine(n, epsilon=0.05, law="gaussian", rs_split=0.8,
                                                        rsphere=4.0) as gauss:
        for eng in (ref_law, gauss):
            eng.load_fixed(ps.positions_u32())
            eng.measure_power_spectrum(True)
            eng.compute(E.PART_PM)
        a, b = ref_law.power_spectrum(25.0), gauss.power_spectrum(25.0)
    # float bin sums per block and atomic deposit order differ between the two runs
    assert np.allclose(a["pk"][1:], b["pk"][1:], rtol=1e-4, atol=0)


@pytest.mark.gpu
def test_power_spectrum_needs_an_evaluation():
    with E.Engine(32, epsilon=0.05) as eng:
        with pytest.raises(E.EngineError):
            eng.power_spectrum(100.0)
