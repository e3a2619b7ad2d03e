"""The autotuner (tpm_autotune): FFT launch shapes leave the forces unchanged;
group shapes change the tree force only within the parity tolerance of the
plain engine (rms 1e-3, 99th percentile 1e-2 against the reference's PM +
tree correction, oracle variant B)."""
import numpy as np
import pytest

from lageunha_b200 import engine as E
from lageunha_b200 import ic
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _rms(e):
    return float(np.sqrt(np.mean(np.square(e))))


def test_fft_tuning_keeps_the_forces():
    b = ic.lattice_box(48, 48, 8100, -2.0, 1.0, 100.0)
    with E.Engine(b.n_mesh, epsilon=0.05, law="gaussian", rs_split=0.9, rsphere=4.5) as eng:
        eng.load_fixed(b.pos)
        eng.compute(E.PART_PM)
        want = eng.forces()
        t = eng.autotune(E.TUNE_FFT)
        assert t["ms_fft"] <= t["ms_fft_default"] * 1.0001
        eng.compute(E.PART_PM)
        got = eng.forces()
    assert np.max(np.abs(got - want)) <= 1e-5 * np.max(np.abs(want))


@pytest.mark.parametrize("n", [40, 64])
def test_group_tuning_stays_within_parity(n):
    ps = ic.workload("clustered256", scale=n)
    pu = ps.positions_u32()
    pos = O.decode(n, ps.indx, ps.offset)
    fr = O.pm_force(n, pos).astype(np.float64) + O.tree_force(n, pos, variant=O.VARIANT_B, eps=0.05)
    with E.Engine(n, epsilon=0.05) as eng:
        eng.load_fixed(pu)
        t = eng.autotune(E.TUNE_FFT | E.TUNE_GROUPS)
        assert t["group_level"] in (2, 3) and t["group_max"] in (16, 32)
        eng.compute(E.PART_ALL)
        f = eng.forces()
        # every group shape, not only the chosen one
        for lev in (2, 3):
            for gm in (16, 32):
                tt = eng.tuning
                tt.group_level, tt.group_max = lev, gm
                eng.tuning = tt
                eng.compute(E.PART_ALL)
                e = O.rel_err(eng.forces(), fr)
                assert _rms(e) <= 1e-3 and np.percentile(e, 99) <= 1e-2, (lev, gm, _rms(e))
    e = O.rel_err(f, fr)
    assert _rms(e) <= 1e-3


def test_tuning_rejects_bad_values():
    with E.Engine(32, epsilon=0.05) as eng:
        t = eng.tuning
        t.group_level = 5
        with pytest.raises(E.EngineError):
            eng.tuning = t
        with pytest.raises(E.EngineError):
            eng.autotune()  # no particles loaded
