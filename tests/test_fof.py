"""Friends-of-friends groups (tpm_fof) against the FP64 oracle: the groups
are the connected components of "distance <= link" (FoF/fof.c:217-290), so
the partition is unique. Labels (smallest caller index of each group of
>= min_members, else -1) are compared exactly; the seeded sets have no pair
within float rounding of the link length."""
import numpy as np
import pytest

from lageunha_b200 import engine as E
from lageunha_b200 import ic
from oracle import oracle as O


def test_oracle_known_answer():
    # a chain of 5 linked across the periodic boundary, a pair, and loners
    n = 16
    pos = np.array([[15.95, 8, 8], [0.1, 8, 8], [0.25, 8, 8], [0.4, 8, 8], [15.8, 8, 8],  # chain (wraps)
                    [5, 5, 5], [5.15, 5, 5],                                                 # pair
                    [10, 10, 10], [12, 2, 7]], np.float64)
    lab, ng = O.fof_labels(n, pos, 0.2, 2)
    assert list(lab) == [0, 0, 0, 0, 0, 5, 5, -1, -1] and ng == 2
    lab, ng = O.fof_labels(n, pos, 0.2, 3)
    assert list(lab) == [0, 0, 0, 0, 0, -1, -1, -1, -1] and ng == 1


@pytest.mark.gpu
@pytest.mark.parametrize("name,n,link,minm", [("clustered256", 32, 0.2, 20), ("clustered256", 48, 0.1, 10),
                                              ("clustered256", 64, 0.15, 5), ("scale512", 32, 0.25, 3)])
def test_fof_matches_oracle(name, n, link, minm):
    ps = ic.workload(name, scale=n)
    pu = ps.positions_u32()
    pos = ic.from_fixed_point(pu, n)
    want, ngw = O.fof_labels(n, pos, link, minm)
    with E.Engine(n, epsilon=0.05) as eng:
        eng.load_fixed(pu)
        lab, ng = eng.fof(link, minm)
        # the context still evaluates forces afterwards
        eng.compute(E.PART_ALL)
        assert np.all(np.isfinite(eng.forces()))
    assert ng == ngw
    assert np.array_equal(lab.astype(np.int64), want)


@pytest.mark.gpu
def test_fof_singletons_and_no_groups():
    n = 16
    ps = ic.workload("plain64", scale=n)
    with E.Engine(n, epsilon=0.05) as eng:
        eng.load_fixed(ps.positions_u32())
        lab, ng = eng.fof(1e-4, 1)          # every particle its own group
        assert ng == ps.np and np.array_equal(lab, np.arange(ps.np, dtype=np.int32))
        lab, ng = eng.fof(1e-4, 2)          # no pair that close
        assert ng == 0 and np.all(lab == -1)
        with pytest.raises(E.EngineError):
            eng.fof(9.0, 2)                 # link of half the box
