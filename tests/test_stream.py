"""Streamed evaluations (tpm_stream_submit / tpm_stream_wait): the results of
pipelined submissions equal the synchronous path's (load, compute, read) on
the same particles, up to the order of the deposit's float atomics (rms
relative difference 1e-7, at most 1e-3 on a particle whose total force
nearly cancels), the loaded particles stay loaded, and a third submission in
flight is refused."""
import numpy as np
import pytest

from lageunha_b200 import engine as E
from lageunha_b200 import ic
from oracle import oracle as O


def _sets(n):
    base = ic.workload("clustered256", scale=n).positions_u32()
    rng = np.random.default_rng(5)
    out = [base]
    for _ in range(2):
        shift = rng.integers(0, 2 ** 32, size=3, dtype=np.uint64).astype(np.uint32)
        out.append((base.astype(np.uint64) + shift).astype(np.uint32))  # the same field, moved periodically
    return out


def _sync_forces(eng, pos):
    eng.load_fixed(pos)
    eng.compute(E.PART_ALL)
    return eng.forces()


@pytest.mark.gpu
def test_streamed_results_match_the_synchronous_path():
    n = 64
    sets = _sets(n)
    with E.Engine(n, epsilon=0.05) as eng:
        want = [_sync_forces(eng, p) for p in sets]
        outs = [np.zeros((p.shape[0], 3), np.float32) for p in sets]
        t0 = eng.stream_submit(sets[0], outs[0])
        t1 = eng.stream_submit(sets[1], outs[1])
        eng.stream_wait(t0)
        t2 = eng.stream_submit(sets[2], outs[2])
        eng.stream_wait(t1)
        eng.stream_wait(t2)
    for got, ref in zip(outs, want):
        e = O.rel_err(got.astype(np.float64), ref.astype(np.float64))
        assert np.sqrt(np.mean(e * e)) <= 1e-5, np.sqrt(np.mean(e * e))
        assert np.max(e) <= 1e-3, np.max(e)


@pytest.mark.gpu
def test_loaded_particles_survive_and_three_in_flight_is_refused():
    n = 32
    sets = _sets(n)
    with E.Engine(n, epsilon=0.05) as eng:
        f_loaded = _sync_forces(eng, sets[0])
        outs = [np.zeros((p.shape[0], 3), np.float32) for p in sets]
        ta = eng.stream_submit(sets[1], outs[1])
        tb = eng.stream_submit(sets[2], outs[2])
        with pytest.raises(E.EngineError):
            eng.stream_submit(sets[0], outs[0])
        eng.stream_wait(ta)
        eng.stream_wait(tb)
        with pytest.raises(E.EngineError):
            eng.stream_wait(ta)          # already waited for
        eng.compute(E.PART_ALL)          # the loaded set, not the streamed ones
        f_again = eng.forces()
    assert np.max(O.rel_err(f_again.astype(np.float64), f_loaded.astype(np.float64))) <= 1e-4


@pytest.mark.gpu
def test_streamed_sizes_may_grow():
    small = ic.workload("plain64", scale=16).positions_u32()
    big = ic.workload("plain64", scale=32).positions_u32()
    with E.Engine(32, epsilon=0.05) as eng:
        want = _sync_forces(eng, big)
        fs = np.zeros((small.shape[0], 3), np.float32)
        fb = np.zeros((big.shape[0], 3), np.float32)
        eng.load_fixed(small)
        t = eng.stream_submit(big, fb)
        eng.stream_wait(t)
        t = eng.stream_submit(small, fs)
        eng.stream_wait(t)
    assert np.max(O.rel_err(fb.astype(np.float64), want.astype(np.float64))) <= 1e-4
    assert np.all(np.isfinite(fs)) and np.any(fs != 0)
