"""Host-side logic that needs no GPU: the ensemble and served workload
generators, the device-memory estimate the request loop admits by, and the
no-device behaviour of the ensemble and server entry points."""
import numpy as np
import pytest

from lageunha_b200 import engine as E
from lageunha_b200 import ic


def _smooth(m):
    for p in (2, 3, 5):
        while m % p == 0:
            m //= p
    return m == 1


def test_fft_friendly_sizes():
    for n in range(16, 300):
        m = ic.fft_friendly(n)
        assert _smooth(m)
        # no 2^a 3^b 5^c size is strictly nearer
        for k in range(1, abs(m - n)):
            assert not _smooth(n - k) and not _smooth(n + k), (n, m)
    assert ic.fft_friendly(64) == 64 and ic.fft_friendly(67) == 64 and ic.fft_friendly(141) == 144


def test_ensemble_box_generator():
    a, b = ic.ensemble_box(7, max_lattice=48), ic.ensemble_box(7, max_lattice=48)
    assert np.array_equal(a.pos, b.pos) and np.array_equal(a.vel, b.vel)  # seeded
    assert 32 <= a.n_lattice <= 48 and a.np == a.n_lattice ** 3
    assert a.n_mesh == ic.fft_friendly(a.n_lattice)
    assert a.pos.dtype == np.uint32 and a.pos.shape == (a.np, 3)
    # the mesh-cell positions are the lattice scaled to the mesh, displaced
    x = ic.from_fixed_point(a.pos, a.n_mesh)
    assert np.all((x >= 0) & (x < a.n_mesh))
    sizes = [ic.ensemble_spec(i)[0] for i in range(64)]
    assert min(sizes) >= 32 and max(sizes) <= 160
    # log-uniform: about half of the boxes below the geometric middle
    assert 20 <= sum(s < np.sqrt(32 * 160) for s in sizes) <= 44


def test_memory_estimate():
    e32, e64, e256 = (E.estimate_bytes(n, n ** 3) for n in (32, 64, 256))
    assert 0 < e32 < e64 < e256
    # per particle: positions, velocities, keys, sorted copies, forces, tree
    per = (e256 - E.estimate_bytes(256, 1)) / (256 ** 3 - 1)
    assert 150 < per < 400, per
    assert E.estimate_bytes(8, 100) == -1 and E.estimate_bytes(64, 0) == -1


def test_evolution_factors_need_no_device():
    f = E.evol_factors(E.cosmology(), 256, 10.0, 0.1)
    assert f["pfact"] == pytest.approx(25.6) and 0 < f["fact1"] < 1


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="checks the no-device path")
def test_server_without_device_is_an_error():
    with pytest.raises(E.EngineError) as ei:
        E.Server(hbm_cap_bytes=10 ** 9)
    assert ei.value.code == -6
    with pytest.raises(E.EngineError):
        E.Server(hbm_cap_bytes=0)
