"""Zel'dovich initial conditions (tpm_ic_noise, tpm_ic_zeldovich) against the
reference's own code: the noise spectrum against PMSeedForce's mode loop run
on the reference's gasdev/ran3 (Cosmos/CosmosIC/PMSeedForce.c:293-399,
nr.c:317-384, compiled into oracle/_ref), the displacement field against the
reference's Zeldovich (Cosmos/CosmosIC/Zeldovich.c:14-100, compiled).

Tolerances: the noise is bit-exact except where the device's double log and
the host's differ in the last bit and the float result rounds the other way
(at most 1 ulp, on a tiny fraction of modes); displacements, velocities and
offsets within 1e-4 of their largest magnitude (float Stockham FFTs against
the oracle's double DFT)."""
import numpy as np
import pytest

from lageunha_b200 import engine as E
from oracle import oracle as O

need_ref = pytest.mark.skipif(not O.ref_available(O.VARIANT_A), reason="oracle/_ref not built (reference tree absent)")


def restated_noise(n, iseed, velpot=None):
    """PMSeedForce's mode loop and kx = 0 completion restated in Python over
    the Python restatement of gasdev/ran3 (small n only)."""
    hx = n // 2 + 1
    spec = np.zeros((n, n, hx), np.complex64)
    modes = []
    for k in range(n):
        kz = k - n if k > n // 2 else k
        for j in range(n):
            ky = j - n if j > n // 2 else j
            for i in range(hx):
                x = i * i + ky * ky + kz * kz
                if x != 0 and x <= (n // 2) ** 2:
                    modes.append((k, j, i, x))
    g = O.gasdev_pairs(-1 if iseed >= 0 else iseed, len(modes))
    for m, (k, j, i, x) in enumerate(modes):
        a, b = g[m]
        if velpot is not None:
            a, b = np.float32(velpot[x] * a), np.float32(velpot[x] * b)
        spec[k, j, i] = complex(a, b)
    c = spec[:, :, 0].copy()
    for kk in range(1, n // 2):
        c[n - kk, 0] = np.conj(c[kk, 0])
        for j in range(1, n // 2):
            c[n - kk, n - j] = np.conj(c[kk, j])
    for j in range(1, n // 2):
        c[0, n - j] = np.conj(c[0, j])
    for kk in range(1, n // 2):
        for j in range(n // 2 + 1, n):
            c[n - kk, n - j] = np.conj(c[kk, j])
    spec[:, :, 0] = c
    return spec


def power_law_velpot(n, slope=-2.0, amp=0.05):
    """An amplitude table of the reference's form pamp*bpower(rk)/rk^2 for a
    power-law P(k) ~ k^slope (bpower = sqrt(P)): a stand-in for a CAMB table."""
    k2 = np.arange((n // 2) ** 2 + 1, dtype=np.float64)
    rk = 2 * np.pi * np.sqrt(np.maximum(k2, 1.0))
    return (amp * rk ** (slope / 2) / rk ** 2 * n ** 3).astype(np.float32)


def test_velpot_table_normalisation():
    from lageunha_b200 import ic
    k = np.exp(np.linspace(np.log(1e-3), np.log(50), 400))
    p = 2e4 * (k / 0.02) / (1 + (k / 0.02) ** 3)
    # scaling to sigma_8 scales the table by sigma_8 / sigma_8(table)
    s = ic.sigma_tophat(k, p)
    v1 = ic.velpot_table(32, 100.0, k, p)
    v2 = ic.velpot_table(32, 100.0, k, p, sigma8=2 * s)
    assert np.allclose(v2[1:], 2 * v1[1:], rtol=1e-6) and v1[0] == 0
    # a power law P = A / k gives velpot ~ k2^(-1/4) / k2 = k2^(-5/4)
    v = ic.velpot_table(64, 100.0, k, 3.0 / k)
    assert np.allclose(v[16] / v[4], (16 / 4) ** -1.25, rtol=1e-5)


def test_ran3_known_answers():
    # ran3 with idum = -1: its state after initialisation gives these first
    # draws (the restatement above), checked against the reference below
    st = O._ran3_stream(-1)
    first = [next(st) for _ in range(3)]
    assert all(0 <= v < 10 ** 9 for v in first)
    g = O.gasdev_pairs(-1, 1000)
    assert abs(float(g.mean())) < 0.1 and abs(float(g.std()) - 1.0) < 0.1


@need_ref
@pytest.mark.parametrize("n,seed", [(8, 5), (16, -7), (12, -3)])
def test_restatement_matches_reference(n, seed):
    vp = None if seed >= 0 else power_law_velpot(n)
    assert np.array_equal(O.ref_ic_noise(n, seed, vp), restated_noise(n, seed, vp))


def _noise_close(got, want):
    """Equal except for rare 1-ulp differences (double log rounding)."""
    diff = got != want
    frac = float(np.mean(diff))
    if frac:
        a, b = got[diff], want[diff]
        for part in (np.real, np.imag):
            pa, pb = part(a).astype(np.float32), part(b).astype(np.float32)
            ulp = np.abs(np.spacing(np.maximum(np.abs(pa), np.abs(pb))))
            assert np.all(np.abs(pa - pb) <= ulp)
    return frac


@pytest.mark.gpu
@need_ref
@pytest.mark.parametrize("n,seed,weighted", [(16, 3, False), (32, -11, True), (48, -5, True), (128, -2024, True),
                                             (256, 7, False), (512, -99, True)])
def test_engine_noise_matches_reference(n, seed, weighted):
    """Sizes from one chunk of the device's jump-ahead stream (16) to many
    (128: 3 level-2 starts, 256: 23, 512: 177 starts over 45,312 chunks)."""
    vp = power_law_velpot(n) if weighted else None
    got = E.ic_noise(n, seed, vp)
    want = O.ref_ic_noise(n, seed, vp)
    assert got.shape == want.shape
    assert _noise_close(got, want) < 1e-4


def _ref_particles(n, seed, vp, fnl, gnl, vamp, pfact):
    fx, fy, fz = O.ref_zeldovich(n, O.ref_ic_noise(n, seed, vp), fnl, gnl)
    f32 = np.float32
    out = {}
    for c, f in zip("xyz", (fx, fy, fz)):
        vel = (f32(vamp) * (f32(vamp) * f.reshape(-1))).astype(np.float32)
        out["v" + c] = vel
        out[c] = (f32(pfact) * vel).astype(np.float32)
    return out


@pytest.mark.gpu
@need_ref
@pytest.mark.parametrize("n,seed,fnl,gnl", [(32, -11, 0.0, 0.0), (32, -11, 60.0, 0.0), (36, -4, 20.0, 3.0e4),
                                             (16, 9, 0.0, 0.0)])
def test_engine_zeldovich_matches_reference(n, seed, fnl, gnl):
    vp = power_law_velpot(n) if seed < 0 else None
    vamp, pfact = 0.83, float(n)
    rec = E.ic_zeldovich(n, seed, vp, fnl=fnl, gnl=gnl, vamp=vamp, pfact=pfact)
    want = _ref_particles(n, seed, vp, fnl, gnl, vamp, pfact)
    assert np.array_equal(rec["indx"], np.arange(n ** 3, dtype=np.uint64))
    for c in ("x", "y", "z", "vx", "vy", "vz"):
        scale = float(np.max(np.abs(want[c])))
        assert scale > 0
        assert np.max(np.abs(rec[c] - want[c])) <= 1e-4 * scale, c


@pytest.mark.gpu
def test_zeldovich_properties_and_forces():
    """At 128^3: the displacement is curl-free and of zero mean; the particles
    load into the engine and give finite forces."""
    n = 128
    vp = power_law_velpot(n, amp=0.02)
    rec = E.ic_zeldovich(n, -99, vp, vamp=1.0, pfact=1.0)
    for c in ("x", "y", "z"):
        assert abs(float(rec[c].astype(np.float64).mean())) <= 1e-5 * float(np.abs(rec[c]).max())
    # curl: d psi_x / dy - d psi_y / dx on the lattice, in k space
    px = rec["x"].reshape(n, n, n).astype(np.float64)
    py = rec["y"].reshape(n, n, n).astype(np.float64)
    kx = np.fft.fftfreq(n)[None, None, :]
    ky = np.fft.fftfreq(n)[None, :, None]
    cx, cy = np.fft.fftn(px), np.fft.fftn(py)
    curl = np.abs(ky * cx - kx * cy)
    div = np.abs(kx * cx + ky * cy)
    nyq = (np.abs(kx) == 0.5) | (np.abs(ky) == 0.5)
    assert float(np.max(np.where(nyq, 0, curl))) <= 1e-4 * float(np.max(div))
    with E.Engine(n, epsilon=0.05) as eng:
        eng.load_lagrangian(rec)
        eng.compute(E.PART_ALL)
        assert np.all(np.isfinite(eng.forces()))


@pytest.mark.gpu
def test_bad_ic_arguments():
    with pytest.raises(E.EngineError):
        E.ic_noise(14, 3)            # 14 = 2 * 7
    with pytest.raises(E.EngineError):
        E.ic_noise(16, -3, None)     # a weighted seed needs the table


@pytest.mark.gpu
def test_ic_power_spectrum_follows_the_table():
    """End to end: particles from a CAMB-like table (sigma_8 = 0.8 at 8 Mpc/h,
    growth 1/50) in a 200 Mpc/h box at 64^3, measured with the engine's
    CorrMeasure P(k) (per unit box volume): times L^3 it follows the table
    times growth^2 within the cosmic variance of the bins."""
    from lageunha_b200 import ic
    n, L, g = 64, 200.0, 1.0 / 50
    k = np.exp(np.linspace(np.log(1e-3), np.log(50), 400))
    p = 2e4 * (k / 0.02) / (1 + (k / 0.02) ** 3)
    rec = E.ic_zeldovich(n, -31, ic.velpot_table(n, L, k, p, growth=g, sigma8=0.8))
    with E.Engine(n, epsilon=0.05) as eng:
        eng.load_lagrangian(rec)
        eng.measure_power_spectrum(True)
        eng.compute(E.PART_PM)
        r = eng.power_spectrum(L)
    p8 = p * (0.8 / ic.sigma_tophat(k, p)) ** 2
    bins = np.arange(2, 13)
    want = g * g * ic._pk_interp(k, p8, 2 * np.pi * bins / L)
    ratio = r["pk"][bins] * L ** 3 / want
    assert np.all((ratio > 0.8) & (ratio < 1.25)), ratio
    assert abs(float(np.mean(ratio)) - 1.0) < 0.1, ratio


@pytest.mark.gpu
@need_ref
@pytest.mark.parametrize("n,seed", [(32, -11), (48, -5), (16, 2)])
def test_engine_2lpt_matches_reference(n, seed):
    """Second order against the reference's TwoLPT and selfdiffphi: the
    velocities and offsets of the combined first- and second-order
    potentials, within 1e-4 of their largest magnitude."""
    vp = power_law_velpot(n) if seed < 0 else None
    vamp, vamp2, damp1, damp2, pfact = 0.83, -0.61, 1.0, -3.0 / 7.0, float(n)
    rec = E.ic_2lpt(n, seed, vp, vamp=vamp, vamp2=vamp2, damp1=damp1, damp2=damp2, pfact=pfact)
    f32 = np.float32
    vel, off = O.ref_two_lpt(n, O.ref_ic_noise(n, seed, vp), f32(pfact) * f32(damp1), f32(pfact) * f32(damp2),
                             vamp, vamp2)
    assert np.array_equal(rec["indx"], np.arange(n ** 3, dtype=np.uint64))
    for a, c in enumerate("xyz"):
        for got, want in ((rec["v" + c], vel[a]), (rec[c], off[a])):
            scale = float(np.max(np.abs(want)))
            assert scale > 0
            assert np.max(np.abs(got - want)) <= 1e-4 * scale, c


@pytest.mark.gpu
@need_ref
@pytest.mark.parametrize("n,fnl,gnl", [(32, 100.0, 0.0), (24, 40.0, 2.0e4)])
def test_engine_2lpt_non_gaussian_matches_reference(n, fnl, gnl):
    """TwoLPT's non-Gaussian branch (TwoLPT.c:284-335: to the real potential,
    the local terms with the growth corrections, and back)."""
    seed, vp = -13, power_law_velpot(n)
    cos = dict(boxsize=200.0, omep=0.3, amax=50.0, growth=0.02)
    vamp, vamp2, damp1, damp2, pfact = 0.83, -0.61, 1.0, -3.0 / 7.0, float(n)
    rec = E.ic_2lpt(n, seed, vp, vamp=vamp, vamp2=vamp2, damp1=damp1, damp2=damp2, pfact=pfact, fnl=fnl, gnl=gnl,
                    **cos)
    f32 = np.float32
    vel, off = O.ref_two_lpt(n, O.ref_ic_noise(n, seed, vp), f32(pfact) * f32(damp1), f32(pfact) * f32(damp2),
                             vamp, vamp2, fnl=fnl, gnl=gnl, **cos)
    for a, c in enumerate("xyz"):
        for got, want in ((rec["v" + c], vel[a]), (rec[c], off[a])):
            assert np.max(np.abs(got - want)) <= 1e-4 * float(np.max(np.abs(want))), c


@pytest.mark.gpu
def test_2lpt_non_gaussian_needs_the_cosmology():
    p = E.TpmIcParams()
    p.n, p.iseed, p.fnl = 16, 3, 10.0
    rec = np.empty(16 ** 3, E.DM_DTYPE)
    assert E.load_library().tpm_ic_2lpt(p, rec.ctypes.data, E.MEM_HOST) == -1  # TPM_E_ARG
