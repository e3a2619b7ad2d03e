"""Seeded synthetic particle sets for the TreePM force engine.

Zel'dovich-displaced lattices of a Gaussian random field with a power-law
spectrum, optionally with Plummer spheres planted in place of field
particles. The reference builds its initial conditions from CAMB spectra
(Cosmos/CosmosIC/Zeldovich.c:14-100, Cosmos/CosmosIC/MakeParticle.c:149-212);
these seeded sets stand in for them with the shapes, sizes and displacement
statistics the workloads name.

Two position encodings are produced:
  * the reference's XYZDBL form: a Lagrangian lattice index
    i + N*(j + N*k) plus a float offset from that lattice point
    (Cosmos/CosmosIC/cosmosic.h:285-288, eunha.h:1228-1232);
  * the engine's form: per axis a uint32 fixed-point coordinate
    u = round(frac(x/N) * 2^32), which wraps exactly with the period.
"""
from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass
class ParticleSet:
    n_mesh: int            # PM mesh cells per side (== lattice size here)
    box_mpc: float         # box side in Mpc/h (metadata)
    indx: np.ndarray       # (np,) uint64 Lagrangian index
    offset: np.ndarray     # (np, 3) float32 displacement from the lattice point, cells
    vel: np.ndarray        # (np, 3) float32 velocities (code units)
    seed: int

    @property
    def np(self) -> int:
        return int(self.indx.shape[0])

    def positions_f64(self) -> np.ndarray:
        """Decoded positions in [0, N) cells, as eunha.h:1228-1232 computes them."""
        return decode_positions(self.n_mesh, self.indx, self.offset)

    def positions_u32(self) -> np.ndarray:
        """(np, 3) uint32 fixed-point positions (engine layout, AoS)."""
        return to_fixed_point(self.positions_f64(), self.n_mesh)


def decode_positions(n: int, indx: np.ndarray, offset: np.ndarray) -> np.ndarray:
    idx = (indx.astype(np.uint64) << np.uint64(8)) >> np.uint64(8)
    nn = np.uint64(n)
    grid = np.stack([idx % nn, (idx % (nn * nn)) // nn, idx // (nn * nn)], axis=1).astype(np.float64)
    return np.fmod(offset.astype(np.float64) + grid + n, float(n))


def to_fixed_point(pos: np.ndarray, n: int) -> np.ndarray:
    """round(frac(x/N) * 2^32) mod 2^32, computed in float64."""
    frac = np.mod(pos / float(n), 1.0)
    u = np.rint(frac * 4294967296.0)
    u = np.where(u >= 4294967296.0, 0.0, u)
    return u.astype(np.uint64).astype(np.uint32)


def from_fixed_point(u: np.ndarray, n: int) -> np.ndarray:
    return u.astype(np.float64) * (float(n) / 4294967296.0)


def _displacement_field_torch(white: np.ndarray, spec_index: float, damp: float, rms_target: float,
                              device: str) -> np.ndarray:
    """The transforms of _displacement_field done by torch.fft on a GPU
    (FP64), for the 512^3 workload; same field up to FFT rounding."""
    import torch
    n = white.shape[0]
    wk = torch.fft.rfftn(torch.from_numpy(white).to(device))
    f = torch.fft.fftfreq(n, dtype=torch.float64, device=device) * 2 * np.pi
    fr = torch.fft.rfftfreq(n, dtype=torch.float64, device=device) * 2 * np.pi
    kz, ky, kx = f[:, None, None], f[None, :, None], fr[None, None, :]
    k2 = kx * kx + ky * ky + kz * kz
    k2[0, 0, 0] = 1.0
    amp = torch.pow(k2, spec_index / 4.0) * torch.exp(-0.5 * damp * damp * k2)
    amp[0, 0, 0] = 0.0
    dk = wk * amp / k2
    del wk, amp
    psi = np.empty((3, n, n, n), dtype=np.float64)
    for c, kc in enumerate((kx, ky, kz)):
        psi[c] = torch.fft.irfftn(1j * kc * dk, s=(n, n, n), dim=(0, 1, 2)).cpu().numpy()
    del dk
    rms = np.sqrt(np.mean(np.sum(psi * psi, axis=0)))
    psi *= rms_target / rms
    return psi


def _displacement_field(n: int, rng: np.random.Generator, spec_index: float, damp: float,
                        rms_target: float, device: str | None = None) -> np.ndarray:
    """Zel'dovich displacement psi = IFFT[i k delta_k / k^2] of a Gaussian
    field with P(k) = A k^n exp(-(damp k)^2) (k in radians per cell), scaled so
    that the rms of |psi| equals rms_target cells. Returns (3, n, n, n) [z][y][x].
    device: do the transforms with torch on that CUDA device."""
    white = rng.standard_normal((n, n, n), dtype=np.float64)
    if device is not None:
        return _displacement_field_torch(white, spec_index, damp, rms_target, device)
    wk = np.fft.rfftn(white)
    kz = 2 * np.pi * np.fft.fftfreq(n)[:, None, None]
    ky = 2 * np.pi * np.fft.fftfreq(n)[None, :, None]
    kx = 2 * np.pi * np.fft.rfftfreq(n)[None, None, :]
    k2 = kx * kx + ky * ky + kz * kz
    k2[0, 0, 0] = 1.0
    amp = np.power(k2, spec_index / 4.0) * np.exp(-0.5 * damp * damp * k2)
    amp[0, 0, 0] = 0.0
    dk = wk * amp
    psi = np.empty((3, n, n, n), dtype=np.float64)
    for c, kc in enumerate((kx, ky, kz)):
        psi[c] = np.fft.irfftn(1j * kc * dk / k2, s=(n, n, n), axes=(0, 1, 2))
    rms = np.sqrt(np.mean(np.sum(psi * psi, axis=0)))
    psi *= rms_target / rms
    return psi


def _wrap_offset(off: np.ndarray, n: int) -> np.ndarray:
    return (off + 0.5 * n) % n - 0.5 * n


def zeldovich(n: int, seed: int, spec_index: float = -2.0, damp: float = 0.5,
              rms_disp: float = 0.3, box_mpc: float = 100.0, vel_factor: float = 0.0,
              device: str | None = None) -> ParticleSet:
    """n^3 particles on an n^3 mesh, displaced from the lattice by psi."""
    rng = np.random.Generator(np.random.PCG64(seed))
    psi = _displacement_field(n, rng, spec_index, damp, rms_disp, device)
    # lattice index i + n*(j + n*k) for the point (x=i, y=j, z=k)
    offset = np.stack([psi[0].ravel(), psi[1].ravel(), psi[2].ravel()], axis=1)
    offset = _wrap_offset(offset, n).astype(np.float32)
    indx = np.arange(n ** 3, dtype=np.uint64)
    vel = (vel_factor * offset).astype(np.float32)
    return ParticleSet(n, box_mpc, indx, offset, vel, seed)


def plant_plummer(ps: ParticleSet, seed: int, n_spheres: int, scale_cells: float,
                  nmin: int, nmax: int) -> ParticleSet:
    """Replace randomly chosen field particles by n_spheres Plummer spheres
    of scale radius scale_cells, each with a particle count drawn uniformly in
    [nmin, nmax]; the total particle count does not change."""
    n = ps.n_mesh
    rng = np.random.Generator(np.random.PCG64(seed + 7919))
    counts = rng.integers(nmin, nmax + 1, size=n_spheres)
    centres = rng.random((n_spheres, 3)) * n
    total = int(counts.sum())
    if total > ps.np // 2:
        raise ValueError("Plummer spheres would replace more than half of the particles")
    chosen = rng.choice(ps.np, size=total, replace=False)
    # Plummer radius from the cumulative mass M(<r)/M = r^3/(r^2+a^2)^{3/2}
    u = rng.random(total) * 0.99
    r = scale_cells / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
    cth = rng.uniform(-1, 1, total)
    phi = rng.uniform(0, 2 * np.pi, total)
    sth = np.sqrt(1 - cth * cth)
    d = np.stack([r * sth * np.cos(phi), r * sth * np.sin(phi), r * cth], axis=1)
    cid = np.repeat(np.arange(n_spheres), counts)
    target = np.mod(centres[cid] + d, n)
    grid = decode_positions(n, ps.indx[chosen], np.zeros((total, 3), np.float32))
    offset = ps.offset.copy()
    offset[chosen] = _wrap_offset(target - grid, n).astype(np.float32)
    vel = ps.vel.copy()
    vel[chosen] = 0.0
    return ParticleSet(n, ps.box_mpc, ps.indx.copy(), offset, vel, ps.seed)


def fft_friendly(n: int) -> int:
    """The 2^a 3^b 5^c size nearest to n (ties to the larger)."""
    best = None
    for m in range(max(2, n - n // 4), n + n // 4 + 2):
        k = m
        for p in (2, 3, 5):
            while k % p == 0:
                k //= p
        if k == 1 and (best is None or abs(m - n) < abs(best - n) or (abs(m - n) == abs(best - n) and m > best)):
            best = m
    return best


@dataclasses.dataclass
class Box:
    """One box of an ensemble or a served request: n_lattice^3 particles on an
    n_mesh^3 PM mesh, in the engine's uint32 fixed-point form."""
    n_mesh: int
    n_lattice: int
    box_mpc: float
    spec_index: float
    pos: np.ndarray        # (np, 3) uint32
    vel: np.ndarray        # (np, 3) float32, cells per unit of the drift factor
    seed: int

    @property
    def np(self) -> int:
        return int(self.pos.shape[0])


def lattice_box(n_lattice: int, n_mesh: int, seed: int, spec_index: float, rms_disp: float, box_mpc: float,
                vel_factor: float = 0.0, damp: float = 0.5) -> Box:
    """n_lattice^3 particles displaced from their lattice by a Zel'dovich
    field (rms displacement rms_disp lattice spacings), placed on an n_mesh^3
    mesh: x = (q + psi) * n_mesh / n_lattice cells."""
    rng = np.random.Generator(np.random.PCG64(seed))
    psi = _displacement_field(n_lattice, rng, spec_index, damp, rms_disp)
    g = np.arange(n_lattice, dtype=np.float64)
    qz, qy, qx = np.meshgrid(g, g, g, indexing="ij")
    scale = n_mesh / n_lattice
    x = np.stack([(qx + psi[0]).ravel(), (qy + psi[1]).ravel(), (qz + psi[2]).ravel()], axis=1) * scale
    vel = (vel_factor * scale * np.stack([psi[0].ravel(), psi[1].ravel(), psi[2].ravel()], axis=1)).astype(np.float32)
    return Box(n_mesh, n_lattice, box_mpc, spec_index, to_fixed_point(np.mod(x, n_mesh), n_mesh), vel, seed)


# The batched ensemble: 64 boxes, N_p^(1/3) log-uniform in [32, 160], mesh the
# nearest 2^a 3^b 5^c size, L uniform in [50, 300] Mpc/h, P(k) ~ k^n with n
# uniform in [-2.5, -1.5], rms displacement 1 spacing, v = 0.5 psi.
ENSEMBLE_BOXES = 64


def ensemble_spec(b: int, max_lattice: int = 160, min_lattice: int = 32) -> tuple:
    """(lattice size, box size in Mpc/h, spectral index) of ensemble box b."""
    rng = np.random.Generator(np.random.PCG64(4000 + b))
    nl = int(round(np.exp(rng.uniform(np.log(min_lattice), np.log(max_lattice)))))
    box = float(rng.uniform(50.0, 300.0))
    ns = float(rng.uniform(-2.5, -1.5))
    return nl, box, ns


def ensemble_box(b: int, max_lattice: int = 160, min_lattice: int = 32) -> Box:
    nl, box, ns = ensemble_spec(b, max_lattice, min_lattice)
    return lattice_box(nl, fft_friendly(nl), 4000 + b, ns, 1.0, box, vel_factor=0.5)


def ensemble(nbox: int = ENSEMBLE_BOXES, max_lattice: int = 160, min_lattice: int = 32) -> list:
    return [ensemble_box(b, max_lattice, min_lattice) for b in range(nbox)]


def workload(name: str, scale: int | None = None, device: str | None = None) -> ParticleSet:
    """The named synthetic workloads. `scale` overrides the mesh size (for
    parity-sized cases with the same statistics).

    plain64:      64^3, L=100 Mpc/h, P(k) = A k^-2 exp(-(0.5 k)^2), rms 0.3
    clustered256: 256^3, L=200, same P(k) form, rms 1.5, plus 200 Plummer
                  spheres (a = 0.5 Mpc/h = 0.64 cells, 2000-20000 particles)
    scale512:     512^3, L=500, P(k) ~ k^-2.5, rms 2, v = 0.5 psi
    """
    if name == "plain64":
        n = scale or 64
        return zeldovich(n, seed=1, spec_index=-2.0, damp=0.5, rms_disp=0.3, box_mpc=100.0)
    if name == "clustered256":
        n = scale or 256
        ps = zeldovich(n, seed=2, spec_index=-2.0, damp=0.5, rms_disp=1.5, box_mpc=200.0)
        frac = (n / 256.0) ** 3
        nsph = max(1, int(round(200 * frac))) if n < 256 else 200
        a_cells = 0.5 / 200.0 * 256.0
        return plant_plummer(ps, seed=2, n_spheres=nsph, scale_cells=a_cells, nmin=2000 if n >= 128 else 200,
                             nmax=20000 if n >= 128 else 2000)
    if name == "scale512":
        n = scale or 512
        return zeldovich(n, seed=3, spec_index=-2.5, damp=0.5, rms_disp=2.0, box_mpc=500.0, vel_factor=0.5,
                         device=device)
    raise KeyError(name)


# ---------------------------------------------------------------- amplitude tables
# The reference scales each noise mode of its initial conditions by
# pamp*bpower(rk)/rk^2 (Cosmos/CosmosIC/PMSeedForce.c:326), with bpower the
# square root of the CAMB power spectrum in its units (P(k) = (pamp bpower)^2
# boxsize^3, PMSeedForce.c:296-297), pamp normalising the top-hat variance at
# 8 Mpc/h to 1/bias, times the growth ratio bini/bnow and N^3 sqrt(1/2)
# (PMSeedForce.c:250-295). Its bpower and the normalising integral are
# Fortran (CosmosIC/sub.lynx.camb.F), which this image cannot compile; the
# table below is built from the same definitions by this module.

def read_pk_table(path: str):
    """(k [h/Mpc], P(k) [(Mpc/h)^3]) from a whitespace-separated two-column
    file such as CAMB's matter power output."""
    a = np.loadtxt(path, usecols=(0, 1), ndmin=2)
    return a[:, 0].astype(np.float64), a[:, 1].astype(np.float64)


def _pk_interp(k_tab, p_tab, k):
    """Log-log interpolation of the table, power-law continued past its ends."""
    lk, lp = np.log(k_tab), np.log(p_tab)
    x = np.log(np.maximum(k, 1e-30))
    y = np.interp(x, lk, lp)
    lo, hi = x < lk[0], x > lk[-1]
    if lo.any():
        s = (lp[1] - lp[0]) / (lk[1] - lk[0])
        y[lo] = lp[0] + s * (x[lo] - lk[0])
    if hi.any():
        s = (lp[-1] - lp[-2]) / (lk[-1] - lk[-2])
        y[hi] = lp[-1] + s * (x[hi] - lk[-1])
    return np.exp(y)


def sigma_tophat(k_tab, p_tab, radius: float = 8.0) -> float:
    """rms density contrast in a top-hat sphere of `radius` Mpc/h:
    sigma^2 = 1/(2 pi^2) int k^2 P(k) W(kR)^2 dk, W(x) = 3 (sin x - x cos x)/x^3
    (the integrand of the reference's bpowint, sub.lynx.camb.F:214-228)."""
    k = np.exp(np.linspace(np.log(1e-4), np.log(1e2), 20001))
    x = k * radius
    w = np.where(x > 0.02, 3 * (np.sin(x) - x * np.cos(x)) / np.maximum(x, 1e-30) ** 3, 1 - x * x / 10)
    f = k ** 3 * _pk_interp(k_tab, p_tab, k) * w * w
    return float(np.sqrt(np.trapezoid(f, np.log(k)) / (2 * np.pi ** 2)))


def velpot_table(n: int, boxsize: float, k_tab, p_tab, growth: float = 1.0, sigma8: float | None = None):
    """The per-k^2 amplitude tpm_ic_zeldovich takes: growth * N^3 sqrt(1/2)
    sqrt(P(k)/L^3) / rk^2 at rk = 2 pi sqrt(k^2), k = rk / L, for integer
    k^2 <= (n/2)^2; with sigma8 the table's P(k) is first scaled to that
    top-hat rms at 8 Mpc/h. growth is D(a_initial)/D(a_final)."""
    p_tab = np.asarray(p_tab, np.float64)
    if sigma8 is not None:
        p_tab = p_tab * (sigma8 / sigma_tophat(k_tab, p_tab)) ** 2
    k2 = np.arange((n // 2) ** 2 + 1, dtype=np.float64)
    rk = 2 * np.pi * np.sqrt(np.maximum(k2, 1.0))
    pk = _pk_interp(np.asarray(k_tab, np.float64), p_tab, rk / boxsize)
    v = growth * float(n) ** 3 * np.sqrt(0.5) * np.sqrt(pk / boxsize ** 3) / rk ** 2
    v[0] = 0.0
    return v.astype(np.float32)
