"""The engine's hand-written pencil FFT and Poisson solve against cuFFT.

The engine replaces FFTW's r2c and c2r (Cosmos/pmmain.c:475,492) around
psolver's Green's function (Cosmos/psolver.c:58-72) with its own Stockham
pencil transforms, the Green's function fused into the z pass. Here cuFFT
(through torch.fft, in FP64) solves the same Poisson problem on the engine's
own deposited density, and the engine's potential must agree within 1e-5 of
the field's largest value, on power-of-two and 2^a 3^b 5^c meshes. cuFFT is
only the check: the engine never calls it.
"""
import numpy as np
import pytest

from lageunha_b200 import engine as E
from lageunha_b200 import ic

pytestmark = pytest.mark.gpu


def _cufft_potential(rho, efold):
    """phi = FFT^-1[ FFT[rho] * (-1/(pi k^2)) exp(-k^2 (pi efold / N)^2) ],
    k = 0 zeroed, unnormalised forward and 1/N^3 in the Green's function:
    torch's default normalisation of irfftn applies that 1/N^3."""
    import torch

    n = rho.shape[0]
    r = torch.from_numpy(rho.astype(np.float64)).cuda()
    spec = torch.fft.rfftn(r, dim=(0, 1, 2))
    w = torch.fft.fftfreq(n, d=1.0 / n, dtype=torch.float64, device="cuda")
    wx = torch.arange(n // 2 + 1, dtype=torch.float64, device="cuda")
    k2 = w[:, None, None] ** 2 + w[None, :, None] ** 2 + wx[None, None, :] ** 2
    g = torch.where(k2 > 0, -1.0 / (np.pi * k2.clamp(min=1.0)) * torch.exp(-k2 * (np.pi * efold / n) ** 2),
                    torch.zeros_like(k2))
    phi = torch.fft.irfftn(spec * g, s=(n, n, n), dim=(0, 1, 2))
    return phi.cpu().numpy()


@pytest.mark.parametrize("n", [64, 96, 120, 256])
def test_potential_matches_cufft(n):
    ps = ic.workload("clustered256", scale=n)
    efold = 0.9
    with E.Engine(n, epsilon=0.05, efold=efold) as eng:
        eng.load_fixed(ps.positions_u32())
        eng.compute(E.PART_PM)
        rho = eng.mesh(E.MESH_DENSITY)
        phi = eng.mesh(E.MESH_POTENTIAL)
    ref = _cufft_potential(rho, efold)
    err = float(np.max(np.abs(phi.astype(np.float64) - ref)))
    scale = float(np.max(np.abs(ref)))
    print(f"n={n}: max |phi_engine - phi_cufft| = {err:.3e} of max |phi| {scale:.3e}")
    assert err <= 1e-5 * scale
