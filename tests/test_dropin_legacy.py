"""The legacy-name boundary: pmmain, treecorrection and TreeMain with the
reference's own signatures (lageunha_b200/gotpm/tpm_gotpm.c), compiled
against the reference's eunha.h and linked with the engine library
(oracle/_ref/libgotpm_dropin.so, made by oracle/Makefile).

The harness fills a one-rank SimParameters and the reference's particle
records as the reference's own harness does, then runs one status half of
the global step the way globalT.c does it (Cosmos/globalT.c:113-134,
85-87): the Hubble drag, pmmain, then TreeMain with the full-step fact2. The
velocities are compared with the reference build's (variant B) on the same
particles and factors: the change beyond the drag within the force bar, rms
relative error <= 1e-3 and 99th percentile <= 1e-2.
"""
import numpy as np
import pytest

from lageunha_b200 import engine as E
from lageunha_b200 import ic
from oracle import oracle as O

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (O.dropin_available() and O.ref_available(O.VARIANT_B)),
                                 reason="oracle/_ref not built (reference tree absent)")]

FIELDS = ("afact", "bfact", "pfact", "fact1", "fact2", "fact1_push", "fact2_push", "fact1_pull", "fact2_pull")


@pytest.mark.parametrize("status", [E.KICK, E.PULL, E.PUSH])
def test_legacy_pmmain_and_treemain_vs_reference_build(status):
    n = 32
    ps = ic.workload("clustered256", scale=n)
    vel = (0.05 * np.random.default_rng(5).standard_normal((ps.np, 3))).astype(np.float32)
    c = E.cosmology()
    anow, astep = 2.0, 0.2
    ef = E.evol_factors(c, n, anow, astep)
    drag = np.float32(E.status_factors(c, n, anow, astep, status)[0])
    v0 = vel * drag
    rc, v1 = O.dropin_pmmain(n, ps.indx, ps.offset, v0, [ef[k] for k in FIELDS], status)
    assert rc == 0
    rc, v2 = O.dropin_treemain(n, ps.indx, ps.offset, v1, ef["fact1"], ef["fact2"], stepcount=2)
    assert rc == 0
    v_ref = O.ref_status_kick(n, ps.indx, ps.offset, vel, status, anow, astep)
    e = O.rel_err(v2.astype(np.float64) - v0, v_ref.astype(np.float64) - v0)
    rms, p99 = float(np.sqrt(np.mean(e * e))), float(np.percentile(e, 99))
    print(f"legacy pmmain + TreeMain, status {status}: rms {rms:.3e} p99 {p99:.3e}")
    assert rms <= 1e-3 and p99 <= 1e-2


def test_legacy_treemain_follows_the_theta_schedule():
    """TreeMain sets the opening angle from the step count before the tree
    correction (Cosmos/Treemain.c:598-601): at step 30 it walks with 0.4."""
    n = 32
    ps = ic.workload("clustered256", scale=n)
    zero = np.zeros((ps.np, 3), np.float32)
    rc, v = O.dropin_treemain(n, ps.indx, ps.offset, zero, 1.0, 1.0, stepcount=30)
    assert rc == 0
    pos = O.decode(n, ps.indx, ps.offset)
    ft = O.tree_force(n, pos, theta=0.4, variant=O.VARIANT_B, eps=0.05)
    ft = ft.astype(np.float64)
    scale = float(np.sqrt(np.mean(np.sum(ft * ft, axis=1))))
    d = np.linalg.norm(v.astype(np.float64) - ft, axis=1) / scale
    assert float(np.sqrt(np.mean(d * d))) <= 1e-3
