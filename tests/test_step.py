"""The global step around the force evaluation.

CPU: the evolution factors (tpm_evol_factors, host code in the engine
library) against GetEvolFactor of the reference build
(Cosmos/CosmosEvolFactor.c:230-255) through the golden fixture
tests/golden/evolfact.npz and, where oracle/_ref is built, live. Scalars:
bit-exact.

GPU: one tpm_step in KICK status (Cosmos/globalT.c:221-305) against the
sequence it stands for, Hubble drag v *= fact1 (Cosmos/globalT.c:102-110),
kicks v += fact2 F_pm + fact2 F_tree, drift x += v pfact
(Cosmos/stepevolv.c:19-29). Velocities: separate force evaluations differ by
float atomic order only and the kick may fuse multiply-adds, so per particle
within 4 ulp of the velocity plus 1e-5 of fact2 times the force scale;
positions: exact, given the velocities.
"""
import numpy as np
import pytest

from lageunha_b200 import engine as E
from lageunha_b200 import ic
from oracle import oracle as O


def _golden_cases(golden_dir):
    g = np.load(f"{golden_dir}/evolfact.npz")
    return int(g["nx"]), list(g["fields"]), g["cases"], g["factors"]


def test_evol_factors_bit_exact_vs_reference_golden(golden_dir):
    nx, fields, cases, facts = _golden_cases(golden_dir)
    assert len(cases) >= 40
    for row, want in zip(cases, facts):
        omep, omeplam, w0, w1, amax, anow, astep = (float(v) for v in row)
        got = E.evol_factors(E.cosmology(omep, omeplam, w0, w1, amax), nx, anow, astep)
        for k, w in zip(fields, want):
            if k in ("afact", "bfact"):
                continue
            assert np.float32(got[k]) == w, (row, k, got[k], w)


def test_evol_factors_cover_every_branch(golden_dir):
    """The fixture reaches the LCDM, constant-w and w(a) branches of gzDE
    (Cosmos/FLRW.c:38-58), the last one with Simpson (tau < 0.8) and Romberg
    (tau >= 0.8) integration."""
    _, _, cases, _ = _golden_cases(golden_dir)
    w = cases[:, 2:4]
    tau = cases[:, 5] / cases[:, 4]
    lcdm = (w[:, 0] == -1) & (w[:, 1] == 0)
    const = (w[:, 1] == 0) & ~lcdm
    wa = w[:, 1] != 0
    assert lcdm.any() and const.any()
    assert (wa & (tau < 0.8)).any() and (wa & (tau >= 0.8)).any()


@pytest.mark.skipif(not O.ref_available(O.VARIANT_A), reason="oracle/_ref not built (reference tree absent)")
def test_evol_factors_live_reference():
    rng = np.random.default_rng(11)
    for _ in range(24):
        c = E.cosmology(float(rng.uniform(0.2, 0.4)), float(rng.uniform(0.6, 0.8)), float(rng.uniform(-1.2, -0.8)),
                        float(rng.choice([0.0, rng.uniform(-0.3, 0.3)])), float(rng.uniform(20, 60)))
        anow = float(rng.uniform(1.0, c.amax * 0.99))
        astep = float(rng.uniform(0.01, 0.2))
        nx = int(rng.choice([64, 256, 2048]))
        got = E.evol_factors(c, nx, anow, astep)
        want = O.ref_evol_factors(nx, c.omep, c.omeplam, c.wlam0, c.wlam1, c.amax, anow, astep)
        for k in O.EVOL_FIELDS[2:]:
            assert np.float32(got[k]) == want[k], (k, got[k], want[k])


def test_evol_factors_rejects_bad_arguments():
    c = E.cosmology()
    for nx, anow, astep in ((0, 1.0, 0.1), (64, 0.0, 0.1), (64, 1.0, -0.1), (64, float("nan"), 0.1)):
        with pytest.raises(E.EngineError):
            E.evol_factors(c, nx, anow, astep)
    with pytest.raises(E.EngineError):
        E.evol_factors(E.cosmology(omep=0.0), 64, 1.0, 0.1)


def test_evol_factors_limits():
    """A zero step leaves velocities alone (fact1 = 1, fact2 = 0, pfact = 0);
    for LCDM fact1 < 1 (expansion drags peculiar velocities)."""
    c = E.cosmology()
    z = E.evol_factors(c, 64, 5.0, 0.0)
    assert z["fact1"] == 1.0 and z["fact2"] == 0.0 and z["pfact"] == 0.0
    f = E.evol_factors(c, 64, 5.0, 0.05)
    assert 0.0 < f["fact1"] < 1.0 and f["fact2"] > 0.0
    assert np.float32(f["pfact"]) == np.float32(np.float32(0.05) * 64)


@pytest.mark.gpu
@pytest.mark.parametrize("law,stepcount", [("reference", 15), ("gaussian", 3)])
def test_step_matches_drag_kick_drift(law, stepcount):
    n = 32
    ps = ic.workload("clustered256", scale=n)
    pu = ps.positions_u32()
    vel = np.random.default_rng(4).standard_normal((ps.np, 3)).astype(np.float32)
    cosmo = E.cosmology()
    anow, astep = 6.0, 0.05
    ef = E.evol_factors(cosmo, n, anow, astep)
    kw = dict(epsilon=0.05, law=law)
    if law == "gaussian":
        kw.update(rs_split=1.2, rsphere=6.0)
    theta = 0.35 if law == "reference" else 0.3
    with E.Engine(n, theta=theta, **kw) as eng:
        eng.load_fixed(pu, vel)
        eng.compute(E.PART_PM)
        fpm = eng.forces()
        eng.compute(E.PART_TREE)
        ftr = eng.forces()
    with E.Engine(n, theta=0.3, **kw) as eng:
        eng.load_fixed(pu, vel)
        eng.step(cosmo, anow, astep, stepcount)
        v1 = eng.velocities()
        p1 = eng.positions()
        th = eng.params.theta
    # TreeAndPreFoFmain's schedule applies to the reference law only
    assert np.float32(th) == np.float32(theta)
    f1, f2 = np.float32(ef["fact1"]), np.float32(ef["fact2"])
    want = (vel * f1 + f2 * fpm) + f2 * ftr
    scale = float(f2) * (1.0 + np.max(np.abs(fpm + ftr)))
    tol = 4 * np.spacing(np.abs(want)) + 1e-5 * scale
    assert np.all(np.abs(v1 - want) <= tol)
    d = np.rint(np.fmod(v1.astype(np.float64) * float(np.float32(ef["pfact"])) * (2.0 ** 32 / n),
                        2.0 ** 32)).astype(np.int64)
    expect = ((pu.astype(np.int64) + d) % (2 ** 32)).astype(np.uint32)
    assert np.array_equal(p1, expect)


@pytest.mark.gpu
def test_hubble_drag_scales_velocities_exactly():
    n = 16
    ps = ic.workload("plain64", scale=n)
    vel = np.random.default_rng(5).standard_normal((ps.np, 3)).astype(np.float32)
    with E.Engine(n, epsilon=0.05) as eng:
        eng.load_fixed(ps.positions_u32(), vel)
        eng.hubble_drag(0.987654)
        v = eng.velocities()
    assert np.array_equal(v, vel * np.float32(0.987654))


# ---------------------------------------------------------------- PMSTATUS
def test_status_factors_follow_the_reference_selection():
    """tpm_status_factors picks what PM_PULL_AND_PUSH (Cosmos/globalT.c:
    119-127), fda4 (Cosmos/fda4.c:48-62) and TREE_HALF (Cosmos/indT.h:
    98-118) pick: the drag and PM factors by status, PUSH's PM factor divided
    by GetFact1(anow, anow + astep/2) = fact1_push, and the full-step fact2
    for the tree in every status. Host only."""
    c = E.cosmology()
    nx, anow, astep = 64, 3.0, 0.25
    e = E.evol_factors(c, nx, anow, astep)
    f32 = np.float32
    assert E.status_factors(c, nx, anow, astep, E.KICK) == (e["fact1"], e["fact2"], e["fact2"])
    assert E.status_factors(c, nx, anow, astep, E.PULL) == (e["fact1_pull"], e["fact2_pull"], e["fact2"])
    d, p, t = E.status_factors(c, nx, anow, astep, E.PUSH)
    assert d == e["fact1_push"] and t == e["fact2"]
    assert f32(p) == f32(f32(e["fact2_push"]) / f32(e["fact1_push"]))


def _status_case():
    n = 32
    ps = ic.workload("clustered256", scale=n)
    vel = (0.05 * np.random.default_rng(5).standard_normal((ps.np, 3))).astype(np.float32)
    return n, ps, vel


@pytest.mark.gpu
@pytest.mark.skipif(not O.ref_available(O.VARIANT_B), reason="oracle/_ref not built (reference tree absent)")
@pytest.mark.parametrize("status", [E.KICK, E.PULL, E.PUSH])
def test_status_kick_vs_reference_build(status):
    """One status half of the global step against the reference's own
    pmmain and treecorrection run with PMSTATUS set (variant B): the velocity
    change beyond the drag, per particle, within the force bar (rms 1e-3,
    99th percentile 1e-2)."""
    n, ps, vel = _status_case()
    c = E.cosmology()
    anow, astep = 2.0, 0.2
    with E.Engine(n, epsilon=0.05) as eng:
        eng.load_fixed(ps.positions_u32(), vel)
        eng.status_kick(c, anow, astep, status)
        v_eng = eng.velocities()
    v_ref = O.ref_status_kick(n, ps.indx, ps.offset, vel, status, anow, astep)
    drag = np.float32(E.status_factors(c, n, anow, astep, status)[0])
    base = vel * drag
    e = O.rel_err(v_eng.astype(np.float64) - base, v_ref.astype(np.float64) - base)
    assert float(np.sqrt(np.mean(e * e))) <= 1e-3
    assert float(np.percentile(e, 99)) <= 1e-2


@pytest.mark.gpu
@pytest.mark.skipif(not O.ref_available(O.VARIANT_B), reason="oracle/_ref not built (reference tree absent)")
def test_sync_step_is_pull_then_push_then_drift():
    """A synchronisation step (tpm_global_step with sync) is the reference's
    PULL half, then its PUSH half on the same positions, then the drift
    (Cosmos/globalT.c:244-291)."""
    n, ps, vel = _status_case()
    c = E.cosmology()
    anow, astep = 2.0, 0.2
    pu = ps.positions_u32()
    with E.Engine(n, epsilon=0.05) as eng:
        eng.load_fixed(pu, vel)
        eng.global_step(c, anow, astep, 2, sync=True)
        v_eng = eng.velocities()
        p_eng = eng.positions()
    v1 = O.ref_status_kick(n, ps.indx, ps.offset, vel, E.PULL, anow, astep)
    v2 = O.ref_status_kick(n, ps.indx, ps.offset, v1, E.PUSH, anow, astep)
    d1 = np.float32(E.status_factors(c, n, anow, astep, E.PULL)[0])
    d2 = np.float32(E.status_factors(c, n, anow, astep, E.PUSH)[0])
    base = vel * d1 * d2
    e = O.rel_err(v_eng.astype(np.float64) - base, v2.astype(np.float64) - base)
    assert float(np.sqrt(np.mean(e * e))) <= 1e-3
    assert float(np.percentile(e, 99)) <= 1e-2
    pfact = E.evol_factors(c, n, anow, astep)["pfact"]
    dq = np.rint(np.fmod(v_eng.astype(np.float64) * pfact * (2.0 ** 32 / n), 2.0 ** 32)).astype(np.int64)
    assert np.array_equal(p_eng, ((pu.astype(np.int64) + dq) % (2 ** 32)).astype(np.uint32))
