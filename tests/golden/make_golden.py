"""Generate the golden fixtures of the force path from the reference itself.

The reference's own force-path sources (Cosmos/pmmain.c, psolver.c, fda4.c,
treecorrection.c, BasicCell.c, OST/ost.ver2.c, Model4TreeForce.c) compiled by
oracle/Makefile into oracle/_ref/libref_{A,B}.so are run on small seeded
particle sets, and their outputs are stored here so that the oracle's C
restatement (and through it the engine) is pinned to the reference on hosts
where the reference tree is absent.

    make -C oracle ref && python tests/golden/make_golden.py

Cases (all seeded, lageunha_b200.ic):
  plain16      16^3 Zel'dovich lattice (the plain64 statistics at N=16):
               TSC density, potential, PM force, tree force A and B,
               the short-range table, FP64 Ewald on 64 targets
  clustered32  32^3 with one planted Plummer sphere: PM and tree forces
               (A and B) on a 4096-particle subsample of targets
  sparse32     300 particles at random in a 32^3 box: tree forces A and B
               (buckets with fewer than 16 sources: DirectSummation)
  evolfact     GetEvolFactor (Cosmos/CosmosEvolFactor.c:230-255) over a grid
               of cosmologies (LCDM, constant w, w(a) with w1 != 0), expansion
               factors and steps

    python tests/golden/make_golden.py evolfact     # one case only
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from lageunha_b200 import ic  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


# (omep, omeplam, wlam0, wlam1, amax)
EVOL_COSMOLOGIES = ((0.26, 0.74, -1.0, 0.0, 48.0), (0.26, 0.74, -0.9, 0.0, 48.0), (0.26, 0.74, -0.9, 0.2, 48.0),
                    (0.3, 0.7, -1.1, -0.3, 31.0))
EVOL_ANOW = (1.0, 3.0, 10.0, 24.9, 30.0, 40.0, 47.95)
EVOL_ASTEP = (0.025, 0.1)
EVOL_NX = 128


def evolfact():
    rows, facts = [], []
    for c in EVOL_COSMOLOGIES:
        for anow in EVOL_ANOW:
            if anow >= c[4]:
                continue
            for astep in EVOL_ASTEP:
                r = O.ref_evol_factors(EVOL_NX, *c, anow, astep)
                rows.append((*c, anow, astep))
                facts.append([r[k] for k in O.EVOL_FIELDS])
    np.savez_compressed(os.path.join(OUT, "evolfact.npz"), nx=EVOL_NX, fields=np.array(O.EVOL_FIELDS),
                        cases=np.array(rows, np.float32), factors=np.array(facts, np.float32))


def main(which=None):
    if not (O.ref_available(O.VARIANT_A) and O.ref_available(O.VARIANT_B)):
        raise SystemExit("oracle/_ref is not built: run `make -C oracle ref` where the reference tree exists")
    if which == "evolfact":
        evolfact()
        return
    if which is not None:
        raise SystemExit(f"unknown case {which}")
    evolfact()

    # ---- plain16
    n = 16
    ps = ic.workload("plain64", scale=n)
    d = dict(n=n, indx=ps.indx, offset=ps.offset)
    d["density"] = O.ref_tsc_density(n, ps.indx, ps.offset)
    d["potential"] = O.ref_potential(n, ps.indx, ps.offset, 0.9)
    d["pm_force"] = O.ref_pm_force(n, ps.indx, ps.offset, 0.9)
    d["tree_force_A"] = O.ref_tree_force(n, ps.indx, ps.offset, variant=O.VARIANT_A, eps=0.05)
    d["tree_force_B"] = O.ref_tree_force(n, ps.indx, ps.offset, variant=O.VARIANT_B, eps=0.05)
    diff, slope = O.ref_spline_table(n, 0.05)
    d["spline_diff"], d["spline_slope"] = diff, slope
    tg = np.arange(0, ps.np, ps.np // 64, dtype=np.int64)[:64]
    d["ewald_targets"] = tg
    d["ewald_force"] = O.ewald_force(n, O.decode(n, ps.indx, ps.offset), tg, eps=0.05)
    np.savez_compressed(os.path.join(OUT, "plain16.npz"), **d)

    # ---- clustered32
    n = 32
    ps = ic.workload("clustered256", scale=n)
    rng = np.random.Generator(np.random.PCG64(32))
    sub = np.sort(rng.choice(ps.np, 4096, replace=False)).astype(np.int64)
    fpm = O.ref_pm_force(n, ps.indx, ps.offset, 0.9)
    fa = O.ref_tree_force(n, ps.indx, ps.offset, variant=O.VARIANT_A, eps=0.05)
    fb = O.ref_tree_force(n, ps.indx, ps.offset, variant=O.VARIANT_B, eps=0.05)
    np.savez_compressed(os.path.join(OUT, "clustered32.npz"), n=n, indx=ps.indx, offset=ps.offset, sub=sub,
                        pm_force=fpm[sub], tree_force_A=fa[sub], tree_force_B=fb[sub])

    # ---- sparse32
    n = 32
    rng = np.random.Generator(np.random.PCG64(5))
    indx = np.sort(rng.choice(n ** 3, 300, replace=False)).astype(np.uint64)
    off = (rng.random((300, 3)) * n - n / 2).astype(np.float32)
    fa = O.ref_tree_force(n, indx, off, variant=O.VARIANT_A, eps=0.05)
    fb = O.ref_tree_force(n, indx, off, variant=O.VARIANT_B, eps=0.05)
    np.savez_compressed(os.path.join(OUT, "sparse32.npz"), n=n, indx=indx, offset=off, tree_force_A=fa,
                        tree_force_B=fb)
    for f in ("plain16.npz", "clustered32.npz", "sparse32.npz", "evolfact.npz"):
        print(f, os.path.getsize(os.path.join(OUT, f)), "bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else None)
