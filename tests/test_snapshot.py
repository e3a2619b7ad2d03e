"""The reference's snapshot files (tpm_snapshot_*): a file written the
reference's way (tests/golden/snap16.00000, made by the reference's own
write_head and record layout) reads back exactly; files the engine writes
round-trip and parse with the reference's read_head; a snapshot loads into
the engine and gives the plain engine's forces."""
import importlib.util
import os

import numpy as np
import pytest

from lageunha_b200 import engine as E
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))


def _golden_module():
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "golden", "make_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_reads_the_reference_written_snapshot(golden_dir):
    g = _golden_module()
    info, rec = E.read_snapshot(os.path.join(golden_dir, "snap16.00000"))
    s = g.SNAP
    assert info["nx"] == info["ny"] == info["nz"] == s["n"]
    assert info["np_dm"] == s["n"] ** 3 and info["np_sph"] == info["np_star"] == info["np_agn"] == 0
    assert info["ptype"] == 0 and info["record_bytes"] == 32
    for k in ("omep", "omeplam", "wlam0", "wlam1", "amax", "boxsize", "theta", "epsilon"):
        assert info[k] == pytest.approx(s["eps" if k == "epsilon" else k], rel=1e-6), k
    assert info["anow"] == pytest.approx(s["anow"]) and info["astep"] == pytest.approx(s["astep"])
    assert info["stepcount"] == s["stepcount"]
    assert rec.tobytes() == g.snap_records().tobytes()


def test_round_trip(tmp_path):
    g = _golden_module()
    rec = g.snap_records()
    path = str(tmp_path / "snap.00000")
    E.write_snapshot(path, rec, 16, anow=2.25, astep=0.05, omep=0.3, omeplam=0.7, stepcount=12, theta=0.35,
                     epsilon=0.04)
    info, back = E.read_snapshot(path)
    assert back.tobytes() == rec.tobytes()
    assert info["anow"] == 2.25 and info["astep"] == 0.05 and info["stepcount"] == 12
    assert info["omep"] == pytest.approx(0.3) and info["theta"] == pytest.approx(0.35)
    # tree-type records
    trec = np.zeros(rec.shape[0], E.TREEDM_DTYPE)
    for f in ("indx", "x", "y", "z", "vx", "vy", "vz"):
        trec[f] = rec[f]
    trec["next"] = 77
    E.write_snapshot(path, trec, 16)
    info, back = E.read_snapshot(path)
    assert info["ptype"] == 1 and info["record_bytes"] == 40 and back.tobytes() == trec.tobytes()


@pytest.mark.skipif(not O.ref_available(O.VARIANT_A), reason="oracle/_ref not built (reference tree absent)")
def test_reference_reads_engine_written_header(tmp_path):
    g = _golden_module()
    path = str(tmp_path / "snap.00000")
    E.write_snapshot(path, g.snap_records(), 16, anow=4.5, astep=0.01, omep=0.27, omeplam=0.73, wlam0=-0.9,
                     wlam1=0.1, amax=50.0, boxsize=200.0, theta=0.4, epsilon=0.06, stepcount=33)
    h = O.ref_read_head(path)
    want = dict(nx=16, ny=16, nz=16, np_dm=4096, np_sph=0, np_star=0, np_agn=0, ptype=0, omep=0.27, omeplam=0.73,
                wlam0=-0.9, wlam1=0.1, amax=50.0, anow=4.5, astep=0.01, theta=0.4, epsilon=0.06, boxsize=200.0,
                stepcount=33)
    for k, v in want.items():
        assert h[k] == pytest.approx(v, rel=1e-6), (k, h[k], v)


def test_bad_files_fail_loudly(tmp_path):
    with pytest.raises(E.EngineError):
        E.read_snapshot(str(tmp_path / "missing.00000"))
    p = tmp_path / "noheader.00000"
    p.write_bytes(b"define Nx = 16\n" + b"\0" * 64)
    with pytest.raises(E.EngineError):
        E.read_snapshot(str(p))
    g = _golden_module()
    full = open(os.path.join(HERE, "golden", "snap16.00000"), "rb").read()
    cut = tmp_path / "cut.00000"
    cut.write_bytes(full[: len(full) // 2])
    with pytest.raises(E.EngineError):
        E.read_snapshot(str(cut))


@pytest.mark.gpu
def test_snapshot_loads_into_the_engine(golden_dir):
    info, rec = E.read_snapshot(os.path.join(golden_dir, "snap16.00000"))
    n = int(info["nx"])
    pos = O.decode(n, rec["indx"], np.stack([rec["x"], rec["y"], rec["z"]], axis=1))
    fr = O.pm_force(n, pos).astype(np.float64) + O.tree_force(n, pos, variant=O.VARIANT_B, eps=0.05)
    with E.Engine(n, epsilon=float(info["epsilon"]), theta=float(info["theta"])) as eng:
        eng.load_lagrangian(rec)
        eng.compute(E.PART_ALL)
        f = eng.forces()
        v = eng.velocities()
    e = O.rel_err(f, fr)
    assert float(np.sqrt(np.mean(e * e))) <= 1e-3 and np.percentile(e, 99) <= 1e-2
    assert np.array_equal(v, np.stack([rec["vx"], rec["vy"], rec["vz"]], axis=1))
