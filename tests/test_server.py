"""The request loop (tpm_server_*): continuous batching of force and step
requests.

Each request runs the plain engine's kernels on its own context, so a
request's result is the same whether it runs alone or among others: the
only difference allowed is the order of float atomic adds in the mass
assignment. Stated tolerance: forces and velocities within 1e-5 of their
scale per particle (one evaluation) and 1e-4 after several steps; positions
within 1e-4 cells.
"""
import numpy as np
import pytest

from lageunha_b200 import engine as E
from lageunha_b200 import ic

pytestmark = pytest.mark.gpu

KW = dict(epsilon=0.05, law="gaussian", rs_split=1.2, rsphere=6.0, theta=0.3)


def _box(i, nl, ng):
    return ic.lattice_box(nl, ng, 7000 + i, -2.0, 1.0, 100.0, vel_factor=0.5)


def _close(a, b, tol):
    return np.max(np.abs(a - b)) <= tol * (1.0 + np.max(np.abs(b)))


def _pos_close(pa, pb, n, tol_cells=1e-4):
    d = (pa.astype(np.int64) - pb.astype(np.int64) + 2 ** 31) % 2 ** 32 - 2 ** 31
    return np.max(np.abs(d)) * n / 2.0 ** 32 <= tol_cells


def _outs(b):
    return (np.empty((b.np, 3), np.uint32), np.empty((b.np, 3), np.float32), np.empty((b.np, 3), np.float32))


def test_force_request_matches_plain_engine():
    b = _box(0, 40, 40)
    with E.Engine(b.n_mesh, **KW) as eng:
        eng.load_fixed(b.pos, b.vel)
        eng.compute(E.PART_ALL)
        want = eng.forces()
    po, vo, fo = _outs(b)
    with E.Server(hbm_cap_bytes=8 * 10 ** 9) as srv:
        rid = srv.submit(b.pos, b.vel, n_mesh=b.n_mesh, force_out=fo, pos_out=po, vel_out=vo, **KW)
        srv.wait(rid)
        inf = srv.info(rid)
        assert inf.state == E.REQ_DONE and inf.status == 0
        assert inf.t_submit <= inf.t_admit <= inf.t_done
    assert _close(fo, want, 1e-5)
    assert np.array_equal(po, b.pos) and np.array_equal(vo, b.vel)


def test_step_request_matches_plain_steps():
    b = _box(1, 36, 36)
    cosmo = E.cosmology()
    anow, astep, nsteps = 5.0, 0.05, 3
    with E.Engine(b.n_mesh, **KW) as eng:
        eng.load_fixed(b.pos, b.vel)
        for s in range(nsteps):
            eng.step(cosmo, anow + s * astep, astep, s)
        pw, vw = eng.positions(), eng.velocities()
    po, vo, fo = _outs(b)
    with E.Server(hbm_cap_bytes=8 * 10 ** 9) as srv:
        rid = srv.submit(b.pos, b.vel, n_mesh=b.n_mesh, nsteps=nsteps, anow=anow, astep=astep, cosmo=cosmo,
                         pos_out=po, vel_out=vo, **KW)
        srv.wait(rid)
    assert _close(vo, vw, 1e-4)
    assert _pos_close(po, pw, b.n_mesh)


def test_result_same_alone_and_in_the_mix():
    target = _box(2, 40, 40)
    cosmo = E.cosmology()
    args = dict(n_mesh=target.n_mesh, nsteps=4, anow=3.0, astep=0.05, cosmo=cosmo, **KW)
    alone = _outs(target)
    with E.Server(hbm_cap_bytes=20 * 10 ** 9) as srv:
        srv.wait(srv.submit(target.pos, target.vel, pos_out=alone[0], vel_out=alone[1], **args))
    others = [_box(10 + i, nl, ic.fft_friendly(nl)) for i, nl in enumerate((32, 48, 64, 45, 56, 72, 36, 50))]
    mixed = _outs(target)
    other_out = [_outs(b) for b in others]
    with E.Server(hbm_cap_bytes=20 * 10 ** 9, max_active=6) as srv:
        ids = []
        for i, b in enumerate(others):
            ids.append(srv.submit(b.pos, b.vel, n_mesh=b.n_mesh, nsteps=1 + i % 5, anow=2.0 + i, astep=0.05,
                                  cosmo=cosmo, pos_out=other_out[i][0], vel_out=other_out[i][1],
                                  force_out=other_out[i][2], **KW))
            if i == 3:
                tid = srv.submit(target.pos, target.vel, pos_out=mixed[0], vel_out=mixed[1], **args)
        srv.wait(-1)
        for rid in ids + [tid]:
            inf = srv.info(rid)
            assert inf.state == E.REQ_DONE and inf.status == 0, rid
        st = srv.stats()
        assert st["done"] == len(others) + 1 and st["failed"] == 0
        assert st["peak_active"] >= 2  # requests overlapped
    assert _close(mixed[1], alone[1], 1e-4)
    assert _pos_close(mixed[0], alone[0], target.n_mesh)


def test_admission_respects_the_memory_cap():
    boxes = [_box(20 + i, nl, ic.fft_friendly(nl)) for i, nl in enumerate((48, 40, 56, 44, 52, 36))]
    need = max(E.estimate_bytes(b.n_mesh, b.np) for b in boxes)
    cap = int(2.2 * need)
    with E.Server(hbm_cap_bytes=cap) as srv:
        ids = [srv.submit(b.pos, b.vel, n_mesh=b.n_mesh, nsteps=2, anow=4.0, astep=0.05, **KW) for b in boxes]
        srv.wait(-1)
        st = srv.stats()
        for rid in ids:
            assert srv.info(rid).state == E.REQ_DONE
    assert st["peak_bytes"] <= cap
    assert st["peak_active"] <= 2
    assert st["deferred_admissions"] > 0


def test_rejects_requests_above_the_cap():
    b = _box(30, 32, 32)
    with E.Server(hbm_cap_bytes=10 ** 6) as srv:
        with pytest.raises(E.EngineError):
            srv.submit(b.pos, b.vel, n_mesh=b.n_mesh, **KW)
        with pytest.raises(E.EngineError):
            srv.submit(b.pos, b.vel, n_mesh=8, **KW)  # mesh below the minimum


def test_arena_memory_is_reused_across_mesh_sizes():
    """Requests of different meshes, one after another under a cap that holds
    about two contexts: idle contexts are evicted and their buffers go back to
    the server's arena, which the next contexts draw from. The arena claims at
    most one growth block beyond what was reserved up front, and the last
    request's forces are the plain engine's."""
    boxes = [_box(40 + i, nl, ic.fft_friendly(nl)) for i, nl in enumerate((48, 40, 56, 44, 52, 36, 60))]
    need = max(E.estimate_bytes(b.n_mesh, b.np) for b in boxes)
    cap = int(2.5 * need)
    last = boxes[-1]
    with E.Engine(last.n_mesh, **KW) as eng:
        eng.load_fixed(last.pos, last.vel)
        eng.compute(E.PART_ALL)
        want = eng.forces()
    fo = np.empty((last.np, 3), np.float32)
    with E.Server(hbm_cap_bytes=cap, reserve_bytes=cap) as srv:
        assert srv.stats()["arena_bytes"] >= cap
        for b in boxes[:-1]:
            srv.wait(srv.submit(b.pos, b.vel, n_mesh=b.n_mesh, nsteps=1, anow=4.0, astep=0.05, **KW))
        srv.wait(srv.submit(last.pos, last.vel, n_mesh=last.n_mesh, force_out=fo, **KW))
        st = srv.stats()
    assert st["done"] == len(boxes) and st["failed"] == 0
    assert st["contexts_evicted"] > 0
    assert st["arena_bytes"] <= cap + (1 << 30)  # at most one 1 GiB growth block beyond the reserve
    assert _close(fo, want, 1e-5)


def test_reserve_above_the_cap_is_refused():
    with E.Server(hbm_cap_bytes=10 ** 9) as srv:
        with pytest.raises(E.EngineError):
            srv.reserve(2 * 10 ** 9)
