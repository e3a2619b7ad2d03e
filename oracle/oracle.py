"""ctypes front end of the CPU oracle — TEST INFRASTRUCTURE ONLY.

Loads oracle/liboracle.so (the C restatement, tpm_oracle.c) and, where built,
oracle/_ref/libref_{A,B}.so (the reference's own force-path sources compiled
with the single-rank harness ref_shim.c). Only tests/, the smoke check and
bench.py's CPU-baseline leg import this module; the engine never does.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
VARIANT_A, VARIANT_B = 0, 1

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_i64 = ctypes.c_int64
_int = ctypes.c_int
_flt = ctypes.c_float
_dbl = ctypes.c_double

_lib = None
_ref = {}


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/liboracle.so is not built (run `make -C oracle oracle`)")
        L = ctypes.CDLL(path)
        L.or_decode.argtypes = [_int, _i64, _u64p, _f32p, _f64p]
        L.or_tsc_density.argtypes = [_int, _i64, _f64p, _f32p]
        L.or_potential.argtypes = [_int, _i64, _f64p, _flt, _f32p]
        L.or_pm_force.argtypes = [_int, _i64, _f64p, _flt, _f32p]
        L.or_fda4_force.argtypes = [_int, _i64, _f64p, _f32p, _f32p]
        L.or_spline_table.argtypes = [_int, _flt, _f64p, _f64p]
        L.or_tree_force.argtypes = [_int, _i64, _f64p, _flt, _flt, _flt, _int, _f32p]
        L.or_direct_short_force.argtypes = [_int, _i64, _f64p, _flt, _flt, _i64, _i64p, _f64p]
        L.or_ewald_force.argtypes = [_int, _i64, _f64p, _flt, _i64, _i64p, _dbl, _dbl, _int, _f64p]
        for f in ("or_decode",):
            getattr(L, f).restype = None
        _lib = L
    return _lib


def ref_available(variant: int = VARIANT_B) -> bool:
    return os.path.exists(_ref_path(variant))


def _ref_path(variant):
    return os.path.join(HERE, "_ref", "libref_%s.so" % ("A" if variant == VARIANT_A else "B"))


def ref(variant: int = VARIANT_B):
    if variant not in _ref:
        path = _ref_path(variant)
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is not built (needs the reference tree; `make -C oracle ref`)")
        L = ctypes.CDLL(path, mode=ctypes.RTLD_LOCAL)
        L.ref_pm_force.argtypes = [_int, _i64, _u64p, _f32p, _flt, _f32p]
        L.ref_tree_force.argtypes = [_int, _i64, _u64p, _f32p, _flt, _flt, _flt, _f32p]
        L.ref_tsc_density.argtypes = [_int, _i64, _u64p, _f32p, _f32p]
        L.ref_potential.argtypes = [_int, _i64, _u64p, _f32p, _flt, _f32p]
        L.ref_spline_table.argtypes = [_int, _flt, _f64p, _f64p]
        L.ref_evol_factors.argtypes = [_int, _flt, _flt, _flt, _flt, _flt, _flt, _flt, _f32p]
        L.ref_status_kick.argtypes = [_int, _i64, _u64p, _f32p, _f32p] + [_flt] * 11 + [_int]
        L.ref_write_snapshot.argtypes = [ctypes.c_char_p, _int, ctypes.c_int64, ctypes.c_void_p] + [_flt] * 5 + \
            [ctypes.c_double] * 2 + [_flt] * 4 + [_int]
        L.ref_read_head.argtypes = [ctypes.c_char_p, ctypes.c_void_p]
        L.ref_power_spectrum.argtypes = [_int, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                                         ctypes.c_void_p]
        _ref[variant] = L
    return _ref[variant]


_dropin = None


def dropin_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libgotpm_dropin.so"))


def dropin():
    """The engine's legacy-name entry points (lageunha_b200/gotpm/tpm_gotpm.c)
    built against the reference's eunha.h with the harness dropin_shim.c."""
    global _dropin
    if _dropin is None:
        path = os.path.join(HERE, "_ref", "libgotpm_dropin.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is not built (needs the reference tree; `make -C oracle ref`)")
        L = ctypes.CDLL(path, mode=ctypes.RTLD_LOCAL)
        L.dropin_pmmain.argtypes = [_int, _i64, _u64p, _f32p, _f32p, _f32p, _int, _flt, _flt]
        L.dropin_treemain.argtypes = [_int, _i64, _u64p, _f32p, _f32p, _flt, _flt, _int, _flt, _flt]
        _dropin = L
    return _dropin


def dropin_pmmain(n, indx, off, vel, evolfact9, status, efold=0.9, eps=0.05):
    """The drop-in pmmain(SimParameters*, EvolFact): returns (status, velocities)."""
    v = np.array(vel, dtype=np.float32, order="C", copy=True)
    ef = np.ascontiguousarray(evolfact9, dtype=np.float32)
    rc = dropin().dropin_pmmain(n, indx.shape[0], _c(indx, np.uint64), _c(off, np.float32), v, ef, status, efold, eps)
    return rc, v


def dropin_treemain(n, indx, off, vel, fact1, fact2, stepcount, rsphere=4.0, eps=0.05):
    """The drop-in TreeMain(SimParameters*, DeterminedEvolFact*)."""
    v = np.array(vel, dtype=np.float32, order="C", copy=True)
    rc = dropin().dropin_treemain(n, indx.shape[0], _c(indx, np.uint64), _c(off, np.float32), v, fact1, fact2,
                                  stepcount, rsphere, eps)
    return rc, v


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


# ---------------------------------------------------------------- restatement
def decode(n, indx, off):
    np_ = indx.shape[0]
    out = np.empty((np_, 3), np.float64)
    lib().or_decode(n, np_, _c(indx, np.uint64), _c(off, np.float32), out)
    return out


def tsc_density(n, pos):
    out = np.empty(n ** 3, np.float32)
    lib().or_tsc_density(n, pos.shape[0], _c(pos, np.float64), out)
    return out.reshape(n, n, n)


def potential(n, pos, efold=0.9):
    out = np.empty(n ** 3, np.float32)
    lib().or_potential(n, pos.shape[0], _c(pos, np.float64), efold, out)
    return out.reshape(n, n, n)


def pm_force(n, pos, efold=0.9):
    out = np.empty((pos.shape[0], 3), np.float32)
    lib().or_pm_force(n, pos.shape[0], _c(pos, np.float64), efold, out)
    return out


def fda4_force(n, pos, phi):
    out = np.empty((pos.shape[0], 3), np.float32)
    lib().or_fda4_force(n, pos.shape[0], _c(pos, np.float64), _c(phi, np.float32), out)
    return out


def spline_table(n, eps):
    d = np.empty((4096, 3), np.float64)
    s = np.empty((4096, 3), np.float64)
    lib().or_spline_table(n, eps, d, s)
    return d, s


def tree_force(n, pos, theta=0.3, rsphere=4.0, eps=0.05, variant=VARIANT_B):
    out = np.empty((pos.shape[0], 3), np.float32)
    lib().or_tree_force(n, pos.shape[0], _c(pos, np.float64), theta, rsphere, eps, variant, out)
    return out


def direct_short_force(n, pos, targets, rsphere=4.0, eps=0.05):
    t = _c(targets, np.int64)
    out = np.empty((t.shape[0], 3), np.float64)
    lib().or_direct_short_force(n, pos.shape[0], _c(pos, np.float64), rsphere, eps, t.shape[0], t, out)
    return out


def ewald_force(n, pos, targets, eps=0.05, rcut=None, alpha=None, kmax=None):
    """FP64 periodic Ewald force (reference units) at the target indices."""
    rcut = rcut if rcut is not None else 0.49 * n
    alpha = alpha if alpha is not None else 3.6 / rcut
    if kmax is None:
        kmax = int(np.ceil(2 * alpha * 3.6 * n / (2 * np.pi)))
    t = _c(targets, np.int64)
    out = np.empty((t.shape[0], 3), np.float64)
    lib().or_ewald_force(n, pos.shape[0], _c(pos, np.float64), eps, t.shape[0], t, rcut, alpha, kmax, out)
    return out


# ------------------------------------------------------- reference (oracle/_ref)
def ref_pm_force(n, indx, off, efold=0.9):
    out = np.empty((indx.shape[0], 3), np.float32)
    ref(VARIANT_A).ref_pm_force(n, indx.shape[0], _c(indx, np.uint64), _c(off, np.float32), efold, out)
    return out


def ref_tree_force(n, indx, off, theta=0.3, rsphere=4.0, eps=0.05, variant=VARIANT_B):
    out = np.empty((indx.shape[0], 3), np.float32)
    ref(variant).ref_tree_force(n, indx.shape[0], _c(indx, np.uint64), _c(off, np.float32), theta,
                                rsphere, eps, out)
    return out


def ref_status_kick(n, indx, off, vel, status, anow, astep, cosmo=(0.26, 0.74, -1.0, 0.0, 48.0), efold=0.9,
                    theta=0.3, rsphere=4.0, eps=0.05, variant=VARIANT_B):
    """One PMSTATUS half of the reference's global step (drag, pmmain, tree
    kick with the full-step fact2): returns the new velocities."""
    v = np.array(vel, dtype=np.float32, order="C", copy=True)
    ref(variant).ref_status_kick(n, indx.shape[0], _c(indx, np.uint64), _c(off, np.float32), v, efold, theta,
                                 rsphere, eps, *[float(c) for c in cosmo], anow, astep, status)
    return v


def ref_tsc_density(n, indx, off):
    out = np.empty(n ** 3, np.float32)
    ref(VARIANT_A).ref_tsc_density(n, indx.shape[0], _c(indx, np.uint64), _c(off, np.float32), out)
    return out.reshape(n, n, n)


def ref_potential(n, indx, off, efold=0.9):
    out = np.empty(n ** 3, np.float32)
    ref(VARIANT_A).ref_potential(n, indx.shape[0], _c(indx, np.uint64), _c(off, np.float32), efold, out)
    return out.reshape(n, n, n)


def ref_spline_table(n, eps):
    d = np.empty((4096, 3), np.float64)
    s = np.empty((4096, 3), np.float64)
    ref(VARIANT_A).ref_spline_table(n, eps, d, s)
    return d, s


EVOL_FIELDS = ("afact", "bfact", "pfact", "fact1", "fact2", "fact1_push", "fact2_push", "fact1_pull", "fact2_pull")


def ref_evol_factors(n, omep, omeplam, wlam0, wlam1, amax, anow, astep):
    out = np.zeros(9, np.float32)
    ref(VARIANT_A).ref_evol_factors(n, omep, omeplam, wlam0, wlam1, amax, anow, astep, out)
    return dict(zip(EVOL_FIELDS, out))


SNAPSHOT_FIELDS = ("nx", "ny", "nz", "np_dm", "np_sph", "np_star", "np_agn", "ptype", "omep", "omeplam", "wlam0",
                   "wlam1", "amax", "anow", "astep", "theta", "epsilon", "rsphere", "boxsize", "stepcount")


def ref_write_snapshot(path, n, records, omep=0.26, omeplam=0.74, wlam0=-1.0, wlam1=0.0, amax=48.0, anow=1.0,
                       astep=0.02, boxsize=100.0, theta=0.3, eps=0.05, rsphere=4.0, stepcount=0):
    """One rank's GOTPM snapshot as the reference's jwrite writes it."""
    rec = np.ascontiguousarray(records)
    rc = ref(VARIANT_A).ref_write_snapshot(path.encode(), n, rec.shape[0], rec.ctypes.data, omep, omeplam, wlam0,
                                           wlam1, amax, anow, astep, boxsize, theta, eps, rsphere, stepcount)
    if rc != rec.dtype.itemsize:
        raise RuntimeError(f"reference record size {rc} != {rec.dtype.itemsize}")


def ref_read_head(path):
    """The header of a snapshot as the reference's read_head parses it."""
    out = np.zeros(len(SNAPSHOT_FIELDS), np.float64)
    if ref(VARIANT_A).ref_read_head(path.encode(), out.ctypes.data) != 0:
        raise RuntimeError(f"cannot read {path}")
    return dict(zip(SNAPSHOT_FIELDS, out))


def ref_power_spectrum(n, indx, off, boxsize):
    """The reference's CorrMeasure (Cosmos/Correlation.c) on one pmmain of
    the particles: {"pk": P(k) for bins 0..N/2-1, "cor": xi at 0..N/2-1 cells,
    "sigma8", "slope"}, parsed from the pmevol.map it writes (7 significant
    digits)."""
    import os
    import tempfile
    idx = np.ascontiguousarray(indx, np.uint64)
    o = np.ascontiguousarray(off, np.float32)
    force = np.zeros((idx.shape[0], 3), np.float32)
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as d:
        os.chdir(d)
        try:
            ref(VARIANT_A).ref_power_spectrum(n, idx.shape[0], idx.ctypes.data, o.ctypes.data, boxsize,
                                              force.ctypes.data)
            lines = open("pmevol.map").read().split("\n")
        finally:
            os.chdir(cwd)
    anow, s8, slope = (float(x) for x in lines[0].split())
    rows = [l.split() for l in lines[1:] if l.strip()]
    pk = np.array([float(r[2]) for r in rows])
    cor = np.array([float(r[3]) for r in rows])
    return {"pk": pk, "cor": cor, "sigma8": s8, "slope": slope}


def fof_labels(n, pos, link, min_members):
    """Friends-of-friends groups (FoF/fof.c:217-290: particles linked when
    their distance is <= link; the groups are the connected components of
    that relation) in FP64 with periodic minimum images: label = smallest
    particle index of the group if it has >= min_members particles, else -1."""
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components
    from scipy.spatial import cKDTree
    p = np.mod(np.asarray(pos, np.float64), n)
    pairs = cKDTree(p, boxsize=float(n)).query_pairs(r=link, output_type="ndarray")
    m = p.shape[0]
    g = coo_matrix((np.ones(len(pairs)), (pairs[:, 0], pairs[:, 1])), shape=(m, m))
    _, comp = connected_components(g, directed=False)
    size = np.bincount(comp)
    first = np.full(comp.max() + 1, m, np.int64)
    np.minimum.at(first, comp, np.arange(m))
    lab = np.where(size[comp] >= min_members, first[comp], -1)
    return lab.astype(np.int64), int(np.sum(size >= min_members))


def rel_err(f, fref):
    """Per-particle |f - fref| / |fref|."""
    num = np.linalg.norm(np.asarray(f, np.float64) - np.asarray(fref, np.float64), axis=1)
    den = np.linalg.norm(np.asarray(fref, np.float64), axis=1)
    return num / np.maximum(den, 1e-300)


# ------------------------------------------------------------- sort oracle
AXIS_BITS = 13


def cell_bits(n):
    c = 0
    while (1 << c) < n:
        c += 1
    return max(c, 3)


def _spread3(v):
    x = v.astype(np.uint64) & np.uint64(0x1FFFFF)
    x = (x | (x << np.uint64(32))) & np.uint64(0x1F00000000FFFF)
    x = (x | (x << np.uint64(16))) & np.uint64(0x1F0000FF0000FF)
    x = (x | (x << np.uint64(8))) & np.uint64(0x100F00F00F00F00F)
    x = (x | (x << np.uint64(4))) & np.uint64(0x10C30C30C30C30C3)
    x = (x | (x << np.uint64(2))) & np.uint64(0x1249249249249249)
    return x


def morton_keys(pos_u32, n):
    """39-bit Morton keys of uint32 fixed-point positions: per axis the
    quantised coordinate q = floor(x_cells * 2^(13 - C)), C = ceil(log2 N)."""
    sub = AXIS_BITS - cell_bits(n)
    p = np.asarray(pos_u32, dtype=np.uint64)
    q = (p * np.uint64(n)) >> np.uint64(32 - sub)
    return _spread3(q[:, 0]) | (_spread3(q[:, 1]) << np.uint64(1)) | (_spread3(q[:, 2]) << np.uint64(2))


def sort_order(keys):
    """The engine's permutation: stable argsort (ties keep input order)."""
    return np.argsort(keys, kind="stable")


# ---------------------------------------------------------------- initial conditions
def _ran3_stream(idum):
    """Numerical Recipes ran3 (Cosmos/CosmosIC/nr.c:317-355) as a generator of
    the integer states mj; ran3's float is float32(mj * 1e-9)."""
    mbig, mseed = 1000000000, 161803398
    ma = [0] * 56
    mj = (mseed - abs(idum)) % mbig
    ma[55] = mj
    mk = 1
    for i in range(1, 55):
        ii = (21 * i) % 55
        ma[ii] = mk
        mk = mj - mk
        if mk < 0:
            mk += mbig
        mj = ma[ii]
    for _ in range(4):
        for i in range(1, 56):
            ma[i] -= ma[1 + (i + 30) % 55]
            if ma[i] < 0:
                ma[i] += mbig
    inext, inextp = 0, 31
    while True:
        inext = 1 if inext + 1 == 56 else inext + 1
        inextp = 1 if inextp + 1 == 56 else inextp + 1
        mj = ma[inext] - ma[inextp]
        if mj < 0:
            mj += mbig
        ma[inext] = mj
        yield mj


def gasdev_pairs(idum, count):
    """The first `count` accepted pairs of gasdev (nr.c:361-384) on ran3, in
    the order gasdev returns them (v2*fac, v1*fac), with the C float and
    double rounding of each operation. A restatement for small counts."""
    f32 = np.float32
    st = _ran3_stream(idum)
    out = np.empty((count, 2), np.float32)
    k = 0
    while k < count:
        v1 = f32(2.0 * float(f32(next(st) * (1.0 / 1e9))) - 1.0)
        v2 = f32(2.0 * float(f32(next(st) * (1.0 / 1e9))) - 1.0)
        rsq = f32(f32(v1 * v1) + f32(v2 * v2))
        if rsq >= 1.0 or rsq == 0.0:
            continue
        fac = f32(np.sqrt(-2.0 * np.log(float(rsq)) / float(rsq)))
        out[k] = (f32(v2 * fac), f32(v1 * fac))
        k += 1
    return out


def ref_ic_noise(n, iseed, velpot=None):
    """The reference's noise spectrum for one rank (ref_shim.c ref_ic_noise:
    PMSeedForce's mode loop and conjugate completion on the reference's own
    gasdev/ran3): complex64 [z][y][kx]."""
    den = np.zeros((n, n, 2 * (n // 2 + 1)), np.float32)
    vp = None if velpot is None else np.ascontiguousarray(velpot, np.float32)
    ref(VARIANT_A).ref_ic_noise(ctypes.c_int(n), ctypes.c_long(iseed),
                                None if vp is None else vp.ctypes.data_as(ctypes.c_void_p),
                                den.ctypes.data_as(ctypes.c_void_p))
    return den.view(np.complex64)


def ref_zeldovich(n, den, fnl=0.0, gnl=0.0):
    """The reference's Zeldovich (Cosmos/CosmosIC/Zeldovich.c) on a noise
    spectrum: (fx, fy, fz) displacement fields as float32 [z][y][x]."""
    d = np.ascontiguousarray(den, np.complex64).view(np.float32).reshape(n, n, 2 * (n // 2 + 1)).copy()
    f = [np.zeros_like(d) for _ in range(3)]
    ref(VARIANT_A).ref_zeldovich(ctypes.c_int(n), ctypes.c_float(fnl), ctypes.c_float(gnl),
                                 d.ctypes.data_as(ctypes.c_void_p), *[a.ctypes.data_as(ctypes.c_void_p) for a in f])
    return tuple(a[:, :, :n] for a in f)


def ref_two_lpt(n, den, amp1, amp2, vamp1, vamp2, fnl=0.0, gnl=0.0, boxsize=100.0, omep=0.3, amax=50.0,
                growth=0.02):
    """The reference's second-order initial conditions for one rank (TwoLPT.c
    with selfdiffphi) on a noise spectrum: (vel, off), each (3, n^3) float32
    in lattice order z, y, x."""
    d = np.ascontiguousarray(den, np.complex64).view(np.float32).reshape(-1).copy()
    vel = np.zeros((3, n ** 3), np.float32)
    off = np.zeros((3, n ** 3), np.float32)
    f = ctypes.c_float
    ref(VARIANT_A).ref_two_lpt(ctypes.c_int(n), d.ctypes.data_as(ctypes.c_void_p), f(amp1), f(amp2), f(vamp1),
                               f(vamp2), f(fnl), f(gnl), f(boxsize), f(omep), f(amax), f(growth),
                               vel.ctypes.data_as(ctypes.c_void_p), off.ctypes.data_as(ctypes.c_void_p))
    return vel, off
