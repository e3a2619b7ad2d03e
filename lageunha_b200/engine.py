"""Python front end of the B200 TreePM force engine (ctypes over the C ABI of
include/tpm_engine.h, implemented by lageunha_b200/libtpm_engine.so).

The engine replaces the GOTPM force evaluation of kjhan0606/LagEunha:
``pmmain`` (Cosmos/pmmain.c:390), ``treecorrection``
(Cosmos/treecorrection.c:225) and ``TreeMain`` (Cosmos/Treemain.c:578). The
methods of the same names here take the reference's particle records (numpy
structured arrays with the GOTPM layouts of eunha.h:390-412) and add
``fact2 * F`` to their velocities, as the reference does.

There is no CPU fallback: constructing an Engine without the built library
or without a CUDA device raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtpm_engine.so")

TPM_OK = 0
TPM_LAW_REFERENCE = 0
TPM_LAW_GAUSSIAN = 1
PART_PM, PART_TREE, PART_ALL = 1, 2, 3
MEM_HOST, MEM_DEVICE = 0, 1
MESH_DENSITY, MESH_POTENTIAL = 0, 1
STAGES = ("sort", "deposit", "fft", "fda4", "tree_build", "tree_walk", "finish")

# GOTPM record layouts (eunha.h:390-412 with GOTPM defined): the flag byte is
# the top byte of the 64-bit index (eunha.h:1176-1212).
DM_DTYPE = np.dtype([("indx", "<u8"), ("x", "<f4"), ("y", "<f4"), ("z", "<f4"),
                     ("vx", "<f4"), ("vy", "<f4"), ("vz", "<f4")])
TREEDM_DTYPE = np.dtype([("next", "<u8"), ("indx", "<u8"), ("x", "<f4"), ("y", "<f4"), ("z", "<f4"),
                         ("vx", "<f4"), ("vy", "<f4"), ("vz", "<f4")])
assert DM_DTYPE.itemsize == 32 and TREEDM_DTYPE.itemsize == 40


class TpmParams(ctypes.Structure):
    _fields_ = [("n_mesh", ctypes.c_int32), ("law", ctypes.c_int32), ("theta", ctypes.c_float),
                ("rsphere", ctypes.c_float), ("epsilon", ctypes.c_float), ("efold", ctypes.c_float),
                ("rs_split", ctypes.c_float), ("particle_mass", ctypes.c_float)]


class TpmCosmology(ctypes.Structure):
    _fields_ = [("omep", ctypes.c_float), ("omeplam", ctypes.c_float), ("wlam0", ctypes.c_float),
                ("wlam1", ctypes.c_float), ("amax", ctypes.c_float)]


class TpmEvolFact(ctypes.Structure):
    _fields_ = [(k, ctypes.c_float) for k in ("afact", "bfact", "pfact", "fact1", "fact2", "fact1_push",
                                              "fact2_push", "fact1_pull", "fact2_pull")]


# WMAP5-like defaults of the reference's parameter file (Params/header.c:122-139)
def cosmology(omep=0.26, omeplam=0.74, wlam0=-1.0, wlam1=0.0, amax=48.0) -> TpmCosmology:
    return TpmCosmology(omep, omeplam, wlam0, wlam1, amax)


class TpmRequest(ctypes.Structure):
    _fields_ = [("params", TpmParams), ("np", ctypes.c_int64), ("pos", ctypes.c_void_p), ("vel", ctypes.c_void_p),
                ("cosmo", TpmCosmology), ("anow", ctypes.c_float), ("astep", ctypes.c_float),
                ("nsteps", ctypes.c_int32), ("pos_out", ctypes.c_void_p), ("vel_out", ctypes.c_void_p),
                ("force_out", ctypes.c_void_p)]


class TpmRequestInfo(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int32), ("status", ctypes.c_int32), ("t_submit", ctypes.c_double),
                ("t_admit", ctypes.c_double), ("t_done", ctypes.c_double), ("device_bytes", ctypes.c_int64)]


REQ_QUEUED, REQ_ACTIVE, REQ_DONE, REQ_FAILED = 0, 1, 2, 3


class TpmTuning(ctypes.Structure):
    _fields_ = [("fft_pencils_x", ctypes.c_int32), ("fft_cols", ctypes.c_int32), ("group_level", ctypes.c_int32),
                ("group_max", ctypes.c_int32), ("ms_fft", ctypes.c_float), ("ms_fft_default", ctypes.c_float),
                ("ms_walk", ctypes.c_float), ("ms_walk_default", ctypes.c_float)]


TUNE_FFT, TUNE_GROUPS = 1, 2


class TpmSnapshotInfo(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int64), ("ny", ctypes.c_int64), ("nz", ctypes.c_int64), ("np_dm", ctypes.c_int64),
                ("np_sph", ctypes.c_int64), ("np_star", ctypes.c_int64), ("np_agn", ctypes.c_int64),
                ("ptype", ctypes.c_int32), ("record_bytes", ctypes.c_int32), ("anow", ctypes.c_double),
                ("astep", ctypes.c_double)] + \
        [(k, ctypes.c_float) for k in ("omep", "omeplam", "wlam0", "wlam1", "amax", "boxsize", "theta", "epsilon",
                                       "rsphere")] + \
        [("stepcount", ctypes.c_int32), ("data_offset", ctypes.c_int64)]


class TpmIcParams(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("n", ctypes.c_int32), ("iseed", ctypes.c_int64),
                ("velpot", ctypes.c_void_p), ("fnl", ctypes.c_float), ("gnl", ctypes.c_float),
                ("vamp", ctypes.c_float), ("pfact", ctypes.c_float), ("vamp2", ctypes.c_float),
                ("damp1", ctypes.c_float), ("damp2", ctypes.c_float), ("boxsize", ctypes.c_float),
                ("omep", ctypes.c_float), ("amax", ctypes.c_float), ("growth", ctypes.c_float)]


class EngineError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"tpm error {code}: {msg}")
        self.code = code


_lib = None

# every function declared in include/tpm_engine.h with its ctypes signature
_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_SIGS = {
    "tpm_default_params": (None, [ctypes.POINTER(TpmParams), ctypes.c_int32]),
    "tpm_last_error": (ctypes.c_char_p, []),
    "tpm_version": (ctypes.c_char_p, []),
    "tpm_device_count": (ctypes.c_int, []),
    "tpm_create": (ctypes.c_int, [ctypes.POINTER(TpmParams), ctypes.c_int, ctypes.POINTER(_P)]),
    "tpm_destroy": (ctypes.c_int, [_P]),
    "tpm_set_params": (ctypes.c_int, [_P, ctypes.POINTER(TpmParams)]),
    "tpm_get_params": (ctypes.c_int, [_P, ctypes.POINTER(TpmParams)]),
    "tpm_load_fixed": (ctypes.c_int, [_P, _I64, _P, _P, ctypes.c_int]),
    "tpm_load_lagrangian": (ctypes.c_int, [_P, _I64, _P, _I64, _I64, _I64, _I64, ctypes.c_int]),
    "tpm_compute_forces": (ctypes.c_int, [_P, ctypes.c_uint]),
    "tpm_read_forces": (ctypes.c_int, [_P, _P, ctypes.c_int]),
    "tpm_kick": (ctypes.c_int, [_P, ctypes.c_float, ctypes.c_float]),
    "tpm_drift": (ctypes.c_int, [_P, ctypes.c_double]),
    "tpm_read_velocities": (ctypes.c_int, [_P, _P, ctypes.c_int]),
    "tpm_read_positions": (ctypes.c_int, [_P, _P, ctypes.c_int]),
    "tpm_store_lagrangian_velocities": (ctypes.c_int, [_P, _P, _I64, _I64, ctypes.c_int]),
    "tpm_sync": (ctypes.c_int, [_P]),
    "tpm_stream": (_P, [_P]),
    "tpm_pmmain": (ctypes.c_int, [_P, _P, _I64, ctypes.c_float]),
    "tpm_treecorrection": (ctypes.c_int, [_P, _P, _I64, ctypes.c_float]),
    "tpm_treemain": (ctypes.c_int, [_P, _P, _I64, ctypes.c_float, ctypes.c_int]),
    "tpm_ewald": (ctypes.c_int, [_P, _I64, _P, _P]),
    "tpm_stage_times": (ctypes.c_int, [_P, _P, ctypes.c_int]),
    "tpm_counters": (ctypes.c_int, [_P, _P, ctypes.c_int]),
    "tpm_launch_count": (_I64, [_P]),
    "tpm_read_order": (ctypes.c_int, [_P, _P, _P]),
    "tpm_read_mesh": (ctypes.c_int, [_P, ctypes.c_int, _P]),
    "tpm_morton_order_noalloc": (ctypes.c_int, [_P, _I64, ctypes.c_int32, _P, _P, _P]),
    "tpm_graph_compute": (ctypes.c_int, [_P, ctypes.c_uint]),
    "tpm_batch_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)]),
    "tpm_batch_destroy": (ctypes.c_int, [_P]),
    "tpm_batch_compute": (ctypes.c_int, [_P, ctypes.c_uint]),
    "tpm_batch_step": (ctypes.c_int, [_P, ctypes.POINTER(TpmCosmology), ctypes.POINTER(ctypes.c_float),
                                      ctypes.POINTER(ctypes.c_float)]),
    "tpm_batch_time": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_float)]),
    "tpm_autotune": (ctypes.c_int, [_P, ctypes.c_uint, ctypes.POINTER(TpmTuning)]),
    "tpm_get_tuning": (ctypes.c_int, [_P, ctypes.POINTER(TpmTuning)]),
    "tpm_set_tuning": (ctypes.c_int, [_P, ctypes.POINTER(TpmTuning)]),
    "tpm_fof": (ctypes.c_int, [_P, ctypes.c_float, ctypes.c_int32, _P, ctypes.c_int, _P]),
    "tpm_set_power_spectrum": (ctypes.c_int, [_P, ctypes.c_int]),
    "tpm_power_spectrum": (ctypes.c_int, [_P, ctypes.c_double, _P, _P, ctypes.c_int32, _P, _P]),
    "tpm_snapshot_info_read": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(TpmSnapshotInfo)]),
    "tpm_snapshot_read_dm": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(TpmSnapshotInfo), _P, _I64, _I64]),
    "tpm_snapshot_write": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(TpmSnapshotInfo), _P]),
    "tpm_estimate_bytes": (ctypes.c_int64, [ctypes.c_int32, ctypes.c_int64]),
    "tpm_server_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int64, ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)]),
    "tpm_server_submit": (ctypes.c_int, [_P, ctypes.POINTER(TpmRequest), ctypes.POINTER(ctypes.c_int64)]),
    "tpm_server_info": (ctypes.c_int, [_P, ctypes.c_int64, ctypes.POINTER(TpmRequestInfo)]),
    "tpm_server_wait": (ctypes.c_int, [_P, ctypes.c_int64, ctypes.c_double]),
    "tpm_server_stats": (ctypes.c_int, [_P, _P, ctypes.c_int]),
    "tpm_server_reserve": (ctypes.c_int, [_P, ctypes.c_int64]),
    "tpm_server_destroy": (ctypes.c_int, [_P]),
    "tpm_evol_factors": (ctypes.c_int, [ctypes.POINTER(TpmCosmology), ctypes.c_int32, ctypes.c_float,
                                        ctypes.c_float, ctypes.POINTER(TpmEvolFact)]),
    "tpm_hubble_drag": (ctypes.c_int, [_P, ctypes.c_float]),
    "tpm_step": (ctypes.c_int, [_P, ctypes.POINTER(TpmCosmology), ctypes.c_float, ctypes.c_float, ctypes.c_int32]),
    "tpm_status_factors": (ctypes.c_int, [ctypes.POINTER(TpmEvolFact), ctypes.c_int32, ctypes.POINTER(ctypes.c_float),
                                          ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]),
    "tpm_status_kick": (ctypes.c_int, [_P, ctypes.POINTER(TpmCosmology), ctypes.c_float, ctypes.c_float,
                                       ctypes.c_int32]),
    "tpm_global_step": (ctypes.c_int, [_P, ctypes.POINTER(TpmCosmology), ctypes.c_float, ctypes.c_float,
                                       ctypes.c_int32, ctypes.c_int32]),
    "tpm_stream_submit": (ctypes.c_int, [_P, _I64, _P, _P, ctypes.c_uint, ctypes.POINTER(ctypes.c_int64)]),
    "tpm_stream_wait": (ctypes.c_int, [_P, _I64]),
    "tpm_ic_noise": (ctypes.c_int, [ctypes.POINTER(TpmIcParams), _P, ctypes.c_int]),
    "tpm_ic_zeldovich": (ctypes.c_int, [ctypes.POINTER(TpmIcParams), _P, ctypes.c_int]),
    "tpm_ic_2lpt": (ctypes.c_int, [ctypes.POINTER(TpmIcParams), _P, ctypes.c_int]),
}


def load_library(path: str = LIB_PATH):
    """Load libtpm_engine.so; raises if it is missing (no silent fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m lageunha_b200.build`")
    lib = ctypes.CDLL(path)
    for name, (res, args) in _SIGS.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _check(rc):
    if rc != TPM_OK:
        raise EngineError(rc, load_library().tpm_last_error().decode())


def _ptr(a):
    """(pointer, mem) of a numpy array (host) or a CUDA torch tensor (device)."""
    if isinstance(a, np.ndarray):
        if not a.flags.c_contiguous:
            raise ValueError("array must be C-contiguous")
        return a.ctypes.data, MEM_HOST
    if hasattr(a, "data_ptr") and hasattr(a, "is_cuda"):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return a.data_ptr(), (MEM_DEVICE if a.is_cuda else MEM_HOST)
    raise TypeError(f"unsupported buffer type {type(a)}")


def default_params(n_mesh: int) -> TpmParams:
    p = TpmParams()
    load_library().tpm_default_params(ctypes.byref(p), n_mesh)
    return p


class Engine:
    """One periodic box on one GPU (a tpm_ctx)."""

    def __init__(self, n_mesh: int, *, theta: float = 0.3, rsphere: float = 4.0, epsilon: float = 0.1,
                 efold: float = 0.9, law: str | int = "reference", rs_split: float = 1.25,
                 particle_mass: float = 1.0, device: int = 0):
        lib = load_library()
        p = default_params(n_mesh)
        p.theta, p.rsphere, p.epsilon, p.efold = theta, rsphere, epsilon, efold
        p.law = {"reference": TPM_LAW_REFERENCE, "gaussian": TPM_LAW_GAUSSIAN}.get(law, law)
        p.rs_split, p.particle_mass = rs_split, particle_mass
        ctx = ctypes.c_void_p()
        _check(lib.tpm_create(ctypes.byref(p), device, ctypes.byref(ctx)))
        self._lib, self._ctx, self.n_mesh, self.np = lib, ctx, n_mesh, 0

    # ---------------------------------------------------------------- lifecycle
    def close(self):
        if self._ctx:
            self._lib.tpm_destroy(self._ctx)
            self._ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def params(self) -> TpmParams:
        p = TpmParams()
        _check(self._lib.tpm_get_params(self._ctx, ctypes.byref(p)))
        return p

    def set_params(self, **kw):
        p = self.params
        for k, v in kw.items():
            if k == "law":
                v = {"reference": TPM_LAW_REFERENCE, "gaussian": TPM_LAW_GAUSSIAN}.get(v, v)
            setattr(p, k, v)
        _check(self._lib.tpm_set_params(self._ctx, ctypes.byref(p)))
        self.n_mesh = p.n_mesh

    @property
    def stream(self) -> int:
        return self._lib.tpm_stream(self._ctx) or 0

    # ---------------------------------------------------------------- state
    def load_fixed(self, pos_u32, vel=None):
        """pos_u32: (np, 3) uint32 fixed point (numpy or CUDA tensor)."""
        np_ = int(pos_u32.shape[0])
        pp, mem = _ptr(pos_u32)
        vp = None
        if vel is not None:
            vp, vmem = _ptr(vel)
            if vmem != mem:
                raise ValueError("positions and velocities must live in the same memory")
        _check(self._lib.tpm_load_fixed(self._ctx, np_, pp, vp, mem))
        self.np = np_

    def load_lagrangian(self, records, off_indx=None, off_pos=None, off_vel=None):
        """records: structured array with DM_DTYPE or TREEDM_DTYPE fields."""
        dt = records.dtype
        oi = dt.fields["indx"][1] if off_indx is None else off_indx
        op = dt.fields["x"][1] if off_pos is None else off_pos
        ov = (dt.fields["vx"][1] if "vx" in dt.fields else -1) if off_vel is None else off_vel
        rp, mem = _ptr(records)
        _check(self._lib.tpm_load_lagrangian(self._ctx, records.shape[0], rp, dt.itemsize, oi, op, ov, mem))
        self.np = int(records.shape[0])

    def compute(self, parts: int = PART_ALL):
        _check(self._lib.tpm_compute_forces(self._ctx, parts))

    def forces(self, out=None):
        if out is None:
            out = np.empty((self.np, 3), np.float32)
        op, mem = _ptr(out)
        _check(self._lib.tpm_read_forces(self._ctx, op, mem))
        return out

    def kick(self, fact2_pm: float, fact2_tree: float):
        _check(self._lib.tpm_kick(self._ctx, fact2_pm, fact2_tree))

    def drift(self, pfact: float):
        _check(self._lib.tpm_drift(self._ctx, pfact))

    def velocities(self, out=None):
        if out is None:
            out = np.empty((self.np, 3), np.float32)
        op, mem = _ptr(out)
        _check(self._lib.tpm_read_velocities(self._ctx, op, mem))
        return out

    def positions(self, out=None):
        if out is None:
            out = np.empty((self.np, 3), np.uint32)
        op, mem = _ptr(out)
        _check(self._lib.tpm_read_positions(self._ctx, op, mem))
        return out

    def sync(self):
        _check(self._lib.tpm_sync(self._ctx))

    # ---------------------------------------------------------------- drop-in
    def pmmain(self, dm_records: np.ndarray, fact2: float = 1.0):
        """pmmain (Cosmos/pmmain.c:390) on GOTPM dmparticletype records:
        v += fact2 * F_PM in place."""
        if dm_records.dtype != DM_DTYPE:
            raise TypeError("pmmain wants DM_DTYPE records")
        _check(self._lib.tpm_pmmain(self._ctx, dm_records.ctypes.data, dm_records.shape[0], fact2))
        self.np = int(dm_records.shape[0])

    def treecorrection(self, tdm_records: np.ndarray, fact2: float = 1.0):
        """treecorrection (Cosmos/treecorrection.c:225) on treedmparticletype
        records: v += fact2 * F_tree in place."""
        if tdm_records.dtype != TREEDM_DTYPE:
            raise TypeError("treecorrection wants TREEDM_DTYPE records")
        _check(self._lib.tpm_treecorrection(self._ctx, tdm_records.ctypes.data, tdm_records.shape[0], fact2))
        self.np = int(tdm_records.shape[0])

    def treemain(self, tdm_records: np.ndarray, fact2: float, stepcount: int):
        """TreeMain for GOTPM (Cosmos/Treemain.c:578-664)."""
        if tdm_records.dtype != TREEDM_DTYPE:
            raise TypeError("treemain wants TREEDM_DTYPE records")
        _check(self._lib.tpm_treemain(self._ctx, tdm_records.ctypes.data, tdm_records.shape[0], fact2, stepcount))
        self.np = int(tdm_records.shape[0])

    def graph_compute(self, parts: int = PART_ALL):
        """tpm_compute_forces replayed from a captured CUDA graph."""
        _check(self._lib.tpm_graph_compute(self._ctx, parts))

    def autotune(self, what: int = TUNE_FFT | TUNE_GROUPS) -> dict:
        t = TpmTuning()
        _check(self._lib.tpm_autotune(self._ctx, what, ctypes.byref(t)))
        return {k: getattr(t, k) for k, _ in TpmTuning._fields_}

    @property
    def tuning(self) -> TpmTuning:
        t = TpmTuning()
        _check(self._lib.tpm_get_tuning(self._ctx, ctypes.byref(t)))
        return t

    @tuning.setter
    def tuning(self, t: TpmTuning):
        _check(self._lib.tpm_set_tuning(self._ctx, ctypes.byref(t)))

    def fof(self, link: float = 0.2, min_members: int = 20):
        """(labels, ngroups): friends-of-friends groups of the loaded
        particles; labels[i] = smallest caller index of i's group or -1."""
        out = np.empty(self.np, np.int32)
        ng = ctypes.c_int64()
        _check(self._lib.tpm_fof(self._ctx, link, min_members, out.ctypes.data, MEM_HOST, ctypes.addressof(ng)))
        return out, ng.value

    def measure_power_spectrum(self, enable: bool = True):
        _check(self._lib.tpm_set_power_spectrum(self._ctx, 1 if enable else 0))

    def power_spectrum(self, boxsize: float) -> dict:
        """P(k), xi, sigma_8 and the xi slope of the last PM evaluation
        (the reference's CorrMeasure)."""
        nb = self.n_mesh + 1
        pk = np.zeros(nb)
        cor = np.zeros(nb)
        s8 = ctypes.c_double()
        sl = ctypes.c_double()
        k = self._lib.tpm_power_spectrum(self._ctx, boxsize, pk.ctypes.data, cor.ctypes.data, nb,
                                         ctypes.addressof(s8), ctypes.addressof(sl))
        _check(k if k < 0 else 0)
        return {"pk": pk[:k], "cor": cor[:k], "sigma8": s8.value, "slope": sl.value}

    def stream_submit(self, pos_host, forces_host, parts: int = PART_ALL) -> int:
        """Queue one evaluation of host positions with its copies overlapped
        (tpm_stream_submit); returns its ticket. Keep both buffers untouched
        until stream_wait(ticket)."""
        pp, pm = _ptr(pos_host)
        fp, fm = _ptr(forces_host)
        if pm != MEM_HOST or fm != MEM_HOST:
            raise ValueError("stream_submit takes host buffers")
        n = pos_host.shape[0]
        t = ctypes.c_int64()
        _check(self._lib.tpm_stream_submit(self._ctx, n, pp, fp, parts, ctypes.byref(t)))
        return t.value

    def stream_wait(self, ticket: int):
        _check(self._lib.tpm_stream_wait(self._ctx, ticket))

    def hubble_drag(self, fact1: float):
        _check(self._lib.tpm_hubble_drag(self._ctx, fact1))

    def step(self, cosmo: TpmCosmology, anow: float, astep: float, stepcount: int):
        """One GOTPM global step in KICK status (Cosmos/globalT.c:221-305)."""
        _check(self._lib.tpm_step(self._ctx, ctypes.byref(cosmo), anow, astep, stepcount))

    def status_kick(self, cosmo: TpmCosmology, anow: float, astep: float, status: int):
        """Drag and kicks of one PMSTATUS (PUSH 0, PULL 1, KICK 2): the body of
        PM_PULL_AND_PUSH plus the tree kick (Cosmos/globalT.c:113-134)."""
        _check(self._lib.tpm_status_kick(self._ctx, ctypes.byref(cosmo), anow, astep, status))

    def global_step(self, cosmo: TpmCosmology, anow: float, astep: float, stepcount: int, sync: bool = False):
        """One global step with the reference's sequencing: KICK, or PULL then
        PUSH at a synchronisation step, then the drift (globalT.c:221-305)."""
        _check(self._lib.tpm_global_step(self._ctx, ctypes.byref(cosmo), anow, astep, stepcount, int(bool(sync))))

    # ---------------------------------------------------------------- diagnostics
    def ewald(self, targets) -> np.ndarray:
        t = np.ascontiguousarray(targets, dtype=np.int64)
        out = np.empty((t.shape[0], 3), np.float64)
        _check(self._lib.tpm_ewald(self._ctx, t.shape[0], t.ctypes.data, out.ctypes.data))
        return out

    def stage_times(self) -> dict:
        ms = np.zeros(len(STAGES), np.float32)
        k = self._lib.tpm_stage_times(self._ctx, ms.ctypes.data, len(STAGES))
        return {STAGES[i]: float(ms[i]) for i in range(k)}

    def counters(self) -> dict:
        c = np.zeros(7, np.int64)
        self._lib.tpm_counters(self._ctx, c.ctypes.data, 7)
        return {"nodes": int(c[0]), "pp": int(c[1]), "pc": int(c[2]), "groups": int(c[3]),
                "walk_iterations": int(c[4]), "walk_nodes": int(c[5]), "walk_max_stack": int(c[6])}

    def launch_count(self) -> int:
        return int(self._lib.tpm_launch_count(self._ctx))

    def order(self):
        keys = np.empty(self.np, np.uint64)
        perm = np.empty(self.np, np.uint32)
        _check(self._lib.tpm_read_order(self._ctx, keys.ctypes.data, perm.ctypes.data))
        return keys, perm

    def mesh(self, which: int = MESH_DENSITY) -> np.ndarray:
        out = np.empty(self.n_mesh ** 3, np.float32)
        _check(self._lib.tpm_read_mesh(self._ctx, which, out.ctypes.data))
        return out.reshape(self.n_mesh, self.n_mesh, self.n_mesh)


class Batch:
    """An ensemble of boxes (Engine objects on one device) evaluated through
    one graph launch per call (tpm_batch_*). The engines stay usable on their
    own; the batch must be closed before them."""

    def __init__(self, engines):
        self.engines = list(engines)
        self._lib = load_library()
        arr = (ctypes.c_void_p * len(self.engines))(*[e._ctx.value for e in self.engines])
        b = ctypes.c_void_p()
        _check(self._lib.tpm_batch_create(arr, len(self.engines), ctypes.byref(b)))
        self._b = b

    def close(self):
        if self._b:
            self._lib.tpm_batch_destroy(self._b)
            self._b = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def compute(self, parts: int = PART_ALL):
        _check(self._lib.tpm_batch_compute(self._b, parts))

    def step(self, cosmo: TpmCosmology, anow, astep):
        n = len(self.engines)
        a = (ctypes.c_float * n)(*np.broadcast_to(np.asarray(anow, np.float32), (n,)))
        s = (ctypes.c_float * n)(*np.broadcast_to(np.asarray(astep, np.float32), (n,)))
        _check(self._lib.tpm_batch_step(self._b, ctypes.byref(cosmo), a, s))

    @property
    def last_ms(self) -> float:
        ms = ctypes.c_float()
        _check(self._lib.tpm_batch_time(self._b, ctypes.byref(ms)))
        return ms.value


SERVER_STATS = ("done", "failed", "peak_active", "peak_bytes", "contexts_created", "contexts_reused",
                "contexts_evicted", "deferred_admissions", "create_us", "upload_us", "capture_us", "reserve_us", "arena_bytes")


def estimate_bytes(n_mesh: int, np_: int) -> int:
    return int(load_library().tpm_estimate_bytes(n_mesh, np_))


class Server:
    """The request loop (tpm_server_*): continuous batching of force and step
    requests for boxes of different sizes on one device. Arrays handed to
    submit() are kept referenced here until the server is closed."""

    def __init__(self, hbm_cap_bytes: int = 150 * 10 ** 9, max_active: int = 64, device: int = 0,
                 reserve_bytes: int = 0):
        self._lib = load_library()
        s = ctypes.c_void_p()
        _check(self._lib.tpm_server_create(device, int(hbm_cap_bytes), max_active, ctypes.byref(s)))
        self._s = s
        self._keep = {}
        if reserve_bytes:
            self.reserve(reserve_bytes)

    def reserve(self, nbytes: int):
        """Claims device memory for the contexts now (tpm_server_reserve)."""
        _check(self._lib.tpm_server_reserve(self._s, int(nbytes)))

    def submit(self, pos, vel=None, *, n_mesh: int, nsteps: int = 0, anow: float = 1.0, astep: float = 0.0,
               cosmo: TpmCosmology | None = None, pos_out=None, vel_out=None, force_out=None, **params) -> int:
        p = default_params(n_mesh)
        for k, v in params.items():
            if k == "law":
                v = {"reference": TPM_LAW_REFERENCE, "gaussian": TPM_LAW_GAUSSIAN}.get(v, v)
            setattr(p, k, v)
        pos = np.ascontiguousarray(pos, np.uint32)
        vel = None if vel is None else np.ascontiguousarray(vel, np.float32)
        r = TpmRequest()
        r.params = p
        r.np = pos.shape[0]
        r.pos = pos.ctypes.data
        r.vel = None if vel is None else vel.ctypes.data
        r.cosmo = cosmo if cosmo is not None else cosmology()
        r.anow, r.astep, r.nsteps = anow, astep, nsteps
        for name, arr in (("pos_out", pos_out), ("vel_out", vel_out), ("force_out", force_out)):
            if arr is not None:
                assert arr.flags["C_CONTIGUOUS"] and arr.shape == (r.np, 3) and arr.itemsize == 4
                setattr(r, name, arr.ctypes.data)
        rid = ctypes.c_int64()
        _check(self._lib.tpm_server_submit(self._s, ctypes.byref(r), ctypes.byref(rid)))
        self._keep[rid.value] = (pos, vel, pos_out, vel_out, force_out)
        return rid.value

    def info(self, rid: int) -> TpmRequestInfo:
        out = TpmRequestInfo()
        _check(self._lib.tpm_server_info(self._s, rid, ctypes.byref(out)))
        return out

    def wait(self, rid: int = -1, timeout: float = 600.0):
        _check(self._lib.tpm_server_wait(self._s, rid, timeout))

    def stats(self) -> dict:
        out = np.zeros(len(SERVER_STATS), np.int64)
        k = self._lib.tpm_server_stats(self._s, out.ctypes.data, len(SERVER_STATS))
        return {SERVER_STATS[i]: int(out[i]) for i in range(k)}

    def close(self):
        if self._s:
            self._lib.tpm_server_destroy(self._s)
            self._s = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def evol_factors(cosmo: TpmCosmology, nx: int, anow: float, astep: float) -> dict:
    """GetEvolFactor (Cosmos/CosmosEvolFactor.c:230-255); host only."""
    out = TpmEvolFact()
    _check(load_library().tpm_evol_factors(ctypes.byref(cosmo), nx, anow, astep, ctypes.byref(out)))
    return {k: getattr(out, k) for k, _ in TpmEvolFact._fields_}


PUSH, PULL, KICK = 0, 1, 2  # PMSTATUS (eunha.h:72-77)


def status_factors(cosmo: TpmCosmology, nx: int, anow: float, astep: float, status: int) -> tuple:
    """(drag, pm_kick, tree_kick) of one status (tpm_status_factors)."""
    lib = load_library()
    e = TpmEvolFact()
    _check(lib.tpm_evol_factors(ctypes.byref(cosmo), nx, anow, astep, ctypes.byref(e)))
    d, p, t = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
    _check(lib.tpm_status_factors(ctypes.byref(e), status, ctypes.byref(d), ctypes.byref(p), ctypes.byref(t)))
    return d.value, p.value, t.value


def read_snapshot(path: str):
    """(header dict, dark-matter records) of a GOTPM snapshot file: records as
    DM_DTYPE (particle type 0) or TREEDM_DTYPE (1), ready for
    Engine.load_lagrangian."""
    lib = load_library()
    info = TpmSnapshotInfo()
    _check(lib.tpm_snapshot_info_read(path.encode(), ctypes.byref(info)))
    rec = np.empty(info.np_dm, DM_DTYPE if info.ptype == 0 else TREEDM_DTYPE)
    _check(lib.tpm_snapshot_read_dm(path.encode(), ctypes.byref(info), rec.ctypes.data, 0, info.np_dm))
    return {k: getattr(info, k) for k, _ in TpmSnapshotInfo._fields_}, rec


def write_snapshot(path: str, records: np.ndarray, n_mesh: int, **header):
    """A GOTPM snapshot of the records (DM_DTYPE or TREEDM_DTYPE) that the
    reference's jread reads; header: omep, omeplam, wlam0, wlam1, amax, anow,
    astep, boxsize, theta, epsilon, stepcount."""
    lib = load_library()
    info = TpmSnapshotInfo()
    info.nx = info.ny = info.nz = n_mesh
    info.np_dm = records.shape[0]
    info.ptype = 0 if records.dtype == DM_DTYPE else 1
    info.omep, info.omeplam, info.wlam0, info.wlam1, info.amax = 0.26, 0.74, -1.0, 0.0, 48.0
    info.anow, info.astep, info.boxsize, info.theta, info.epsilon = 1.0, 0.02, 100.0, 0.3, 0.1
    for k, v in header.items():
        setattr(info, k, v)
    rec = np.ascontiguousarray(records)
    _check(lib.tpm_snapshot_write(path.encode(), ctypes.byref(info), rec.ctypes.data))


def dm_records(ps) -> np.ndarray:
    """GOTPM dmparticletype records of a ParticleSet (lageunha_b200.ic)."""
    r = np.zeros(ps.np, DM_DTYPE)
    r["indx"] = ps.indx
    r["x"], r["y"], r["z"] = ps.offset[:, 0], ps.offset[:, 1], ps.offset[:, 2]
    r["vx"], r["vy"], r["vz"] = ps.vel[:, 0], ps.vel[:, 1], ps.vel[:, 2]
    return r


def treedm_records(ps) -> np.ndarray:
    r = np.zeros(ps.np, TREEDM_DTYPE)
    r["indx"] = ps.indx
    r["x"], r["y"], r["z"] = ps.offset[:, 0], ps.offset[:, 1], ps.offset[:, 2]
    r["vx"], r["vy"], r["vz"] = ps.vel[:, 0], ps.vel[:, 1], ps.vel[:, 2]
    return r


def _ic_params(n, iseed, velpot, fnl, gnl, vamp, pfact, device):
    p = TpmIcParams()
    p.device, p.n, p.iseed = device, n, iseed
    p.fnl, p.gnl, p.vamp, p.pfact = fnl, gnl, vamp, pfact
    keep = None
    if velpot is not None:
        keep = np.ascontiguousarray(velpot, dtype=np.float32)
        if keep.shape[0] < (n // 2) ** 2 + 1:
            raise ValueError("velpot needs (n/2)^2 + 1 entries")
        p.velpot = keep.ctypes.data
    return p, keep


def ic_noise(n: int, iseed: int, velpot=None, device: int = 0) -> np.ndarray:
    """The reference's Zel'dovich noise spectrum (tpm_ic_noise) as complex64
    [z][y][kx], kx in [0, n/2]."""
    lib = load_library()
    p, keep = _ic_params(n, iseed, velpot, 0.0, 0.0, 1.0, 1.0, device)
    out = np.empty((n, n, n // 2 + 1), np.complex64)
    _check(lib.tpm_ic_noise(ctypes.byref(p), out.ctypes.data, MEM_HOST))
    del keep
    return out


def ic_zeldovich(n: int, iseed: int, velpot=None, fnl: float = 0.0, gnl: float = 0.0, vamp: float = 1.0,
                 pfact: float | None = None, device: int = 0, out=None):
    """Zel'dovich particles (tpm_ic_zeldovich): n^3 DM_DTYPE records, lattice
    order z, y, x; pfact defaults to the reference's AI * NX = n. `out`: a
    device tensor of n^3 * 32 bytes to receive the records instead of a new
    host array."""
    lib = load_library()
    p, keep = _ic_params(n, iseed, velpot, fnl, gnl, vamp, float(n if pfact is None else pfact), device)
    if out is not None:
        if out.numel() * out.element_size() < n ** 3 * DM_DTYPE.itemsize:
            raise ValueError("out is smaller than n^3 records")
        ptr, mem = _ptr(out)
        _check(lib.tpm_ic_zeldovich(ctypes.byref(p), ptr, mem))
        del keep
        return out
    rec = np.empty(n ** 3, DM_DTYPE)
    _check(lib.tpm_ic_zeldovich(ctypes.byref(p), rec.ctypes.data, MEM_HOST))
    del keep
    return rec


def ic_2lpt(n: int, iseed: int, velpot=None, vamp: float = 1.0, vamp2: float = 0.0, damp1: float = 1.0,
            damp2: float = -3.0 / 7.0, pfact: float | None = None, device: int = 0, out=None, fnl: float = 0.0,
            gnl: float = 0.0, boxsize: float = 0.0, omep: float = 0.0, amax: float = 0.0, growth: float = 0.0):
    """Second-order Lagrangian particles (tpm_ic_2lpt): n^3 DM_DTYPE records
    (or into the device tensor `out`); fnl/gnl need boxsize, omep, amax and
    growth (COS_GROWTH)."""
    lib = load_library()
    p, keep = _ic_params(n, iseed, velpot, fnl, gnl, vamp, float(n if pfact is None else pfact), device)
    p.vamp2, p.damp1, p.damp2 = vamp2, damp1, damp2
    p.boxsize, p.omep, p.amax, p.growth = boxsize, omep, amax, growth
    if out is not None:
        if out.numel() * out.element_size() < n ** 3 * DM_DTYPE.itemsize:
            raise ValueError("out is smaller than n^3 records")
        ptr, mem = _ptr(out)
        _check(lib.tpm_ic_2lpt(ctypes.byref(p), ptr, mem))
        del keep
        return out
    rec = np.empty(n ** 3, DM_DTYPE)
    _check(lib.tpm_ic_2lpt(ctypes.byref(p), rec.ctypes.data, MEM_HOST))
    del keep
    return rec
