"""ctypes binding of libcgfd.so, the B200 CGFD solver (include/cgfd.h).

The binding is a thin host-side mirror of the reference's device runtime,
class ChildProcs (src/typedata.h:114-217): create the solver from a
description, upload metric / media / PML factors / sources / receivers
(ParH2D, src/calculate.cu:2050-2228), step (the RKite loop of
src/simulation.cc:252-711) and read seismograms (PWpick/PWgather).

Every call goes to the CUDA library; there is no Python or CPU fallback.  If
the library is missing the import fails with the build command to run.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "libcgfd.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing; build it with `make -C {os.path.dirname(_HERE)}`")
_lib = C.CDLL(LIB_PATH)

OK, ERR_ARG, ERR_CUDA, ERR_STATE, ERR_NOMEM, ERR_TIMEOUT, ERR_NONFINITE, ERR_NODEVICE = range(8)
STORE_F32, STORE_F16, STORE_BF16 = 0, 1, 2
KERNEL_FUSED, KERNEL_SIMPLE, KERNEL_SCALAR = 0, 1, 2
BATCH_PERSISTENT, BATCH_MEMBERS = 0, 1  # cgfd_batch_set_launch
SET_FW, SET_W, SET_TW = 0, 1, 2
COMPONENTS = ("Vx", "Vy", "Vz", "Txx", "Tyy", "Tzz", "Txy", "Txz", "Tyz")
STF_TYPES = {"Gauss": 0, "gauss": 1, "Ricker": 2, "ricker": 3, "Bell": 4,
             "bell": 5, "BELL": 6, "Step": 7}


class Desc(C.Structure):
    _fields_ = [("ni", C.c_int), ("nj", C.c_int), ("nk", C.c_int),
                ("steph", C.c_double), ("stept", C.c_double), ("nt", C.c_int),
                ("con_index", C.c_int), ("hybrid_grid", C.c_int),
                ("nabs", C.c_int * 6), ("storage", C.c_int), ("device", C.c_int),
                ("kernel", C.c_int)]


_P = C.c_void_p
_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)

_SIGS = {
    "cgfd_create": (C.c_int, [C.POINTER(Desc), C.POINTER(_P)]),
    "cgfd_destroy": (C.c_int, [_P]),
    "cgfd_last_error": (C.c_int, [_P, C.c_char_p, C.c_size_t]),
    "cgfd_upload_metric": (C.c_int, [_P, _dp, _dp, _dp, _dp]),
    "cgfd_upload_media": (C.c_int, [_P, _fp, _fp, _fp]),
    "cgfd_upload_pml": (C.c_int, [_P] + [_dp] * 9),
    "cgfd_upload_moments": (C.c_int, [_P, C.c_int, _ip, _fp, C.c_int, _fp]),
    "cgfd_upload_forces": (C.c_int, [_P, C.c_int, _ip, _fp, C.c_int, _fp]),
    "cgfd_set_receivers": (C.c_int, [_P, C.c_int, _ip]),
    "cgfd_prepare": (C.c_int, [_P]),
    "cgfd_step": (C.c_int, [_P, C.c_int]),
    "cgfd_step_timed": (C.c_int, [_P, C.c_int, _fp, _fp]),
    "cgfd_rk_stage": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
    "cgfd_sync": (C.c_int, [_P, C.c_double]),
    "cgfd_steps_done": (C.c_int, [_P, _ip]),
    "cgfd_get_seismograms": (C.c_int, [_P, _fp, _ip]),
    "cgfd_get_field": (C.c_int, [_P, C.c_int, C.c_int, _fp]),
    "cgfd_set_field": (C.c_int, [_P, C.c_int, C.c_int, _fp]),
    "cgfd_check_finite": (C.c_int, [_P, C.POINTER(C.c_longlong)]),
    "cgfd_set_field_scales": (C.c_int, [_P, _ip]),
    "cgfd_autotune": (C.c_int, [_P, C.c_int, _fp]),
    "cgfd_test_withhold_copy": (C.c_int, [_P, C.c_double, C.c_int]),
    "cgfd_set_boundary_mlp": (C.c_int, [_P, C.c_int, C.c_void_p]),
    "cgfd_set_boundary_mlp_gains": (C.c_int, [_P, _fp]),
    "cgfd_upload_focal": (C.c_int, [_P, C.c_int, _ip, C.c_int, C.c_double, _fp]),
    "cgfd_set_source_smoothing": (C.c_int, [_P, C.c_int, C.c_int, _dp]),
    "cgfd_locate_points": (C.c_int, [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, C.c_double,
                                     C.c_int, _dp, _ip, _dp]),
    "cgfd_source_smoothing": (C.c_int, [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, C.c_int,
                                        C.c_int, _dp, _ip, _dp]),
    "cgfd_media_volume": (C.c_int, [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, C.c_int, C.c_int,
                                    C.c_int, _dp, _dp, _dp, _fp, _fp, _fp, C.c_double,
                                    C.c_double, C.c_int, C.c_int, C.c_int, _fp, _fp, _fp]),
    "cgfd_grid_vmap": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, _ip, _ip, _dp, C.c_int,
                                 C.c_double, _dp, _dp, _dp, _ip]),
    "cgfd_boundary_mlp_cells": (C.c_int, [_P, _ip, _ip]),
    "cgfd_boundary_mlp_features": (C.c_int, [_P, _fp, _fp, _fp]),
    "cgfd_mlp_gradient": (C.c_int, [C.c_void_p, _fp, _fp, C.c_int, _fp, _fp]),
    "cgfd_enable_peak_velocity": (C.c_int, [_P, C.c_int]),
    "cgfd_get_peak_velocity": (C.c_int, [_P, _fp]),
    "cgfd_get_snapshot": (C.c_int, [_P, C.c_int, _ip, _ip, _ip, C.c_int, _fp]),
    "cgfd_write_seismograms_nc": (C.c_int, [_P, C.c_char_p, _fp]),
    "cgfd_write_peak_velocity_nc": (C.c_int, [_P, C.c_char_p]),
    "cgfd_batch_create": (C.c_int, [C.POINTER(Desc), C.c_int, C.POINTER(_P)]),
    "cgfd_batch_solver": (C.c_int, [_P, C.c_int, C.POINTER(_P)]),
    "cgfd_batch_prepare": (C.c_int, [_P]),
    "cgfd_batch_step": (C.c_int, [_P, C.c_int]),
    "cgfd_batch_step_timed": (C.c_int, [_P, C.c_int, _fp]),
    "cgfd_batch_sync": (C.c_int, [_P, C.c_double]),
    "cgfd_batch_autotune": (C.c_int, [_P, C.c_int, _fp]),
    "cgfd_batch_set_launch": (C.c_int, [_P, C.c_int]),
    "cgfd_get_work_shape": (C.c_int, [_P, _ip, _ip, C.POINTER(C.c_double)]),
    "cgfd_set_work_shape": (C.c_int, [_P, C.c_int, C.c_int, C.c_double]),
    "cgfd_batch_get_launch": (C.c_int, [_P, _ip]),
    "cgfd_batch_last_error": (C.c_int, [_P, C.c_char_p, C.c_size_t]),
    "cgfd_batch_destroy": (C.c_int, [_P]),
    "cgfd_get_field_scales": (C.c_int, [_P, _ip]),
    "cgfd_count_nonfinite_noalloc": (C.c_int, [C.c_void_p, C.c_size_t, C.POINTER(C.c_longlong),
                                               C.c_void_p]),
    "cgfd_read_media_volume_nc": (C.c_int, [C.c_char_p, _ip, _ip, _ip, _dp, _dp, _dp, _fp, _fp,
                                            _fp]),
    "cgfd_read_focal_nc": (C.c_int, [C.c_char_p, _ip, _ip, _dp, _dp, _dp, _dp, _fp]),
    "cgfd_metric_from_coords": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double,
                                          _dp, _dp, _dp, C.POINTER(_dp)]),
    "cgfd_cfs_factors": (C.c_int, [C.c_int, C.c_int, C.c_int, _ip, _dp, _dp, _dp,
                                   _dp, _dp, _dp] + [_dp] * 9),
    "cgfd_stf": (C.c_int, [C.c_int, C.c_double, C.c_double, C.c_double, C.c_int,
                           C.c_double, _fp]),
    "cgfd_angle2moment": (C.c_int, [C.c_double, C.c_double, C.c_double, _dp]),
}
for _name, (_res, _args) in _SIGS.items():
    _f = getattr(_lib, _name)
    _f.restype = _res
    _f.argtypes = _args

EXPORTED = tuple(_SIGS)


class CgfdError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"cgfd status {status}: {msg}")
        self.status = status


def _d(a):
    return a.ctypes.data_as(_dp)


def _f(a):
    return a.ctypes.data_as(_fp)


def _i(a):
    return a.ctypes.data_as(_ip)


def _as(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def _sized(a, dtype, n, what):
    """a as a contiguous flat array of n values: the C ABI reads exactly n
    through the pointer, so a shorter array would be read past its end."""
    v = np.ascontiguousarray(a, dtype=dtype).reshape(-1)
    if v.size != n:
        raise ValueError(f"{what}: {v.size} values, the model needs {n}")
    return v


def last_error(handle=None) -> str:
    buf = C.create_string_buffer(1024)
    _lib.cgfd_last_error(handle, buf, 1024)
    return buf.value.decode(errors="replace")


def make_desc(ni, nj, nk, steph, stept, nt, con_index, nabs, storage=STORE_F32,
              device=0, kernel=KERNEL_FUSED, hybrid_grid=1) -> Desc:
    d = Desc()
    d.ni, d.nj, d.nk = ni, nj, nk
    d.steph, d.stept, d.nt = steph, stept, nt
    d.con_index, d.hybrid_grid = con_index, hybrid_grid
    for q in range(6):
        d.nabs[q] = int(nabs[q])
    d.storage, d.device, d.kernel = storage, device, kernel
    return d


class Solver:
    """One solver on one GPU (mirrors ChildProcs)."""

    def __init__(self, desc: Desc, _handle=None):
        if _handle is None:
            h = _P()
            st = _lib.cgfd_create(C.byref(desc), C.byref(h))
            if st:
                raise CgfdError(st, last_error(None))
            self._owned = True
        else:  # a member of a Batch: the batch owns it
            h = _handle
            self._owned = False
        self._h = h
        self.desc = desc
        self.shape = (desc.ni + 6, desc.nj + 6, desc.nk + 6)
        self.nrecv = 0

    def _chk(self, st):
        if st:
            raise CgfdError(st, last_error(self._h))

    def close(self):
        if getattr(self, "_h", None):
            if self._owned:
                _lib.cgfd_destroy(self._h)
            self._h = None

    def set_boundary_mlp(self, width: int, weights):
        """Learned layer correction (weights: CGFD_MLP_PARAMS values, stored
        as FP16; None disables)."""
        if weights is None:
            self._chk(_lib.cgfd_set_boundary_mlp(self._h, width, None))
            self._mlp_width = 0
            return
        w = _sized(weights, np.float16, MLP_PARAMS, "MLP weights")
        self._chk(_lib.cgfd_set_boundary_mlp(self._h, width, w.ctypes.data_as(C.c_void_p)))
        self._mlp_width = int(width)

    def set_boundary_mlp_gains(self, gains=None):
        """Per (depth, component) gains of the correction, [width][9]; None: 1."""
        if gains is None:
            self._chk(_lib.cgfd_set_boundary_mlp_gains(self._h, None))
            return
        g = _sized(gains, np.float32, 9 * getattr(self, "_mlp_width", 0), "layer gains")
        self._chk(_lib.cgfd_set_boundary_mlp_gains(self._h, _f(g)))

    def boundary_mlp_cells(self) -> np.ndarray:
        n = C.c_int(0)
        self._chk(_lib.cgfd_boundary_mlp_cells(self._h, None, C.byref(n)))
        out = np.empty((n.value, 3), np.int32)
        self._chk(_lib.cgfd_boundary_mlp_cells(self._h, _i(out), C.byref(n)))
        return out

    def boundary_mlp_features(self):
        """(x [n][45], scale [n], rho*vp [n]) of the layer's cells now."""
        n = len(self.boundary_mlp_cells())
        x = np.empty((n, 45), np.float32)
        sc = np.empty(n, np.float32)
        z = np.empty(n, np.float32)
        self._chk(_lib.cgfd_boundary_mlp_features(self._h, _f(x), _f(sc), _f(z)))
        return x, sc, z

    def enable_peak_velocity(self, on: bool = True):
        self._chk(_lib.cgfd_enable_peak_velocity(self._h, int(on)))

    def peak_velocity(self) -> np.ndarray:
        """max |V| per component over the steps since enabling, [3][ni][nj]."""
        out = np.empty((3, self.desc.ni, self.desc.nj), np.float32)
        self._chk(_lib.cgfd_get_peak_velocity(self._h, _f(out)))
        return out

    def snapshot(self, start, count, stride=(1, 1, 1), comps=range(9), set_=SET_FW):
        """Sub-volume of a field set (reference full-array indices), returned
        as [component][i][j][k]."""
        mask = 0
        for c in comps:
            mask |= 1 << c
        n = bin(mask).count("1")
        out = np.empty((n,) + tuple(int(c) for c in count), np.float32)
        a = [np.ascontiguousarray(x, np.int32) for x in (start, count, stride)]
        self._chk(_lib.cgfd_get_snapshot(self._h, set_, _i(a[0]), _i(a[1]), _i(a[2]), mask,
                                         _f(out)))
        return out

    def write_seismograms_nc(self, path: str, pos=None):
        p = None if pos is None else _as(pos, np.float32).reshape(-1)
        self._chk(_lib.cgfd_write_seismograms_nc(self._h, path.encode(),
                                                 None if p is None else _f(p)))

    def write_peak_velocity_nc(self, path: str):
        self._chk(_lib.cgfd_write_peak_velocity_nc(self._h, path.encode()))

    def autotune(self, steps: int = 3) -> float:
        """Picks the fastest work-list shape (state unchanged); returns its
        milliseconds per step."""
        ms = C.c_float()
        self._chk(_lib.cgfd_autotune(self._h, steps, C.byref(ms)))
        return ms.value

    @property
    def work_shape(self) -> tuple:
        """(items per resident CTA, shortest z-chunk, PML cost weight) of the
        work list in use (cgfd_get_work_shape; after prepare)."""
        a, b, c = C.c_int(), C.c_int(), C.c_double()
        self._chk(_lib.cgfd_get_work_shape(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return (a.value, b.value, c.value)

    @work_shape.setter
    def work_shape(self, shape):
        self._chk(_lib.cgfd_set_work_shape(self._h, int(shape[0]), int(shape[1]),
                                           float(shape[2])))

    def test_withhold_copy(self, wait_limit_s: float, withhold: int):
        """Test hook of the bounded device waits (cgfd_test_withhold_copy):
        the first velocity CTA withholds one tensor copy and every wait gives
        up after wait_limit_s; withhold < 0 restores normal operation."""
        self._chk(_lib.cgfd_test_withhold_copy(self._h, float(wait_limit_s), int(withhold)))

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def upload_metric(self, zeta_x, zeta_y, zeta_z, jac):
        n = int(np.prod(self.shape))
        arrs = [_sized(a, np.float64, n, "metric array") for a in (zeta_x, zeta_y, zeta_z, jac)]
        self._chk(_lib.cgfd_upload_metric(self._h, *[_d(a) for a in arrs]))

    def upload_media(self, alpha, beta, rho):
        n = int(np.prod(self.shape))
        arrs = [_sized(a, np.float32, n, "media array") for a in (alpha, beta, rho)]
        self._chk(_lib.cgfd_upload_media(self._h, *[_f(a) for a in arrs]))

    def upload_pml(self, apd, b, db):
        """CFS-PML profiles: apd, b and db each a triple of arrays over the
        full x, y and z index ranges (CalCFSfactors' APD, B and DB)."""
        arrs = [_sized(a, np.float64, self.shape[q % 3], "PML profile")
                for q, a in enumerate((*apd, *b, *db))]
        self._chk(_lib.cgfd_upload_pml(self._h, *[_d(a) for a in arrs]))

    def upload_moments(self, loc, m6, stf):
        loc = _as(loc, np.int32).reshape(-1, 3)
        m6 = _sized(m6, np.float32, 6 * len(loc), "moment tensors").reshape(-1, 6)
        stf = _as(stf, np.float32).reshape(len(loc), -1)
        self._chk(_lib.cgfd_upload_moments(self._h, len(loc), _i(loc), _f(m6),
                                           stf.shape[1], _f(stf)))

    def upload_forces(self, loc, f3, stf):
        loc = _as(loc, np.int32).reshape(-1, 3)
        f3 = _sized(f3, np.float32, 3 * len(loc), "force vectors").reshape(-1, 3)
        stf = _as(stf, np.float32).reshape(len(loc), -1)
        self._chk(_lib.cgfd_upload_forces(self._h, len(loc), _i(loc), _f(f3),
                                          stf.shape[1], _f(stf)))

    def upload_focal(self, loc, fdt, mom):
        """Finite-fault points: loc (n, 3), mom [6][n][fnt] moment series
        sampled every fdt seconds (cgfd_upload_focal); n = 0 removes them."""
        loc = _as(loc, np.int32).reshape(-1, 3)
        mom = _as(mom, np.float32).reshape(6, len(loc), -1) if len(loc) else np.zeros(1, np.float32)
        fnt = mom.shape[-1] if len(loc) else 1
        self._chk(_lib.cgfd_upload_focal(self._h, len(loc), _i(loc), fnt, float(fdt), _f(mom)))

    def set_source_smoothing(self, kind, weights):
        """Spread the uploaded sources of one kind (0 moments, 1 forces, 2
        focal points) over 7^3 nodes with weights [n][7][7][7] from
        source_smoothing(); None turns it off (cgfd_set_source_smoothing)."""
        if weights is None:
            self._chk(_lib.cgfd_set_source_smoothing(self._h, int(kind), 0, None))
            return
        w = _as(weights, np.float64).reshape(-1, 343)
        self._chk(_lib.cgfd_set_source_smoothing(self._h, int(kind), len(w), _d(w)))

    def set_receivers(self, loc):
        loc = _as(loc, np.int32).reshape(-1, 3)
        self._chk(_lib.cgfd_set_receivers(self._h, len(loc), _i(loc)))
        self.nrecv = len(loc)

    def prepare(self):
        self._chk(_lib.cgfd_prepare(self._h))

    def step(self, n=1):
        self._chk(_lib.cgfd_step(self._h, int(n)))

    def step_timed(self, n, per_stage=False):
        """Runs n steps; returns (device ms for the n steps, mean ms of one
        stage kernel or None).  per_stage issues the stages without graphs."""
        ms = C.c_float()
        sms = C.c_float()
        self._chk(_lib.cgfd_step_timed(self._h, int(n), C.byref(ms),
                                       C.byref(sms) if per_stage else None))
        return ms.value, (sms.value if per_stage else None)

    def rk_stage(self, rk, curr_t, x, y, z):
        self._chk(_lib.cgfd_rk_stage(self._h, rk, curr_t, x, y, z))

    def sync(self, timeout_s=600.0):
        self._chk(_lib.cgfd_sync(self._h, float(timeout_s)))

    def steps_done(self) -> int:
        n = C.c_int()
        self._chk(_lib.cgfd_steps_done(self._h, C.byref(n)))
        return n.value

    def seismograms(self) -> np.ndarray:
        """(9, nrecv, nt) float32, as HPW."""
        out = np.zeros((9, max(self.nrecv, 0), self.desc.nt), np.float32)
        n = C.c_int()
        self._chk(_lib.cgfd_get_seismograms(self._h, _f(out), C.byref(n)))
        return out

    def get_field(self, comp, fset=SET_FW) -> np.ndarray:
        out = np.zeros(self.shape, np.float32)
        self._chk(_lib.cgfd_get_field(self._h, fset, comp, _f(out)))
        return out

    def set_field(self, comp, values, fset=SET_FW):
        v = _as(values, np.float32).reshape(self.shape)
        self._chk(_lib.cgfd_set_field(self._h, fset, comp, _f(v)))

    def check_finite(self) -> int:
        n = C.c_longlong()
        st = _lib.cgfd_check_finite(self._h, C.byref(n))
        if st not in (OK, ERR_NONFINITE):
            self._chk(st)
        return n.value

    def set_field_scales(self, exp2) -> None:
        """Scale exponents of 16-bit storage per component (stored value s
        stands for s * 2**exp2[c])."""
        e = (C.c_int * 9)(*[int(x) for x in exp2])
        self._chk(_lib.cgfd_set_field_scales(self._h, e))

    def field_scales(self) -> list:
        e = (C.c_int * 9)()
        self._chk(_lib.cgfd_get_field_scales(self._h, e))
        return list(e)


MLP_PARAMS = 7689


def mlp_gradient(weights, x, t):
    """Mean squared error of the layer MLP on samples (x [n][45] -> t [n][9])
    and its gradient (device kernel); returns (loss, grad)."""
    w = np.ascontiguousarray(weights, np.float16)
    x = _as(x, np.float32)
    t = _as(t, np.float32)
    g = np.empty(MLP_PARAMS, np.float32)
    loss = C.c_float()
    st = _lib.cgfd_mlp_gradient(w.ctypes.data_as(C.c_void_p), _f(x), _f(t), len(x), _f(g),
                                C.byref(loss))
    if st:
        raise CgfdError(st, last_error(None))
    return loss.value, g


class Batch:
    """Several models stepped together in one persistent launch per stage
    part (cgfd_batch_*); models[i] is the member Solver for uploads, fields
    and seismograms."""

    def __init__(self, descs):
        arr = (Desc * len(descs))(*descs)
        h = _P()
        st = _lib.cgfd_batch_create(arr, len(descs), C.byref(h))
        if st:
            raise CgfdError(st, last_error(None))
        self._h = h
        self.models = []
        for i, d in enumerate(descs):
            m = _P()
            self._chk(_lib.cgfd_batch_solver(self._h, i, C.byref(m)))
            self.models.append(Solver(d, _handle=m))

    def _chk(self, st):
        if st:
            buf = C.create_string_buffer(1024)
            _lib.cgfd_batch_last_error(self._h, buf, 1024)
            raise CgfdError(st, buf.value.decode(errors="replace"))

    @property
    def cells(self) -> int:
        return sum(d.ni * d.nj * d.nk for d in (m.desc for m in self.models))

    def prepare(self):
        self._chk(_lib.cgfd_batch_prepare(self._h))

    def step(self, n: int):
        self._chk(_lib.cgfd_batch_step(self._h, n))

    def sync(self, timeout_s: float = 600.0):
        self._chk(_lib.cgfd_batch_sync(self._h, timeout_s))

    def step_timed(self, n: int) -> float:
        ms = C.c_float()
        self._chk(_lib.cgfd_batch_step_timed(self._h, n, C.byref(ms)))
        return ms.value

    def autotune(self, steps: int = 2) -> float:
        ms = C.c_float()
        self._chk(_lib.cgfd_batch_autotune(self._h, steps, C.byref(ms)))
        return ms.value

    @property
    def launch(self) -> int:
        """BATCH_PERSISTENT or BATCH_MEMBERS (cgfd_batch_get_launch)."""
        v = C.c_int()
        self._chk(_lib.cgfd_batch_get_launch(self._h, C.byref(v)))
        return v.value

    @launch.setter
    def launch(self, shape: int):
        self._chk(_lib.cgfd_batch_set_launch(self._h, shape))

    def close(self):
        if getattr(self, "_h", None):
            for m in self.models:
                m._h = None
            _lib.cgfd_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


NOALLOC_MAX_VALUES = 16384 * 8192


def count_nonfinite_noalloc(device_ptr: int, n: int, stream: int = 0) -> int:
    """NaN/Inf count of n floats at a device address, without any device
    allocation (cgfd_count_nonfinite_noalloc).  Raises CgfdError on argument
    or CUDA errors; returns the count otherwise."""
    out = C.c_longlong()
    st = _lib.cgfd_count_nonfinite_noalloc(C.c_void_p(device_ptr), n, C.byref(out),
                                           C.c_void_p(stream) if stream else None)
    if st not in (OK, ERR_NONFINITE):
        raise CgfdError(st, last_error(None))
    return out.value


# ------------------------- host pre-processing ------------------------------

def metric_from_coords(ni, nj, nk, steph, x, y, z):
    """gridmesh::calmetric: returns dict of 10 full arrays (FP64)."""
    shape = (ni + 6, nj + 6, nk + 6)
    xs = [_as(a, np.float64).reshape(shape) for a in (x, y, z)]
    names = ("xi_x", "xi_y", "xi_z", "eta_x", "eta_y", "eta_z",
             "zeta_x", "zeta_y", "zeta_z", "jac")
    outs = [np.zeros(shape, np.float64) for _ in names]
    ptrs = (_dp * 10)(*[_d(o) for o in outs])
    st = _lib.cgfd_metric_from_coords(ni, nj, nk, steph, *[_d(a) for a in xs], ptrs)
    if st:
        raise CgfdError(st, "metric_from_coords")
    return dict(zip(names, outs))


def cfs_factors(ni, nj, nk, nabs, velabs, bmax, amax, dlx, dly, dlz):
    """absorb::CalCFSfactors: returns (apd, b, db), each a tuple of 3 arrays."""
    nabs = _as(nabs, np.int32)
    v, bm, am = (_as(a, np.float64) for a in (velabs, bmax, amax))
    dl = [_as(a, np.float64) for a in (dlx, dly, dlz)]
    n3 = (ni + 6, nj + 6, nk + 6)
    outs = [np.zeros(n3[q % 3], np.float64) for q in range(9)]
    st = _lib.cgfd_cfs_factors(ni, nj, nk, _i(nabs), _d(v), _d(bm), _d(am),
                               *[_d(a) for a in dl], *[_d(o) for o in outs])
    if st:
        raise CgfdError(st, last_error(None) or "cfs_factors")
    return tuple(outs[0:3]), tuple(outs[3:6]), tuple(outs[6:9])


def stf(kind, start, t0, f0, n, dt) -> np.ndarray:
    out = np.zeros(n, np.float32)
    st = _lib.cgfd_stf(STF_TYPES[kind] if isinstance(kind, str) else int(kind),
                       start, t0, f0, n, dt, _f(out))
    if st:
        raise CgfdError(st, "stf")
    return out


def grid_vmap(ni, nj, nk, gridpoints, equalspacing, anchor, hybrid=False, convers_depth=0.0):
    """Node coordinates of a vmap grid (cgfd_grid_vmap): anchor [ni][nj][2 +
    nsurf] = x, y, z of each interface from the top down; returns (x, y, z)
    full arrays (ni+6, nj+6, nk+6) and ConIndex."""
    anchor = np.ascontiguousarray(anchor, np.float64)
    nsurf = anchor.shape[-1] - 2
    gp = np.ascontiguousarray(gridpoints, np.int32)
    eq = np.ascontiguousarray(equalspacing, np.int32)
    shape = (ni + 6, nj + 6, nk + 6)
    x, y, z = (np.zeros(shape, np.float64) for _ in range(3))
    con = C.c_int()
    st = _lib.cgfd_grid_vmap(ni, nj, nk, nsurf, _i(gp), _i(eq), _d(anchor), int(bool(hybrid)),
                             float(convers_depth), _d(x), _d(y), _d(z), C.byref(con))
    if st:
        raise CgfdError(st, last_error(None))
    return x, y, z, con.value


def media_volume(x, y, z, vx, vy, vz, vp, vs, rho, crit_value=50.0, crit_perc=0.05,
                 samp=(1, 1, 1)):
    """(alpha, beta, rho) full arrays from a volume model (cgfd_media_volume):
    x, y, z grid coordinates (ni+6, nj+6, nk+6); vp, vs, rho [nvx][nvy][nvz]
    on increasing axes vx, vy, vz."""
    x, y, z = (np.ascontiguousarray(a, np.float64) for a in (x, y, z))
    ni, nj, nk = (d - 6 for d in x.shape)
    vx, vy, vz = (np.ascontiguousarray(a, np.float64) for a in (vx, vy, vz))
    vp, vs, rho = (np.ascontiguousarray(a, np.float32) for a in (vp, vs, rho))
    out = [np.zeros(x.shape, np.float32) for _ in range(3)]
    st = _lib.cgfd_media_volume(ni, nj, nk, _d(x), _d(y), _d(z), len(vx), len(vy), len(vz),
                                _d(vx), _d(vy), _d(vz), _f(vp), _f(vs), _f(rho),
                                float(crit_value), float(crit_perc), int(samp[0]), int(samp[1]),
                                int(samp[2]), _f(out[0]), _f(out[1]), _f(out[2]))
    if st:
        raise CgfdError(st, last_error(None))
    return tuple(out)


def locate_points(x, y, z, pos, hyper_height):
    """Nearest valid node of each point (cgfd_locate_points): x, y, z full
    node arrays (ni+6, nj+6, nk+6), pos (n, 3).  Returns (loc (n, 3) int32,
    posz (n,)): points above hyper_height go to the nearest surface node in
    x-y and take its z."""
    x, y, z = (np.ascontiguousarray(a, np.float64) for a in (x, y, z))
    ni, nj, nk = (d - 6 for d in x.shape)
    pos = np.ascontiguousarray(pos, np.float64).reshape(-1, 3)
    loc = np.zeros((len(pos), 3), np.int32)
    posz = np.zeros(len(pos), np.float64)
    st = _lib.cgfd_locate_points(ni, nj, nk, _d(x), _d(y), _d(z), float(hyper_height), len(pos),
                                 _d(pos), _i(loc), _d(posz))
    if st:
        raise CgfdError(st, last_error(None))
    return loc, posz


def source_smoothing(x, y, z, kind, pos, loc):
    """Smoothing weights (cgfd_source_smoothing): kind 0 forces, 1 moment or
    focal points; pos (n, 3) with z as locate_points returns it, loc (n, 3)
    from locate_points.  Returns (loc, weights (n, 7, 7, 7)); loc moves to
    the nearest node of the sub-cell position for kind 1."""
    x, y, z = (np.ascontiguousarray(a, np.float64) for a in (x, y, z))
    ni, nj, nk = (d - 6 for d in x.shape)
    pos = np.ascontiguousarray(pos, np.float64).reshape(-1, 3)
    loc = np.array(loc, np.int32).reshape(-1, 3)
    w = np.zeros((len(pos), 7, 7, 7), np.float64)
    st = _lib.cgfd_source_smoothing(ni, nj, nk, _d(x), _d(y), _d(z), int(kind), len(pos),
                                    _d(pos), _i(loc), _d(w))
    if st:
        raise CgfdError(st, last_error(None))
    return loc, w


def read_media_volume_nc(path):
    """(vx, vy, vz, vp, vs, rho) of a volume media file in NetCDF classic
    format (cgfd_read_media_volume_nc); vp, vs, rho [nvx][nvy][nvz]."""
    n = [C.c_int() for _ in range(3)]
    b = path.encode()
    st = _lib.cgfd_read_media_volume_nc(b, *[C.byref(x) for x in n], None, None, None, None,
                                        None, None)
    if st:
        raise CgfdError(st, last_error(None))
    nv = [x.value for x in n]
    ax = [np.zeros(k) for k in nv]
    vol = [np.zeros(nv, np.float32) for _ in range(3)]
    st = _lib.cgfd_read_media_volume_nc(b, *[C.byref(x) for x in n], *[_d(a) for a in ax],
                                        *[_f(v) for v in vol])
    if st:
        raise CgfdError(st, last_error(None))
    return (*ax, *vol)


def read_focal_nc(path):
    """(dt, pos (np, 3), mom [6][np][nt]) of a finite-fault series file in
    NetCDF classic format (cgfd_read_focal_nc)."""
    npt, nt, dt = C.c_int(), C.c_int(), C.c_double()
    b = path.encode()
    st = _lib.cgfd_read_focal_nc(b, C.byref(npt), C.byref(nt), C.byref(dt), None, None, None,
                                 None)
    if st:
        raise CgfdError(st, last_error(None))
    pos = [np.zeros(npt.value) for _ in range(3)]
    mom = np.zeros((6, npt.value, nt.value), np.float32)
    st = _lib.cgfd_read_focal_nc(b, C.byref(npt), C.byref(nt), C.byref(dt), *[_d(p) for p in pos],
                                 _f(mom))
    if st:
        raise CgfdError(st, last_error(None))
    return dt.value, np.stack(pos, axis=1), mom


def angle2moment(strike, dip, rake) -> np.ndarray:
    m = np.zeros(6, np.float64)
    _lib.cgfd_angle2moment(strike, dip, rake, _d(m))
    return m
