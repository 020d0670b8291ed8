"""ctypes wrapper of the CPU oracle (liboracle.so, built from cgfd_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU legs as the checker / CPU baseline, never by the product.
The interface mirrors cgfd.Solver so that one model loader feeds both.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


if not os.path.exists(LIB_PATH):
    build()
_lib = C.CDLL(LIB_PATH)

_P = C.c_void_p
_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)
_SIGS = {
    "orc_create": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(_P)]),
    "orc_destroy": (C.c_int, [_P]),
    "orc_last_error": (C.c_int, [_P, C.c_char_p, C.c_size_t]),
    "orc_upload_metric": (C.c_int, [_P, _dp, _dp, _dp, _dp]),
    "orc_upload_media": (C.c_int, [_P, _fp, _fp, _fp]),
    "orc_upload_pml": (C.c_int, [_P] + [_dp] * 9),
    "orc_upload_moments": (C.c_int, [_P, C.c_int, _ip, _fp, C.c_int, _fp]),
    "orc_upload_forces": (C.c_int, [_P, C.c_int, _ip, _fp, C.c_int, _fp]),
    "orc_set_receivers": (C.c_int, [_P, C.c_int, _ip]),
    "orc_upload_focal": (C.c_int, [_P, C.c_int, _ip, C.c_int, C.c_double, _fp]),
    "orc_set_source_smoothing": (C.c_int, [_P, C.c_int, C.c_int, _dp]),
    "orc_rk_stage": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
    "orc_step": (C.c_int, [_P, C.c_int]),
    "orc_steps_done": (C.c_int, [_P, _ip]),
    "orc_get_seismograms": (C.c_int, [_P, _dp]),
    "orc_get_field": (C.c_int, [_P, C.c_int, C.c_int, _dp]),
    "orc_set_field": (C.c_int, [_P, C.c_int, C.c_int, _dp]),
    "orc_get_aux": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, _dp, C.POINTER(C.c_long)]),
    "orc_get_matv": (C.c_int, [_P, _dp, _dp]),
    "orc_set_storage_emulation": (C.c_int, [_P, C.c_int, C.c_int, _dp, C.c_int, C.c_int,
                                            C.c_int]),
    "orc_metric_from_coords": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double,
                                         _dp, _dp, _dp, C.POINTER(_dp)]),
    "orc_cfs_factors": (C.c_int, [C.c_int, C.c_int, C.c_int, _ip, _dp, _dp, _dp,
                                  _dp, _dp, _dp] + [_dp] * 9),
    "orc_stf": (C.c_int, [C.c_int, C.c_double, C.c_double, C.c_double, C.c_int,
                          C.c_double, _dp]),
    "orc_angle2moment": (C.c_int, [C.c_double, C.c_double, C.c_double, _dp]),
}
for _n, (_r, _a) in _SIGS.items():
    _fn = getattr(_lib, _n)
    _fn.restype = _r
    _fn.argtypes = _a


def _d(a):
    return a.ctypes.data_as(_dp)


def _f(a):
    return a.ctypes.data_as(_fp)


def _i(a):
    return a.ctypes.data_as(_ip)


class OracleError(RuntimeError):
    pass


class OracleSolver:
    """FP64 (prec=0) or FP32 (prec=1) CPU restatement of the reference path."""

    def __init__(self, desc, prec: int = 0):
        h = _P()
        st = _lib.orc_create(C.byref(desc), prec, C.byref(h))
        if st:
            raise OracleError(f"orc_create {st}: {self._err(None)}")
        self._h = h
        self.desc = desc
        self.shape = (desc.ni + 6, desc.nj + 6, desc.nk + 6)
        self.nrecv = 0

    @staticmethod
    def _err(h):
        buf = C.create_string_buffer(512)
        _lib.orc_last_error(h, buf, 512)
        return buf.value.decode()

    def _chk(self, st):
        if st:
            raise OracleError(f"oracle status {st}: {self._err(self._h)}")

    def close(self):
        if getattr(self, "_h", None):
            _lib.orc_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def upload_metric(self, zx, zy, zz, jac):
        a = [np.ascontiguousarray(v, np.float64).reshape(-1) for v in (zx, zy, zz, jac)]
        self._chk(_lib.orc_upload_metric(self._h, *[_d(v) for v in a]))

    def upload_media(self, alpha, beta, rho):
        a = [np.ascontiguousarray(v, np.float32).reshape(-1) for v in (alpha, beta, rho)]
        self._chk(_lib.orc_upload_media(self._h, *[_f(v) for v in a]))

    def upload_pml(self, apd, b, db):
        a = [np.ascontiguousarray(v, np.float64) for v in (*apd, *b, *db)]
        self._chk(_lib.orc_upload_pml(self._h, *[_d(v) for v in a]))

    def upload_moments(self, loc, m6, stf):
        loc = np.ascontiguousarray(loc, np.int32).reshape(-1, 3)
        m6 = np.ascontiguousarray(m6, np.float32).reshape(-1, 6)
        stf = np.ascontiguousarray(stf, np.float32).reshape(len(loc), -1)
        self._chk(_lib.orc_upload_moments(self._h, len(loc), _i(loc), _f(m6), stf.shape[1], _f(stf)))

    def upload_forces(self, loc, f3, stf):
        loc = np.ascontiguousarray(loc, np.int32).reshape(-1, 3)
        f3 = np.ascontiguousarray(f3, np.float32).reshape(-1, 3)
        stf = np.ascontiguousarray(stf, np.float32).reshape(len(loc), -1)
        self._chk(_lib.orc_upload_forces(self._h, len(loc), _i(loc), _f(f3), stf.shape[1], _f(stf)))

    def upload_focal(self, loc, fdt, mom):
        loc = np.ascontiguousarray(loc, np.int32).reshape(-1, 3)
        mom = np.ascontiguousarray(mom, np.float32).reshape(6, len(loc), -1)
        self._chk(_lib.orc_upload_focal(self._h, len(loc), _i(loc), mom.shape[-1], float(fdt),
                                        _f(mom)))

    def set_source_smoothing(self, kind, weights):
        """kind 0 moments, 1 forces, 2 focal points; weights [n][7][7][7]
        or None (off)."""
        if weights is None:
            self._chk(_lib.orc_set_source_smoothing(self._h, kind, 0, None))
            return
        w = np.ascontiguousarray(weights, np.float64).reshape(-1, 343)
        self._chk(_lib.orc_set_source_smoothing(self._h, kind, len(w), _d(w)))

    def set_receivers(self, loc):
        loc = np.ascontiguousarray(loc, np.int32).reshape(-1, 3)
        self._chk(_lib.orc_set_receivers(self._h, len(loc), _i(loc)))
        self.nrecv = len(loc)

    def rk_stage(self, rk, curr_t, x, y, z):
        self._chk(_lib.orc_rk_stage(self._h, rk, curr_t, x, y, z))

    def step(self, n=1):
        self._chk(_lib.orc_step(self._h, int(n)))

    def steps_done(self):
        n = C.c_int()
        self._chk(_lib.orc_steps_done(self._h, C.byref(n)))
        return n.value

    def seismograms(self):
        out = np.zeros((9, self.nrecv, self.desc.nt), np.float64)
        self._chk(_lib.orc_get_seismograms(self._h, _d(out)))
        return out

    def get_field(self, comp, fset=0):
        out = np.zeros(self.shape, np.float64)
        self._chk(_lib.orc_get_field(self._h, fset, comp, _d(out)))
        return out

    def set_field(self, comp, values, fset=0):
        v = np.ascontiguousarray(values, np.float64).reshape(self.shape)
        self._chk(_lib.orc_set_field(self._h, fset, comp, _d(v)))

    def get_aux(self, direction, aset, comp):
        n = C.c_long()
        self._chk(_lib.orc_get_aux(self._h, direction, aset, comp, None, C.byref(n)))
        out = np.zeros(n.value, np.float64)
        self._chk(_lib.orc_get_aux(self._h, direction, aset, comp, _d(out), C.byref(n)))
        return out

    def set_storage_emulation(self, ebits, mbits, scale=None, mask=7, flags=0, adapt=-1):
        """Rounds the stored field sets to an (ebits, mbits) binary format with
        per-component scales (orc_set_storage_emulation); ebits 0 = off."""
        sc = None if scale is None else np.ascontiguousarray(scale, np.float64)
        self._chk(_lib.orc_set_storage_emulation(self._h, ebits, mbits,
                                                 None if sc is None else _d(sc), mask, flags,
                                                 adapt))

    def matv(self):
        nx, ny = self.shape[0], self.shape[1]
        mx = np.zeros((nx, ny, 9), np.float64)
        my = np.zeros((nx, ny, 9), np.float64)
        self._chk(_lib.orc_get_matv(self._h, _d(mx), _d(my)))
        return mx, my


def metric_from_coords(ni, nj, nk, steph, x, y, z):
    shape = (ni + 6, nj + 6, nk + 6)
    xs = [np.ascontiguousarray(a, np.float64).reshape(shape) for a in (x, y, z)]
    names = ("xi_x", "xi_y", "xi_z", "eta_x", "eta_y", "eta_z",
             "zeta_x", "zeta_y", "zeta_z", "jac")
    outs = [np.zeros(shape, np.float64) for _ in names]
    ptrs = (_dp * 10)(*[_d(o) for o in outs])
    st = _lib.orc_metric_from_coords(ni, nj, nk, steph, *[_d(a) for a in xs], ptrs)
    if st:
        raise OracleError("metric")
    return dict(zip(names, outs))


def cfs_factors(ni, nj, nk, nabs, velabs, bmax, amax, dlx, dly, dlz):
    nabs = np.ascontiguousarray(nabs, np.int32)
    v, bm, am = (np.ascontiguousarray(a, np.float64) for a in (velabs, bmax, amax))
    dl = [np.ascontiguousarray(a, np.float64) for a in (dlx, dly, dlz)]
    n3 = (ni + 6, nj + 6, nk + 6)
    outs = [np.zeros(n3[q % 3], np.float64) for q in range(9)]
    _lib.orc_cfs_factors(ni, nj, nk, _i(nabs), _d(v), _d(bm), _d(am),
                         *[_d(a) for a in dl], *[_d(o) for o in outs])
    return tuple(outs[0:3]), tuple(outs[3:6]), tuple(outs[6:9])


def stf(kind: int, start, t0, f0, n, dt):
    out = np.zeros(n, np.float64)
    if _lib.orc_stf(kind, start, t0, f0, n, dt, _d(out)):
        raise OracleError("stf")
    return out


def angle2moment(strike, dip, rake):
    m = np.zeros(6, np.float64)
    _lib.orc_angle2moment(strike, dip, rake, _d(m))
    return m
