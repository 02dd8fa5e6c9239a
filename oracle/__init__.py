"""TEST INFRASTRUCTURE ONLY -- ctypes bindings for the CPU oracle and the reference shim.

``Oracle`` wraps ``oracle/lib/liboracle.so`` (the C restatement in ``rtm_oracle.c``).
``Reference`` wraps ``oracle/_ref/librtmref.so`` (the reference's own CPU platform, built from its
sources by ``oracle/Makefile``) and ``oracle/_ref/RTM3D.bin``.  Only the test-suite, the smoke
check and bench.py's CPU-baseline leg use this module; the product never does.

Arrays are numpy float32, C-contiguous, padded volumes in the reference layout
(x slowest, z fastest).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "lib", "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "librtmref.so")
REF_BIN = os.path.join(HERE, "_ref", "RTM3D.bin")

_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)


def build(ref: bool = True) -> None:
    """Compile the oracle (and the reference, when its sources are present)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    if ref:
        subprocess.run(["make", "-s", "-j8", "-C", HERE, "ref"], check=True)


def fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"], (a.dtype, a.flags)
    return a.ctypes.data_as(_fp)


class OrcParams(C.Structure):
    """Mirror of ``orc_params`` in rtm_oracle.h."""

    _fields_ = [(n, C.c_int) for n in ("nx", "ny", "nz", "blen", "order", "nt", "ntstep")] + \
               [(n, C.c_float) for n in ("dx", "dy", "dz", "dt", "fpeak", "taper_factor")] + \
               [(n, C.c_int) for n in ("sx", "sy", "sz", "rsx", "rsy", "rdz", "rdx", "rdy", "rcx", "rcy")]

    @classmethod
    def from_dict(cls, d: dict) -> "OrcParams":
        p = cls()
        for name, _ in cls._fields_:
            setattr(p, name, d[name])
        return p


class Oracle:
    def __init__(self, path: str = ORACLE_LIB):
        if not os.path.exists(path):
            build(ref=False)
        L = C.CDLL(path)
        self.L = L
        for name, args, res in [
            ("orc_laplacian_coefs", [C.c_int, _fp], None),
            ("orc_stencil_coefs", [C.c_int, C.c_float, C.c_float, C.c_float, _fp], None),
            ("orc_taper_vector", [C.c_int, C.c_float, _fp], None),
            ("orc_ricker", [C.c_int, C.c_float, C.c_float, _fp], None),
            ("orc_extend_borders", [_fp, C.c_int, C.c_int, C.c_int, C.c_int, _fp], None),
            ("orc_init_borders_abc", [_fp, C.c_int, C.c_int, C.c_int, C.c_int], None),
            ("orc_init_borders_rbc", [_fp, C.c_int, C.c_int, C.c_int, C.c_int], None),
            ("orc_init_borders_hbc", [_fp, C.c_int, C.c_int, C.c_int, C.c_int], None),
            ("orc_v2dt2", [_fp, C.c_size_t, C.c_float], None),
            ("orc_step", [C.c_int] * 4 + [_fp, _fp, _fp, _fp], C.c_int),
            ("orc_taper_all", [C.c_int] * 4 + [_fp, _fp], None),
            ("orc_taper_upper", [C.c_int] * 4 + [_fp, _fp], None),
            ("orc_apply_source", [C.c_int] * 6 + [C.c_float, _fp], None),
            ("orc_save_receivers", [C.POINTER(OrcParams), C.c_int, _fp, _fp], None),
            ("orc_restore_receivers", [C.POINTER(OrcParams), C.c_int, _fp, _fp], None),
            ("orc_save_upb", [C.c_int] * 6 + [_fp, _fp], None),
            ("orc_restore_upb", [C.c_int] * 6 + [_fp, _fp], None),
            ("orc_image", [C.c_int] * 4 + [_fp, _fp, _fp], None),
            ("orc_filter_remove", [C.c_int] * 4 + [C.c_float] * 3 + [_fp, _fp], None),
            ("orc_model_shot", [C.POINTER(OrcParams), _fp, _fp], C.c_int),
            ("orc_migrate_hbc", [C.POINTER(OrcParams), _fp, _fp, _fp], C.c_int),
            ("orc_migrate_rbc", [C.POINTER(OrcParams), _fp, _fp, _fp], C.c_int),
            ("orc_step2d", [C.c_int] * 5 + [_fp, _fp, _fp, _fp], C.c_int),
            ("orc_fmig_nw", [C.c_int, C.c_float, C.c_float, C.c_float], C.c_int),
            ("orc_fmig_tables", [C.c_int, C.c_float, C.c_float, C.c_float, C.c_int, _fp, _fp, _fp], None),
            ("orc_migrate_fmig", [C.POINTER(OrcParams), _fp, _fp, C.c_float, C.c_float, C.c_int, _fp], C.c_int),
        ]:
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res

    # host math -------------------------------------------------------------
    def stencil_coefs(self, order, dx, dy, dz):
        out = np.zeros(3 * (order + 1), np.float32)
        self.L.orc_stencil_coefs(order, dx, dy, dz, fptr(out))
        return out

    def taper_vector(self, blen, factor):
        out = np.zeros(blen, np.float32)
        self.L.orc_taper_vector(blen, factor, fptr(out))
        return out

    def ricker(self, nt, dt, fpeak):
        out = np.zeros(nt, np.float32)
        self.L.orc_ricker(nt, dt, fpeak, fptr(out))
        return out

    # velocity --------------------------------------------------------------
    def extend_init_borders(self, v: np.ndarray, blen: int, bc: str, seed: int | None = None):
        nx, ny, nz = v.shape
        ve = np.zeros((nx + 2 * blen, ny + 2 * blen, nz + 2 * blen), np.float32)
        self.L.orc_extend_borders(fptr(np.ascontiguousarray(v, np.float32)), nx, ny, nz, blen, fptr(ve))
        if seed is not None:
            C.CDLL(None).srand(C.c_uint(seed))
        fn = {"abc": self.L.orc_init_borders_abc, "rbc": self.L.orc_init_borders_rbc,
              "hbc": self.L.orc_init_borders_hbc, "none": None}[bc]
        if fn is not None:
            fn(fptr(ve), *ve.shape, blen)
        return ve

    def v2dt2(self, ve: np.ndarray, dt: float):
        out = np.ascontiguousarray(ve, np.float32).copy()
        self.L.orc_v2dt2(fptr(out), out.size, dt)
        return out

    # operators -------------------------------------------------------------
    def step(self, order, coefs, P, PP, v2dt2):
        PP = PP.copy()
        nan = self.L.orc_step(*P.shape, order, fptr(coefs), fptr(P), fptr(PP), fptr(v2dt2))
        return PP, nan

    def step2d(self, order, coefs, P, PP, v2dt2, blen):
        PP = PP.copy()
        nan = self.L.orc_step2d(*P.shape, blen, order, fptr(coefs), fptr(P), fptr(PP), fptr(v2dt2))
        return PP, nan

    def taper(self, g, blen, taper, upper=False):
        g = g.copy()
        (self.L.orc_taper_upper if upper else self.L.orc_taper_all)(*g.shape, blen, fptr(taper), fptr(g))
        return g

    def image(self, img, ps, pr, blen):
        img = img.copy()
        self.L.orc_image(*img.shape, blen, fptr(img), fptr(ps), fptr(pr))
        return img

    def filter_remove(self, img, blen, dx, dy, dz):
        nxe, nye, nze = img.shape
        out = np.zeros((nxe - 2 * blen, nye - 2 * blen, nze - 2 * blen), np.float32)
        self.L.orc_filter_remove(nxe, nye, nze, blen, dx, dy, dz, fptr(img), fptr(out))
        return out

    # loops -----------------------------------------------------------------
    def model_shot(self, p: dict, v2dt2: np.ndarray):
        op = OrcParams.from_dict(p)
        rec = np.zeros((p["nt"] // p["ntstep"], p["rcx"], p["rcy"], p["ntstep"]), np.float32)
        rc = self.L.orc_model_shot(C.byref(op), fptr(v2dt2), fptr(rec))
        return rec, rc

    def migrate(self, p: dict, v2dt2: np.ndarray, rec: np.ndarray, bc: str):
        op = OrcParams.from_dict(p)
        img = np.zeros(v2dt2.shape, np.float32)
        fn = self.L.orc_migrate_hbc if bc == "hbc" else self.L.orc_migrate_rbc
        rc = fn(C.byref(op), fptr(v2dt2), fptr(np.ascontiguousarray(rec, np.float32)), fptr(img))
        return img, rc

    def fmig_tables(self, nt: int, dt: float, fmin: float, fmax: float):
        nw = self.L.orc_fmig_nw(nt, dt, fmin, fmax)
        w2 = np.zeros(max(nw, 1), np.float32)
        kre = np.zeros((max(nw, 1), nt), np.float32)
        kim = np.zeros((max(nw, 1), nt), np.float32)
        self.L.orc_fmig_tables(nt, dt, fmin, fmax, nw, fptr(w2), fptr(kre), fptr(kim))
        return w2[:nw], kre[:nw], kim[:nw]

    def migrate_fmig(self, p: dict, v2dt2: np.ndarray, rec: np.ndarray, fmin: float, fmax: float, nwstep: int = 0):
        op = OrcParams.from_dict(p)
        img = np.zeros(v2dt2.shape, np.float32)
        rc = self.L.orc_migrate_fmig(C.byref(op), fptr(v2dt2), fptr(np.ascontiguousarray(rec, np.float32)),
                                     fmin, fmax, nwstep, fptr(img))
        return img, rc


class Reference:
    """The reference's own CPU operators (built from its sources into oracle/_ref/)."""

    def __init__(self, path: str = REF_LIB):
        L = C.CDLL(path)
        self.L = L
        for name, args, res in [
            ("ref_set_threads", [C.c_int], None),
            ("ref_srand", [C.c_uint], None),
            ("ref_stencil_coefs", [C.c_int, C.c_float, C.c_float, C.c_float, _fp], None),
            ("ref_taper_vector", [C.c_int, C.c_float, _fp], None),
            ("ref_ricker", [C.c_int, C.c_float, C.c_float, _fp], None),
            ("ref_step", [C.c_int] * 5 + [C.c_float] * 3 + [_fp, _fp, _fp], C.c_int),
            ("ref_taper", [C.c_int] * 5 + [C.c_float, _fp], None),
            ("ref_apply_source", [C.c_int] * 8 + [C.c_float, C.c_float, C.c_int, _fp], None),
            ("ref_save_receivers", [C.c_int] * 4 + [_ip, C.c_int, C.c_int, _fp, _fp], None),
            ("ref_restore_receivers", [C.c_int] * 4 + [_ip, C.c_int, C.c_int, _fp, _fp], None),
            ("ref_upb", [C.c_int] * 8 + [_fp, _fp], None),
            ("ref_image", [C.c_int] * 4 + [_fp, _fp, _fp], None),
            ("ref_extend_init_borders", [C.c_int] * 5 + [_fp, _fp], None),
            ("ref_filter_remove", [C.c_int] * 4 + [C.c_float] * 3 + [_fp, _fp], None),
        ]:
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res

    @staticmethod
    def available() -> bool:
        return os.path.exists(REF_LIB) and os.path.exists(REF_BIN)

    def stencil_coefs(self, order, dx, dy, dz):
        out = np.zeros(3 * (order + 1), np.float32)
        self.L.ref_stencil_coefs(order, dx, dy, dz, fptr(out))
        return out

    def taper_vector(self, blen, factor):
        out = np.zeros(blen, np.float32)
        self.L.ref_taper_vector(blen, factor, fptr(out))
        return out

    def ricker(self, nt, dt, fpeak):
        out = np.zeros(nt, np.float32)
        self.L.ref_ricker(nt, dt, fpeak, fptr(out))
        return out

    def step(self, nx, ny, nz, blen, order, dx, dy, dz, P, PP, v2dt2):
        PP = PP.copy()
        rc = self.L.ref_step(nx, ny, nz, blen, order, dx, dy, dz, fptr(P), fptr(PP), fptr(v2dt2))
        return PP, rc

    def taper(self, g, nx, ny, nz, blen, factor, upper=False):
        g = g.copy()
        self.L.ref_taper(int(upper), nx, ny, nz, blen, factor, fptr(g))
        return g

    def image(self, img, ps, pr, nx, ny, nz, blen):
        img = img.copy()
        self.L.ref_image(nx, ny, nz, blen, fptr(img), fptr(ps), fptr(pr))
        return img

    def extend_init_borders(self, v, blen, bc: str, seed: int | None = None):
        nx, ny, nz = v.shape
        ve = np.zeros((nx + 2 * blen, ny + 2 * blen, nz + 2 * blen), np.float32)
        if seed is not None:
            self.L.ref_set_threads(1)
            self.L.ref_srand(seed)
        code = {"none": 0, "abc": 1, "hbc": 2, "rbc": 3}[bc]
        self.L.ref_extend_init_borders(nx, ny, nz, blen, code, fptr(np.ascontiguousarray(v, np.float32)), fptr(ve))
        return ve

    def filter_remove(self, img, blen, dx, dy, dz):
        nxe, nye, nze = img.shape
        out = np.zeros((nxe - 2 * blen, nye - 2 * blen, nze - 2 * blen), np.float32)
        self.L.ref_filter_remove(nxe, nye, nze, blen, dx, dy, dz, fptr(img), fptr(out))
        return out
