"""ctypes binding of librtm3d_b200.so (the C ABI declared in include/rtm3d_b200.h).

The library does all the work on the GPU; this module only marshals arguments.  Device buffers are
passed as raw pointers, so any CUDA allocator works (the tests and bench.py use torch tensors).
Importing the module never falls back to anything: if the shared library is missing or fails to
load, ``load()`` raises.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

PKG_ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
# the in-tree build; RTMB_LIB names another build of the same library (for example one made with
# other compile-time tuning: make -C rtm3d-demo_b200 NVCC="nvcc -DRTMB_PLANE_UNROLL=1" LIB=...)
LIB_PATH = os.environ.get("RTMB_LIB") or os.path.join(PKG_ROOT, "lib", "librtm3d_b200.so")
BIN_PATH = os.path.join(PKG_ROOT, "bin", "rtm3d_b200")

RTMB_OK, RTMB_EINVAL, RTMB_ENOMEM, RTMB_ECUDA, RTMB_ENAN, RTMB_ETIMEOUT, RTMB_EIO = range(7)
BC = {"abc": 1, "hbc": 2, "rbc": 3}
FLAG_FAST_FMA = 0x1
FLAG_RCV_ADD = 0x2
FLAG_IMG_FULL_Z = 0x4
FLAG_NO_TAPER_QUIRK = 0x8
FLAG_USE_GRAPH = 0x10
FLAG_NO_TMA = 0x20
FLAG_STORE_F16 = 0x40
FLAG_STORE_BF16 = 0x80
FLAG_IMG_F64 = 0x100
FLAG_NO_DUAL = 0x200
FLAG_NO_TAPER_STORE = 0x400
FLAG_STORE_DIFF = 0x800
BC_ABC, BC_HBC, BC_RBC, BC_LEARNED = 1, 2, 3, 4
CLOSURE_NPARAM, CLOSURE_NIN = 3169, 64

# every symbol include/rtm3d_b200.h declares: (name, argtypes, restype)
_vp, _fp, _u32, _i32 = C.c_void_p, C.POINTER(C.c_float), C.c_uint32, C.c_int32


class RtmbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"rtmb error {code}: {msg}")
        self.code = code


class Params(C.Structure):
    _fields_ = [
        ("nx", _u32), ("ny", _u32), ("nz", _u32), ("blen", _u32), ("nt", _u32), ("ntstep", _u32),
        ("stencil_order", _u32),
        ("dx", C.c_float), ("dy", C.c_float), ("dz", C.c_float), ("dt", C.c_float),
        ("fpeak", C.c_float), ("taper_factor", C.c_float),
        ("receiver_start_x", _u32), ("receiver_start_y", _u32), ("receiver_depth_z", _u32),
        ("receiver_distance_x", _u32), ("receiver_distance_y", _u32),
        ("receiver_count_x", _u32), ("receiver_count_y", _u32),
        ("boundary", _i32), ("flags", _u32), ("device", _i32),
    ]

    @classmethod
    def from_input(cls, d: dict, flags: int = 0, device: int = -1) -> "Params":
        """Build from input.json keys (RTMParam names)."""
        p = cls()
        for k in ("nx", "ny", "nz", "blen", "nt", "ntstep", "stencil_order", "dx", "dy", "dz", "dt",
                  "fpeak", "taper_factor", "receiver_start_x", "receiver_start_y", "receiver_depth_z",
                  "receiver_distance_x", "receiver_distance_y", "receiver_count_x", "receiver_count_y"):
            setattr(p, k, d[k])
        p.boundary = BC.get(str(d.get("boundary_condition", "hbc")).lower(), BC["hbc"])
        p.flags = flags
        p.device = device
        return p


SYMBOLS = [
    ("rtmb_abi_version", [], C.c_int),
    ("rtmb_create", [C.POINTER(Params), C.POINTER(_vp)], C.c_int),
    ("rtmb_destroy", [_vp], C.c_int),
    ("rtmb_last_error", [_vp], C.c_char_p),
    ("rtmb_set_stream", [_vp, _vp], C.c_int),
    ("rtmb_sync", [_vp], C.c_int),
    ("rtmb_launch_count", [_vp], C.c_uint64),
    ("rtmb_profile", [_vp, C.c_int], C.c_int),
    ("rtmb_profile_read", [_vp, C.POINTER(C.c_double), C.POINTER(C.c_uint64)], C.c_int),
    ("rtmb_stencil_coefs", [_u32, C.c_float, C.c_float, C.c_float, _fp], C.c_int),
    ("rtmb_taper_vector", [_u32, C.c_float, _fp], C.c_int),
    ("rtmb_ricker", [_u32, C.c_float, C.c_float, _fp], C.c_int),
    ("rtmb_prepare_velocity", [_fp, _u32, _u32, _u32, _u32, _i32, C.c_int64, _fp], C.c_int),
    ("rtmb_v2dt2_host", [_fp, C.c_size_t, C.c_float], C.c_int),
    ("rtmb_step", [_vp, _vp, _vp, _vp], C.c_int),
    ("rtmb_taper_all_borders", [_vp, _vp], C.c_int),
    ("rtmb_taper_upper_borders", [_vp, _vp], C.c_int),
    ("rtmb_apply_source", [_vp, _vp, _u32, _u32, _u32, _u32], C.c_int),
    ("rtmb_save_receiver_data", [_vp, _vp, _vp, _u32], C.c_int),
    ("rtmb_restore_receiver_data", [_vp, _vp, _vp, _u32], C.c_int),
    ("rtmb_save_upper_border", [_vp, _vp, _vp, _u32], C.c_int),
    ("rtmb_restore_upper_border", [_vp, _vp, _vp, _u32], C.c_int),
    ("rtmb_image_condition", [_vp, _vp, _vp, _vp], C.c_int),
    ("rtmb_image_finalize", [_vp, _vp, _vp], C.c_int),
    ("rtmb_image_stack", [_vp, _vp, _vp], C.c_int),
    ("rtmb_load_v2dt2", [_vp, _vp, C.c_int], C.c_int),
    ("rtmb_model_shot", [_vp, _u32, _u32, _u32, _vp], C.c_int),
    ("rtmb_migrate_shot", [_vp, _u32, _u32, _u32, _vp, _vp], C.c_int),
    ("rtmb_model_shot_host", [_vp, _u32, _u32, _u32, _vp], C.c_int),
    ("rtmb_migrate_shot_host", [_vp, _u32, _u32, _u32, _vp, _vp], C.c_int),
    ("rtmb_model_shot_noalloc", [C.POINTER(Params), _vp, _u32, _u32, _u32, _vp, _vp], C.c_int),
    ("rtmb_migrate_shot_acc64", [_vp, _u32, _u32, _u32, _vp, _vp], C.c_int),
    ("rtmb_migrate_shot_fmig", [_vp, _u32, _u32, _u32, _vp, C.c_float, C.c_float, _u32, _vp], C.c_int),
    ("rtmb_fmig_nw", [C.c_float, _u32, C.c_float, C.c_float], C.c_int),
    ("rtmb_fmig_tables", [C.c_float, _u32, C.c_float, C.c_float, _vp, _vp, _vp], C.c_int),
    ("rtmb_step_multiwave", [_vp, _vp, _vp, _vp, _vp, _vp], C.c_int),
    ("rtmb_fmig_update_freq", [_vp, _u32, _u32, _u32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp], C.c_int),
    ("rtmb_fmig_image_condition", [_vp, _u32, _u32, _vp, _vp, _vp, _vp, _vp, _vp], C.c_int),
    ("rtmb_model_shot_f64", [_vp, _u32, _u32, _u32, _vp], C.c_int),
    ("rtmb_migrate_shot_f64", [_vp, _u32, _u32, _u32, _vp, _vp], C.c_int),
    ("rtmb_closure_param_count", [], C.c_int),
    ("rtmb_closure_init", [_fp, C.c_uint64], C.c_int),
    ("rtmb_closure_forward", [_vp, _vp, C.c_uint64, _vp, _vp], C.c_int),
    ("rtmb_closure_grad", [_vp, _vp, _vp, _u32, _vp, _vp, _vp], C.c_int),
    ("rtmb_closure_train", [_vp, _vp, _vp, C.c_uint64, _u32, _u32, C.c_float, C.c_float, C.c_uint64, _fp, _vp],
     C.c_int),
    ("rtmb_closure_collect", [_vp, _u32, _u32, _u32, _u32, _u32, _u32, C.c_uint64, C.c_float, _vp, _vp,
                              C.c_uint64, C.POINTER(C.c_uint64)], C.c_int),
    ("rtmb_closure_set", [_vp, _vp, C.c_float, C.c_float], C.c_int),
    ("rtmb_autotune", [_vp, C.POINTER(_u32), C.POINTER(C.c_float)], C.c_int),
    ("rtmb_autotune_full", [_vp, _vp], C.c_int),
    ("rtmb_closure_judge", [_vp, _vp, _vp, _u32, _u32, _u32, C.POINTER(C.c_float), C.POINTER(C.c_float)], C.c_int),
    ("rtmb_model_shot_judged", [_vp, _vp, _u32, _u32, _u32, _vp, C.POINTER(_i32)], C.c_int),
    ("rtmb_set_batch_group", [_vp, _u32], C.c_int),
    ("rtmb_autotune_batch", [_vp, _u32, _vp, C.POINTER(_u32), C.POINTER(C.c_float)], C.c_int),
    ("rtmb_set_tuning", [_vp, _vp], C.c_int),
    ("rtmb_migrate_batch", [_vp, _u32, _vp, _vp, _u32, _u32, _u32], C.c_int),
    ("rtmb_set_chunk", [_vp, _u32], C.c_int),
]

_LIB = None


def build() -> None:
    """Compile librtm3d_b200.so (and the CLI) for sm_100a."""
    subprocess.run(["make", "-s", "-j8", "-C", PKG_ROOT], check=True)


def load(path: str = LIB_PATH):
    """Load the shared library and bind every declared symbol; raises if anything is missing."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built; run rtmb.build() (make -C rtm3d-demo_b200)")
    lib = C.CDLL(path)
    for name, args, res in SYMBOLS:
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _LIB = lib
    return lib


def _ptr(t) -> int:
    """Device (or host) address of a torch tensor / numpy array / int."""
    if t is None:
        return None
    if isinstance(t, int):
        return t
    if hasattr(t, "cuda_stream"):
        return t.cuda_stream
    if hasattr(t, "data_ptr"):
        return t.data_ptr()
    return t.ctypes.data


class Tuning(C.Structure):
    """rtmb_tuning: the launch choices rtmb_autotune_full measured for a context."""
    _fields_ = [("variant", _u32), ("chunk", _u32), ("dual", _u32), ("dual_chunk", _u32),
                ("ms_step", C.c_float), ("ms_backward", C.c_float), ("dual_variant", _u32)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Shot(C.Structure):
    """rtmb_shot: one shot of a batch (aperture geometry, source, receivers, device buffers)."""
    _fields_ = [
        ("nx", _u32), ("ny", _u32), ("nz", _u32), ("ox", _u32), ("oy", _u32), ("oz", _u32),
        ("sx", _u32), ("sy", _u32), ("sz", _u32),
        ("receiver_start_x", _u32), ("receiver_start_y", _u32), ("receiver_depth_z", _u32),
        ("receiver_distance_x", _u32), ("receiver_distance_y", _u32),
        ("receiver_count_x", _u32), ("receiver_count_y", _u32),
        ("v2dt2", _vp), ("rec", _vp),
    ]


class Context:
    """One rtmb_ctx: the context of one shot geometry on one device."""

    def __init__(self, params: Params, stream=None):
        self.L = load()
        self.params = params
        h = _vp()
        rc = self.L.rtmb_create(C.byref(params), C.byref(h))
        if rc != RTMB_OK:
            raise RtmbError(rc, "rtmb_create failed: " + self.L.rtmb_last_error(None).decode())
        self.h = h
        if stream is not None:
            self._check(self.L.rtmb_set_stream(self.h, _ptr(stream) if not isinstance(stream, int) else stream))

    def _check(self, rc: int) -> None:
        if rc != RTMB_OK:
            raise RtmbError(rc, self.L.rtmb_last_error(self.h).decode())

    def close(self) -> None:
        if getattr(self, "h", None):
            self.L.rtmb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # properties -------------------------------------------------------------
    @property
    def padded_shape(self):
        p = self.params
        return (p.nx + 2 * p.blen, p.ny + 2 * p.blen, p.nz + 2 * p.blen)

    @property
    def launches(self) -> int:
        return int(self.L.rtmb_launch_count(self.h))

    PROF_NAMES = ("model", "forward", "backward_source", "backward_receiver", "other", "backward_dual",
                  "fmig_step", "fmig_freq")

    def profile(self, enable: bool = True) -> None:
        """Time every driver launch with CUDA events (per category); enabling clears the totals."""
        self._check(self.L.rtmb_profile(self.h, int(enable)))

    def profile_read(self) -> dict:
        ms = (C.c_double * len(self.PROF_NAMES))()
        n = (C.c_uint64 * len(self.PROF_NAMES))()
        self._check(self.L.rtmb_profile_read(self.h, ms, n))
        return {name: {"ms": ms[k], "launches": int(n[k])} for k, name in enumerate(self.PROF_NAMES)}

    def set_stream(self, stream) -> None:
        self._check(self.L.rtmb_set_stream(self.h, stream))

    def sync(self) -> None:
        self._check(self.L.rtmb_sync(self.h))

    # per-step operators ------------------------------------------------------
    def step(self, P, PP, V):
        self._check(self.L.rtmb_step(self.h, _ptr(P), _ptr(PP), _ptr(V)))

    def taper_all(self, P):
        self._check(self.L.rtmb_taper_all_borders(self.h, _ptr(P)))

    def taper_upper(self, P):
        self._check(self.L.rtmb_taper_upper_borders(self.h, _ptr(P)))

    def apply_source(self, PP, sx, sy, sz, it):
        self._check(self.L.rtmb_apply_source(self.h, _ptr(PP), sx, sy, sz, it))

    def save_receivers(self, PP, rec, lt):
        self._check(self.L.rtmb_save_receiver_data(self.h, _ptr(PP), _ptr(rec), lt))

    def restore_receivers(self, PP, rec, lt):
        self._check(self.L.rtmb_restore_receiver_data(self.h, _ptr(PP), _ptr(rec), lt))

    def save_upb(self, P, upb, lt):
        self._check(self.L.rtmb_save_upper_border(self.h, _ptr(P), _ptr(upb), lt))

    def restore_upb(self, P, upb, lt):
        self._check(self.L.rtmb_restore_upper_border(self.h, _ptr(P), _ptr(upb), lt))

    def image(self, img, ps, pr):
        self._check(self.L.rtmb_image_condition(self.h, _ptr(img), _ptr(ps), _ptr(pr)))

    def image_finalize(self, img, out):
        self._check(self.L.rtmb_image_finalize(self.h, _ptr(img), _ptr(out)))

    def image_stack(self, acc, img):
        self._check(self.L.rtmb_image_stack(self.h, _ptr(acc), _ptr(img)))

    # drivers -----------------------------------------------------------------
    def load_v2dt2(self, v2dt2, from_host: bool):
        self._check(self.L.rtmb_load_v2dt2(self.h, _ptr(v2dt2), int(from_host)))

    def model_shot(self, sx, sy, sz, rec):
        self._check(self.L.rtmb_model_shot(self.h, sx, sy, sz, _ptr(rec)))

    def migrate_shot(self, sx, sy, sz, rec, img):
        self._check(self.L.rtmb_migrate_shot(self.h, sx, sy, sz, _ptr(rec), _ptr(img)))

    def step_multiwave(self, P0, PP0, P1, PP1, v2dt2):
        self._check(self.L.rtmb_step_multiwave(self.h, _ptr(P0), _ptr(PP0), _ptr(P1), _ptr(PP1), _ptr(v2dt2)))

    def fmig_update_freq(self, it, iw, lw, ps, pr, sre, sim, rre, rim, kre, kim):
        self._check(self.L.rtmb_fmig_update_freq(self.h, it, iw, lw, _ptr(ps), _ptr(pr), _ptr(sre), _ptr(sim),
                                                  _ptr(rre), _ptr(rim), _ptr(kre), _ptr(kim)))

    def fmig_image_condition(self, iw, lw, w2, img, sre, sim, rre, rim):
        self._check(self.L.rtmb_fmig_image_condition(self.h, iw, lw, _ptr(w2), _ptr(img), _ptr(sre), _ptr(sim),
                                                      _ptr(rre), _ptr(rim)))

    def migrate_shot_fmig(self, sx, sy, sz, rec, img, fmin, fmax, nwstep=0):
        """Frequency-domain RTM of one shot into img (padded, device, float32, overwritten)."""
        self._check(self.L.rtmb_migrate_shot_fmig(self.h, sx, sy, sz, _ptr(rec), fmin, fmax, nwstep, _ptr(img)))

    def migrate_shot_acc64(self, sx, sy, sz, rec, stack):
        """Adds this shot's image to an FP64 stack (padded, device, float64)."""
        self._check(self.L.rtmb_migrate_shot_acc64(self.h, sx, sy, sz, _ptr(rec), _ptr(stack)))

    def model_shot_f64(self, sx, sy, sz, rec64):
        """FP64 GPU oracle modeling: rec64 is a float64 device record in file layout."""
        self._check(self.L.rtmb_model_shot_f64(self.h, sx, sy, sz, _ptr(rec64)))

    def migrate_shot_f64(self, sx, sy, sz, rec, img64):
        """FP64 GPU oracle migration: rec float32, img64 float64 padded image (overwritten)."""
        self._check(self.L.rtmb_migrate_shot_f64(self.h, sx, sy, sz, _ptr(rec), _ptr(img64)))

    def closure_set(self, params, min_scale: float = 0.0, damp: float = 0.0):
        """Installs the learned closure (device or host float32 params) in a BC_LEARNED context."""
        self._check(self.L.rtmb_closure_set(self.h, _ptr(params), min_scale, damp))

    def closure_judge(self, hbc: "Context", wide: "Context", sx: int, sy: int, sz: int):
        """Judges this learned context against the taper border (rtmb_closure_judge); returns
        (reflection of the learned strip, reflection of the taper border, passed)."""
        rl, rh = C.c_float(0), C.c_float(0)
        self._check(self.L.rtmb_closure_judge(self.h, hbc.h, wide.h, sx, sy, sz, C.byref(rl), C.byref(rh)))
        return float(rl.value), float(rh.value), bool(rl.value <= rh.value)

    def model_shot_judged(self, fallback: "Context", sx: int, sy: int, sz: int, rec) -> int:
        """Modeling with the judged boundary; returns the boundary that ran (BC_LEARNED or the
        fallback's)."""
        ran = _i32(0)
        self._check(self.L.rtmb_model_shot_judged(self.h, fallback.h, sx, sy, sz, _ptr(rec), C.byref(ran)))
        return int(ran.value)

    def closure_collect(self, sx, sy, sz, t0, tstride, per_step, seed, min_scale, X, R) -> int:
        """Training pairs from a modeling shot on this (wide) context; returns the row count."""
        cnt = C.c_uint64(0)
        self._check(self.L.rtmb_closure_collect(self.h, sx, sy, sz, t0, tstride, per_step, seed, min_scale,
                                                _ptr(X), _ptr(R), R.numel(), C.byref(cnt)))
        return int(cnt.value)

    def migrate_batch(self, shots, stack):
        """shots: list of Shot; stack: float64 survey volume (device), added to."""
        arr = (Shot * len(shots))(*shots)
        nx, ny, nz = stack.shape
        self._check(self.L.rtmb_migrate_batch(self.h, len(shots), C.cast(arr, _vp), _ptr(stack), nx, ny, nz))

    def set_batch_group(self, shots_per_launch: int) -> None:
        self._check(self.L.rtmb_set_batch_group(self.h, shots_per_launch))

    def autotune_batch(self, shots):
        """Picks the shots per launch of migrate_batch; returns (group size, G point-updates/s)."""
        arr = (Shot * len(shots))(*shots)
        g, r = _u32(0), C.c_float(0)
        self._check(self.L.rtmb_autotune_batch(self.h, len(shots), C.cast(arr, _vp), C.byref(g), C.byref(r)))
        return int(g.value), float(r.value)

    def autotune(self):
        """Picks the fastest x-chunk length for this context; returns (chunk, ms per step)."""
        c, ms = _u32(0), C.c_float(0)
        self._check(self.L.rtmb_autotune(self.h, C.byref(c), C.byref(ms)))
        return int(c.value), float(ms.value)

    def autotune_full(self) -> dict:
        """Picks the launch variant (tile shape, ring depths), the x-chunk lengths, the dual backward
        step's variant (split or merged form, tile, ring depths) and the dual step or two launches
        for this context; returns the rtmb_tuning fields."""
        t = Tuning()
        self._check(self.L.rtmb_autotune_full(self.h, C.byref(t)))
        return t.as_dict()

    # the library's own choice for a field the caller leaves out (dual_variant 5: the merged dual step)
    TUNING_DEFAULTS = {"dual_variant": 5}

    def set_tuning(self, t: dict) -> None:
        """Applies rtmb_tuning fields (as autotune_full returns them); a missing field is 0, except
        dual_variant, which keeps the library's default."""
        tt = Tuning(**{k: t.get(k, self.TUNING_DEFAULTS.get(k, 0)) for k, _ in Tuning._fields_})
        self._check(self.L.rtmb_set_tuning(self.h, C.byref(tt)))

    def set_chunk(self, chunk: int):
        self._check(self.L.rtmb_set_chunk(self.h, chunk))

    def model_shot_host(self, sx, sy, sz, rec_host):
        self._check(self.L.rtmb_model_shot_host(self.h, sx, sy, sz, _ptr(rec_host)))

    def migrate_shot_host(self, sx, sy, sz, rec_host, img_host):
        self._check(self.L.rtmb_migrate_shot_host(self.h, sx, sy, sz, _ptr(rec_host), _ptr(img_host)))


def model_shot_noalloc(params: Params, v2dt2, sx: int, sy: int, sz: int, rec, stream=None) -> None:
    """Modeling through rtmb_model_shot_noalloc: no context and no device allocation (v2dt2 and rec
    are device buffers the caller owns; the library's fixed 64 MiB scratch holds everything else)."""
    L = load()
    rc = L.rtmb_model_shot_noalloc(C.byref(params), _ptr(v2dt2), sx, sy, sz, _ptr(rec), stream)
    if rc != RTMB_OK:
        raise RtmbError(rc, L.rtmb_last_error(None).decode())


# host-side tables (no GPU needed) ----------------------------------------------
def _np():
    import numpy as np
    return np


def stencil_coefs(order, dx, dy, dz):
    np = _np()
    out = np.zeros(3 * (order + 1), np.float32)
    rc = load().rtmb_stencil_coefs(order, dx, dy, dz, out.ctypes.data_as(_fp))
    if rc:
        raise RtmbError(rc, "rtmb_stencil_coefs")
    return out


def taper_vector(blen, factor):
    np = _np()
    out = np.zeros(max(blen, 1), np.float32)
    load().rtmb_taper_vector(blen, factor, out.ctypes.data_as(_fp))
    return out[:blen]


def ricker(nt, dt, fpeak):
    np = _np()
    out = np.zeros(nt, np.float32)
    load().rtmb_ricker(nt, dt, fpeak, out.ctypes.data_as(_fp))
    return out


def fmig_nw(dt: float, nt: int, fmin: float, fmax: float) -> int:
    """Number of frequencies of a frequency-domain migration (0 when there is none)."""
    return int(load().rtmb_fmig_nw(dt, nt, fmin, fmax))


def fmig_tables(dt: float, nt: int, fmin: float, fmax: float):
    """(w2[nw], kre[nw][nt], kim[nw][nt]) of a frequency-domain migration."""
    np = _np()
    nw = fmig_nw(dt, nt, fmin, fmax)
    w2 = np.zeros(max(nw, 1), np.float32)
    kre = np.zeros((max(nw, 1), nt), np.float32)
    kim = np.zeros((max(nw, 1), nt), np.float32)
    load().rtmb_fmig_tables(dt, nt, fmin, fmax, w2.ctypes.data, kre.ctypes.data, kim.ctypes.data)
    return w2[:nw], kre[:nw], kim[:nw]


def prepare_velocity(v, blen: int, bc: str, seed: int = -1):
    """extendBorders + initBorders on the host; bc in {'none', 'abc', 'hbc', 'rbc'}."""
    np = _np()
    v = np.ascontiguousarray(v, np.float32)
    nx, ny, nz = v.shape
    ve = np.zeros((nx + 2 * blen, ny + 2 * blen, nz + 2 * blen), np.float32)
    code = 0 if bc == "none" else BC[bc]
    rc = load().rtmb_prepare_velocity(v.ctypes.data_as(_fp), nx, ny, nz, blen, code, seed, ve.ctypes.data_as(_fp))
    if rc:
        raise RtmbError(rc, "rtmb_prepare_velocity")
    return ve


def v2dt2(ve, dt):
    np = _np()
    out = np.ascontiguousarray(ve, np.float32).copy()
    load().rtmb_v2dt2_host(out.ctypes.data_as(_fp), out.size, dt)
    return out


# ---------------------------------------------------------------- learned boundary closure (no context)
def _check_noctx(rc: int) -> None:
    if rc != RTMB_OK:
        raise RtmbError(rc, load().rtmb_last_error(None).decode())


def closure_init(seed: int):
    """Seeded initial parameters (numpy float32, CLOSURE_NPARAM)."""
    import numpy as np
    p = np.zeros(CLOSURE_NPARAM, np.float32)
    _check_noctx(load().rtmb_closure_init(p.ctypes.data_as(C.POINTER(C.c_float)), seed))
    return p


def closure_forward(params, X, y, stream=None) -> None:
    """y = network(X); params float32, X bfloat16 [n, 64], y float32 [n] (device tensors)."""
    _check_noctx(load().rtmb_closure_forward(_ptr(params), _ptr(X), X.shape[0], _ptr(y), _ptr(stream)))


def closure_grad(params, X, R, grad, loss, stream=None) -> None:
    _check_noctx(load().rtmb_closure_grad(_ptr(params), _ptr(X), _ptr(R), X.shape[0], _ptr(grad), _ptr(loss),
                                          _ptr(stream)))


def closure_train(params, X, R, n: int, steps: int, batch: int, lr: float, seed: int, noise: float = 0.0,
                  stream=None):
    """Adam training in place; returns the per-step batch losses (numpy)."""
    import numpy as np
    losses = np.zeros(steps, np.float32)
    _check_noctx(load().rtmb_closure_train(_ptr(params), _ptr(X), _ptr(R), n, steps, batch, lr, noise, seed,
                                           losses.ctypes.data_as(C.POINTER(C.c_float)), _ptr(stream)))
    return losses


def closure_falls_back(learned_reflection: float, hbc_reflection: float) -> bool:
    """The fallback test of the learned closure: a run falls back to the plain 32-cell border when the
    closure's reflected energy (record rel-L2 against a wide-padded run of the same shot) exceeds
    the 32-cell border's."""
    return not (learned_reflection <= hbc_reflection)
