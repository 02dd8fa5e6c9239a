"""CPU tests of librtm3d_b200.so: it loads, exports every declared symbol, and its host-side tables
and velocity preparation are bit-identical to the oracle (no GPU calls here)."""
import os
import re

import numpy as np
import pytest

import rtmb
from rtm_cases import bitexact

HEADER = os.path.join(os.path.dirname(__file__), "..", "include", "rtm3d_b200.h")


def declared_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char \*|uint64_t)\s*\*?\s*(rtmb_\w+)\s*\(", src, re.M)))


def test_library_exports_every_declared_symbol():
    lib = rtmb.load()
    names = declared_symbols()
    assert len(names) >= 25, names
    bound = {n for n, _, _ in rtmb.SYMBOLS}
    for n in names:
        assert hasattr(lib, n), n
        assert n in bound, f"{n} missing from the Python binding"
    assert lib.rtmb_abi_version() == 2


@pytest.mark.parametrize("order", [2, 4, 6, 8, 10, 12, 14, 16])
def test_stencil_coefs(oracle, order):
    assert bitexact(rtmb.stencil_coefs(order, 10.0, 12.5, 6.25), oracle.stencil_coefs(order, 10.0, 12.5, 6.25))


def test_tables(oracle):
    for blen, f in ((8, 0.2), (32, 0.2), (40, 0.05), (21, 0.7)):
        assert bitexact(rtmb.taper_vector(blen, f), oracle.taper_vector(blen, f))
    for nt, dt, fp in ((1000, 0.001, 15.0), (3000, 0.001, 12.0), (2500, 0.00125, 10.0)):
        assert bitexact(rtmb.ricker(nt, dt, fp), oracle.ricker(nt, dt, fp))


@pytest.mark.parametrize("bc", ["abc", "rbc", "hbc"])
def test_prepare_velocity(oracle, bc):
    rng = np.random.default_rng(4)
    v = (1500 + 3000 * rng.random((11, 13, 9))).astype(np.float32)
    a = rtmb.prepare_velocity(v, 7, bc, seed=77)
    b = oracle.extend_init_borders(v, 7, bc, seed=77)
    assert bitexact(a, b)
    assert bitexact(rtmb.v2dt2(a, 0.001), oracle.v2dt2(b, 0.001))


def test_invalid_arguments_are_errors_not_exits():
    lib = rtmb.load()
    p = rtmb.Params()
    p.nx = p.ny = p.nz = 8
    p.nt, p.ntstep, p.stencil_order = 10, 3, 8   # nt % ntstep != 0
    import ctypes as C
    h = C.c_void_p()
    assert lib.rtmb_create(C.byref(p), C.byref(h)) == rtmb.RTMB_EINVAL
    p.ntstep = 5
    p.stencil_order = 7                            # odd order
    assert lib.rtmb_create(C.byref(p), C.byref(h)) == rtmb.RTMB_EINVAL
    assert lib.rtmb_stencil_coefs(3, 1.0, 1.0, 1.0, None) == rtmb.RTMB_EINVAL


def test_storage_flag_combinations_are_checked_before_any_device_work():
    """rtmb_create rejects storage-form flags the library cannot honour (no CUDA call is made)."""
    import ctypes as C
    lib = rtmb.load()
    h = C.c_void_p()

    def create(order, nz, blen, flags):
        p = rtmb.Params()
        p.nx = p.ny = 16
        p.nz, p.blen, p.nt, p.ntstep, p.stencil_order, p.flags = nz, blen, 10, 5, order, flags
        return lib.rtmb_create(C.byref(p), C.byref(h))

    both = rtmb.FLAG_STORE_F16 | rtmb.FLAG_STORE_BF16
    assert create(8, 16, 8, both) == rtmb.RTMB_EINVAL
    assert b"choose one" in lib.rtmb_last_error(None)
    assert create(8, 16, 8, rtmb.FLAG_IMG_F64) == rtmb.RTMB_EINVAL      # FP64 image needs 16-bit storage
    assert create(4, 16, 8, rtmb.FLAG_STORE_F16) == rtmb.RTMB_EINVAL    # order 8 only
    assert create(8, 17, 8, rtmb.FLAG_STORE_BF16) == rtmb.RTMB_EINVAL   # nz + 2 blen = 33: not a multiple of 8
    assert b"multiple of 8" in lib.rtmb_last_error(None)
    assert create(8, 16, 8, rtmb.FLAG_STORE_DIFF) == rtmb.RTMB_EINVAL   # increment storage needs a 16-bit type
    assert b"STORE_DIFF" in lib.rtmb_last_error(None)


def test_survey_shot_list_and_partition_follow_the_reference():
    """rtmb.survey: the reference's source grid (x outer, y inner) dealt round-robin over ranks."""
    from rtmb import survey
    p = dict(nx=64, ny=64, nz=32, source_count_x=2, source_count_y=3, source_distance_x=20, source_distance_y=10,
             source_start_x=5, source_start_y=7, source_depth_z=1)
    assert survey.shot_positions(p) == [(5, 7, 1), (5, 17, 1), (5, 27, 1), (25, 7, 1), (25, 17, 1), (25, 27, 1)]
    assert survey.rank_shots(6, 0, 4) == [0, 4] and survey.rank_shots(6, 3, 4) == [3]
    assert list(survey.iter_rank_positions(survey.shot_positions(p), 1, 4)) == [(1, (5, 17, 1)), (5, (25, 27, 1))]


@pytest.mark.parametrize("nt,dt,fmin,fmax", [(120, 0.001, 5.0, 40.0), (90, 0.0012, 2.0, 30.0), (3000, 0.001, 0.0, 30.0),
                                             (100, 0.001, 10.0, 10.5)])
def test_fmig_frequency_count(oracle, nt, dt, fmin, fmax):
    """The library's nw of a frequency-domain migration is the oracle's (the reference's float mix)."""
    import rtmb
    assert rtmb.fmig_nw(dt, nt, fmin, fmax) == oracle.L.orc_fmig_nw(nt, dt, fmin, fmax)


def test_fmig_tables(oracle):
    """The library's DFT tables of a frequency-domain migration are the oracle's bit for bit."""
    import rtmb
    for args in ((120, 0.001, 5.0, 40.0), (90, 0.0012, 2.0, 30.0)):
        got = rtmb.fmig_tables(args[1], args[0], args[2], args[3])
        ref = oracle.fmig_tables(*args)
        for a, b in zip(got, ref):
            assert bitexact(a, b)
