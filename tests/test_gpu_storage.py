"""The FP64 GPU oracle, the 16-bit storage forms and the FP64 image stack.

* The FP64 GPU oracle runs the reference's operator sequence in double precision on the FP32
  scheme, so it must agree with the (bit-exact FP32) CPU oracle to FP32 rounding: record rel-L2
  <= 1e-5 and image rel-L2 <= 1e-4, the tolerances of the plain FP32 form.
* The 16-bit storage forms (FP16 / BF16 with a power-of-two scale per stored level, FP32
  arithmetic) are measured against the FP64 oracle; the bounds below are the measured errors on
  these cases with about 3x headroom.
* rtmb_migrate_shot_acc64 adds a shot's image to an FP64 stack.
"""
import numpy as np
import pytest

import rtmb
from rtm_cases import CASES, layered_model, lib_input, oracle_params, rel_l2

pytestmark = pytest.mark.gpu

# measured rel-L2 against the FP64 oracle on the mid case (nt=200): record f16 2.1e-3, bf16 2.0e-2;
# image f16 1.0e-3, bf16 3.8e-2.  Bounds: about 3x those.
TOL_REC = {"f16": 6e-3, "bf16": 6e-2}
TOL_IMG = {"f16": 3e-3, "bf16": 1.2e-1}
STORE_FLAG = {"f16": rtmb.FLAG_STORE_F16, "bf16": rtmb.FLAG_STORE_BF16}


def dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


def host(t):
    return t.detach().cpu().numpy()


def ctx_for(case, bc, flags=0):
    return rtmb.Context(rtmb.Params.from_input(lib_input(case, bc), flags=flags, device=0))


def rec_shape(case):
    return (case["nt"] // case["ntstep"], case["rcx"], case["rcy"], case["ntstep"])


def velocity(oracle, case, bc):
    ve = oracle.extend_init_borders(layered_model(case), case["blen"], bc, seed=7)
    return oracle.v2dt2(ve, case["dt"])


def model_f64(case, v2, cuda, bc="hbc"):
    import torch
    ctx = ctx_for(case, bc)
    ctx.load_v2dt2(v2, from_host=True)
    rec = torch.zeros(rec_shape(case), dtype=torch.float64, device=cuda)
    ctx.model_shot_f64(case["sx"], case["sy"], case["sz"], rec)
    return host(rec)


def migrate_f64(case, v2, rec, bc, cuda):
    import torch
    ctx = ctx_for(case, bc)
    ctx.load_v2dt2(v2, from_host=True)
    img = torch.zeros(ctx.padded_shape, dtype=torch.float64, device=cuda)
    ctx.migrate_shot_f64(case["sx"], case["sy"], case["sz"], dev(rec, cuda), img)
    return host(img)


def model_form(case, v2, cuda, flags):
    import torch
    ctx = ctx_for(case, "hbc", flags)
    ctx.load_v2dt2(v2, from_host=True)
    rec = torch.zeros(rec_shape(case), dtype=torch.float32, device=cuda)
    ctx.model_shot(case["sx"], case["sy"], case["sz"], rec)
    return host(rec)


def migrate_form(case, v2, rec, cuda, flags, bc="rbc"):
    import torch
    ctx = ctx_for(case, bc, flags)
    ctx.load_v2dt2(v2, from_host=True)
    img = torch.zeros(ctx.padded_shape, dtype=torch.float32, device=cuda)
    ctx.migrate_shot(case["sx"], case["sy"], case["sz"], dev(rec, cuda), img)
    ctx.sync()
    return host(img)


@pytest.mark.parametrize("cname", ["golden", "mid"])
def test_f64_oracle_model_matches_cpu_oracle(cuda, oracle, cname):
    case = CASES[cname]
    v2 = velocity(oracle, case, "abc")
    ref, rc = oracle.model_shot(oracle_params(case), v2)
    assert rc == 0
    got = model_f64(case, v2, cuda)
    err = rel_l2(got, ref)
    assert 0 < err <= 1e-5, err  # nonzero: the FP64 path is not the FP32 one


@pytest.mark.parametrize("bc", ["hbc", "rbc"])
@pytest.mark.parametrize("cname", ["golden", "mid"])
def test_f64_oracle_migration_matches_cpu_oracle(cuda, oracle, cname, bc):
    case = CASES[cname]
    p = oracle_params(case)
    v2m = velocity(oracle, case, "abc")
    rec, _ = oracle.model_shot(p, v2m)
    v2 = velocity(oracle, case, bc)
    ref, rc = oracle.migrate(p, v2, rec, bc)
    assert rc == 0
    got = migrate_f64(case, v2, rec, bc, cuda)
    err = rel_l2(got, ref)
    assert 0 < err <= 1e-4, err


@pytest.mark.parametrize("store", ["f16", "bf16"])
def test_storage_model_record(cuda, oracle, store):
    case = CASES["mid"]
    v2 = velocity(oracle, case, "abc")
    ref = model_f64(case, v2, cuda)
    got = model_form(case, v2, cuda, STORE_FLAG[store])
    fp32 = model_form(case, v2, cuda, rtmb.FLAG_FAST_FMA)
    err, err32 = rel_l2(got, ref), rel_l2(fp32, ref)
    print(f"record rel-L2 vs FP64: {store} {err:.3e}, fp32 {err32:.3e}")
    assert err <= TOL_REC[store], err
    assert err32 <= 1e-5, err32


@pytest.mark.parametrize("img64", [False, True], ids=["img32", "img64"])
@pytest.mark.parametrize("store", ["f16", "bf16"])
def test_storage_migration_image(cuda, oracle, store, img64):
    case = CASES["mid"]
    p = oracle_params(case)
    rec, _ = oracle.model_shot(p, velocity(oracle, case, "abc"))
    v2 = velocity(oracle, case, "rbc")
    ref = migrate_f64(case, v2, rec, "rbc", cuda)
    flags = STORE_FLAG[store] | (rtmb.FLAG_IMG_F64 if img64 else 0)
    got = migrate_form(case, v2, rec, cuda, flags)
    fp32 = migrate_form(case, v2, rec, cuda, rtmb.FLAG_FAST_FMA)
    err, err32 = rel_l2(got, ref), rel_l2(fp32, ref)
    print(f"image rel-L2 vs FP64: {store} img64={img64} {err:.3e}, fp32 {err32:.3e}")
    assert err <= TOL_IMG[store], err
    assert err32 <= 1e-4, err32


def test_acc64_fp32_storage_adds_the_fp32_image(cuda, oracle):
    import torch
    case = CASES["mid"]
    p = oracle_params(case)
    rec, _ = oracle.model_shot(p, velocity(oracle, case, "abc"))
    v2 = velocity(oracle, case, "rbc")
    img = migrate_form(case, v2, rec, cuda, 0)
    ctx = ctx_for(case, "rbc")
    ctx.load_v2dt2(v2, from_host=True)
    stack = torch.zeros(ctx.padded_shape, dtype=torch.float64, device=cuda)
    r = dev(rec, cuda)
    ctx.migrate_shot_acc64(case["sx"], case["sy"], case["sz"], r, stack)
    ctx.sync()
    assert np.array_equal(host(stack), img.astype(np.float64))
    ctx.migrate_shot_acc64(case["sx"], case["sy"], case["sz"], r, stack)  # a second shot adds
    ctx.sync()
    assert np.array_equal(host(stack), img.astype(np.float64) * 2.0)


def test_acc64_store_matches_fp64_image_form(cuda, oracle):
    """With 16-bit storage, acc64 accumulates straight into the stack; rtmb_migrate_shot with
    RTMB_FLAG_IMG_F64 runs the same kernels into its own FP64 image and rounds it at the end."""
    import torch
    case = CASES["mid"]
    p = oracle_params(case)
    rec, _ = oracle.model_shot(p, velocity(oracle, case, "abc"))
    v2 = velocity(oracle, case, "rbc")
    flags = rtmb.FLAG_STORE_F16 | rtmb.FLAG_IMG_F64
    img = migrate_form(case, v2, rec, cuda, flags)
    ctx = ctx_for(case, "rbc", flags)
    ctx.load_v2dt2(v2, from_host=True)
    stack = torch.zeros(ctx.padded_shape, dtype=torch.float64, device=cuda)
    ctx.migrate_shot_acc64(case["sx"], case["sy"], case["sz"], dev(rec, cuda), stack)
    ctx.sync()
    assert np.array_equal(host(stack).astype(np.float32), img)


def test_storage_rejects_hbc_migration(cuda, oracle):
    import torch
    case = CASES["mid"]
    ctx = ctx_for(case, "hbc", rtmb.FLAG_STORE_F16)
    ctx.load_v2dt2(velocity(oracle, case, "hbc"), from_host=True)
    img = torch.zeros(ctx.padded_shape, dtype=torch.float32, device=cuda)
    rec = torch.zeros(rec_shape(case), dtype=torch.float32, device=cuda)
    with pytest.raises(rtmb.RtmbError) as e:
        ctx.migrate_shot(case["sx"], case["sy"], case["sz"], rec, img)
    assert e.value.code == rtmb.RTMB_EINVAL


@pytest.mark.parametrize("img64", [False, True], ids=["img32", "img64"])
@pytest.mark.parametrize("store", ["f16", "bf16"])
def test_increment_storage_migration_image(cuda, oracle, store, img64):
    """RTMB_FLAG_STORE_DIFF: the level and its increment each in 16 bits.  The image stays within
    the two-level form's bound against the FP64 oracle and is closer to it than the two-level form
    on the same case (the increment keeps the precision that p(t) - p(t-1) loses)."""
    case = CASES["mid"]
    p = oracle_params(case)
    rec, _ = oracle.model_shot(p, velocity(oracle, case, "abc"))
    v2 = velocity(oracle, case, "rbc")
    ref = migrate_f64(case, v2, rec, "rbc", cuda)
    extra = rtmb.FLAG_IMG_F64 if img64 else 0
    got = migrate_form(case, v2, rec, cuda, STORE_FLAG[store] | rtmb.FLAG_STORE_DIFF | extra)
    two = migrate_form(case, v2, rec, cuda, STORE_FLAG[store] | extra)
    err, err2 = rel_l2(got, ref), rel_l2(two, ref)
    print(f"image rel-L2 vs FP64: {store} increment {err:.3e}, two-level {err2:.3e}")
    assert err <= TOL_IMG[store], err
    assert err < err2, (err, err2)


def test_increment_storage_scope(cuda, oracle):
    """The increment form migrates with RBC; modeling and HBC migration are refused, and so is the
    flag without a 16-bit type."""
    import torch
    case = CASES["mid"]  # nz + 2 blen = 128: rows of 16-bit values in whole 16-byte units
    flags = rtmb.FLAG_STORE_F16 | rtmb.FLAG_STORE_DIFF
    for bc, call in (("hbc", "model"), ("hbc", "migrate")):
        ctx = ctx_for(case, bc, flags)
        ctx.load_v2dt2(velocity(oracle, case, bc), from_host=True)
        rec = torch.zeros(rec_shape(case), dtype=torch.float32, device=cuda)
        with pytest.raises(rtmb.RtmbError) as e:
            if call == "model":
                ctx.model_shot(case["sx"], case["sy"], case["sz"], rec)
            else:
                img = torch.zeros(ctx.padded_shape, dtype=torch.float32, device=cuda)
                ctx.migrate_shot(case["sx"], case["sy"], case["sz"], rec, img)
        assert e.value.code == rtmb.RTMB_EINVAL
    with pytest.raises(rtmb.RtmbError):
        ctx_for(case, "rbc", rtmb.FLAG_STORE_DIFF)
