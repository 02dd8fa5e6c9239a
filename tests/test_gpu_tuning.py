"""The autotuner's launch choices on the GPU (no reference counterpart: the reference launches a
fixed 10^3-thread block grid, RTMGPUPlatform.cpp:167-196).

Every launch variant of the step kernel (in-plane tile 64 x 16, 32 x 32, 64 x 8, or 64 x 16 with
shallower load rings), every launch variant of the dual backward step (64 x 8, 32 x 16, 32 x 16 with
deeper rings, and the merged form where each thread steps both wavefields), every x-chunk length and
the dual backward step against two launches change only how the work is split across CTAs and
threads: the RBC migration image must stay the same bit for bit, in
the exact form (which is the reference CPU path's arithmetic, checked against the oracle) and in the
FMA form."""
import numpy as np
import pytest

import rtmb
from rtm_cases import CASES, bitexact, layered_model, lib_input, oracle_params

pytestmark = pytest.mark.gpu


def _migrate(cuda, case, v2, rec, flags, tuning=None, autotune=False):
    import torch
    ctx = rtmb.Context(rtmb.Params.from_input(lib_input(case, "rbc"), flags=flags, device=0))
    ctx.load_v2dt2(v2, from_host=True)
    t = None
    if autotune:
        t = ctx.autotune_full()
    if tuning is not None:
        ctx.set_tuning(tuning)
    img = torch.zeros(ctx.padded_shape, device=cuda)
    ctx.migrate_shot(case["sx"], case["sy"], case["sz"], torch.from_numpy(rec).to(cuda), img)
    ctx.sync()
    ctx.close()
    return img.cpu().numpy(), t


@pytest.fixture(scope="module")
def mid_inputs(oracle):
    case = CASES["mid"]
    p = oracle_params(case)
    rec, _ = oracle.model_shot(p, oracle.v2dt2(oracle.extend_init_borders(layered_model(case), case["blen"], "abc"),
                                               case["dt"]))
    v2 = oracle.v2dt2(oracle.extend_init_borders(layered_model(case), case["blen"], "rbc", seed=7), case["dt"])
    return case, v2, rec


@pytest.mark.parametrize("form", ["exact", "fma"])
def test_every_launch_variant_gives_the_same_image(cuda, oracle, mid_inputs, form):
    case, v2, rec = mid_inputs
    flags = 0 if form == "exact" else rtmb.FLAG_FAST_FMA
    want, _ = _migrate(cuda, case, v2, rec, flags)
    if form == "exact":
        ref, rc = oracle.migrate(oracle_params(case), v2, rec, "rbc")
        assert rc == 0 and bitexact(want, ref)
    for variant in range(4):
        for chunk in (8, 48):
            for dual, dv in ((0, 0),) + tuple((1, dv) for dv in range(8)):
                t = dict(variant=variant, chunk=chunk, dual=dual, dual_chunk=chunk, dual_variant=dv)
                got, _ = _migrate(cuda, case, v2, rec, flags, tuning=t)
                assert bitexact(got, want), (variant, chunk, dual, dv)


@pytest.fixture(scope="module")
def golden_inputs(oracle):
    case = CASES["golden"]
    p = oracle_params(case)
    rec, _ = oracle.model_shot(p, oracle.v2dt2(oracle.extend_init_borders(layered_model(case), case["blen"], "abc"),
                                               case["dt"]))
    v2 = oracle.v2dt2(oracle.extend_init_borders(layered_model(case), case["blen"], "rbc", seed=7), case["dt"])
    return case, v2, rec


@pytest.mark.parametrize("form", ["exact", "fma"])
@pytest.mark.parametrize("rcv", ["overwrite", "add"])
def test_launch_variants_on_partial_tiles(cuda, oracle, golden_inputs, form, rcv):
    """The small case's padded grid (40 x 36 x 44, 28 computed y rows) leaves every tile shape of
    both step kernels partly outside the grid in y and z.  Every launch variant, and every dual step
    variant against the two launches (RTMB_FLAG_NO_DUAL), gives the same image bit for bit, with the
    receivers overwriting the receiver wavefield (the reference's injection) or added to it
    (RTMB_FLAG_RCV_ADD); the exact form with overwriting receivers is also the oracle's image."""
    case, v2, rec = golden_inputs
    flags = (0 if form == "exact" else rtmb.FLAG_FAST_FMA) | (rtmb.FLAG_RCV_ADD if rcv == "add" else 0)
    want, _ = _migrate(cuda, case, v2, rec, flags | rtmb.FLAG_NO_DUAL)
    if form == "exact" and rcv == "overwrite":
        ref, rc = oracle.migrate(oracle_params(case), v2, rec, "rbc")
        assert rc == 0 and bitexact(want, ref)
    for variant in range(4):
        for chunk in (8, 48):
            for dual, dv in ((0, 0),) + tuple((1, dv) for dv in range(8)):
                t = dict(variant=variant, chunk=chunk, dual=dual, dual_chunk=chunk, dual_variant=dv)
                got, _ = _migrate(cuda, case, v2, rec, flags, tuning=t)
                assert bitexact(got, want), (variant, chunk, dual, dv)


def test_autotune_full_keeps_results(cuda, mid_inputs):
    case, v2, rec = mid_inputs
    want, _ = _migrate(cuda, case, v2, rec, rtmb.FLAG_FAST_FMA)
    got, t = _migrate(cuda, case, v2, rec, rtmb.FLAG_FAST_FMA, autotune=True)
    assert t["variant"] in range(4) and t["chunk"] in (8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256)
    assert t["ms_step"] > 0 and t["ms_backward"] > 0 and t["dual"] in (0, 1) and t["dual_variant"] in range(8)
    assert bitexact(got, want)


def test_set_tuning_rejects_bad_values(cuda):
    case = CASES["golden"]
    ctx = rtmb.Context(rtmb.Params.from_input(lib_input(case, "rbc"), device=0))
    with pytest.raises(rtmb.RtmbError):
        ctx.set_tuning(dict(variant=9, chunk=8, dual=0, dual_chunk=8))
    with pytest.raises(rtmb.RtmbError):
        ctx.set_tuning(dict(variant=0, chunk=0, dual=0, dual_chunk=8))
    with pytest.raises(rtmb.RtmbError):
        ctx.set_tuning(dict(variant=0, chunk=8, dual=1, dual_chunk=8, dual_variant=8))
