"""GPU parity of the per-shot drivers (modeling, HBC and RBC migration) against the CPU oracle and
against the reference's own golden outputs.

Exact form: shot record and image BIT-EXACT.  FMA form: record rel-L2 <= 1e-5 and image rel-L2
<= 1e-4 (the tolerances set for the plain FP32 form)."""
import numpy as np
import pytest

import rtmb
from rtm_cases import CASES, bitexact, layered_model, lib_input, oracle_params, rel_l2

pytestmark = pytest.mark.gpu


def dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


def host(t):
    return t.detach().cpu().numpy()


def ctx_for(case, bc="hbc", flags=0):
    return rtmb.Context(rtmb.Params.from_input(lib_input(case, bc), flags=flags, device=0))


def rec_shape(case):
    return (case["nt"] // case["ntstep"], case["rcx"], case["rcy"], case["ntstep"])


def model_gpu(case, v2, cuda, flags=0):
    import torch
    ctx = ctx_for(case, flags=flags)
    ctx.load_v2dt2(dev(v2, cuda), from_host=False)
    rec = torch.zeros(rec_shape(case), dtype=torch.float32, device=cuda)
    ctx.model_shot(case["sx"], case["sy"], case["sz"], rec)
    return host(rec)


def migrate_gpu(case, v2, rec, bc, cuda, flags=0):
    import torch
    ctx = ctx_for(case, bc, flags)
    ctx.load_v2dt2(v2, from_host=True)
    img = torch.zeros(ctx.padded_shape, dtype=torch.float32, device=cuda)
    ctx.migrate_shot(case["sx"], case["sy"], case["sz"], dev(rec, cuda), img)
    out = torch.zeros((case["nx"], case["ny"], case["nz"]), dtype=torch.float32, device=cuda)
    ctx.image_finalize(img, out)
    ctx.sync()
    return host(img), host(out)


@pytest.mark.parametrize("flags", [0, rtmb.FLAG_NO_TAPER_STORE, rtmb.FLAG_NO_TMA], ids=["tma", "tma_raw", "plain"])
@pytest.mark.parametrize("cname", ["golden", "odd", "mid"])
def test_model_bitexact(cuda, oracle, cname, flags):
    case = CASES[cname]
    ve = oracle.extend_init_borders(layered_model(case), case["blen"], "abc")
    v2 = oracle.v2dt2(ve, case["dt"])
    ref, rc = oracle.model_shot(oracle_params(case), v2)
    assert rc == 0
    got = model_gpu(case, v2, cuda, flags=flags)
    assert bitexact(got, ref), rel_l2(got, ref)


@pytest.mark.parametrize("nt", [1, 2, 3, 4, 7])
@pytest.mark.parametrize("form", ["exact", "fma"])
def test_tapered_storage_matches_raw_fields(cuda, oracle, form, nt):
    """Modeling keeps the fields tapered in HBM: the record equals the taper-on-load form's bit for
    bit, in both arithmetic forms, for short and longer runs.  The source sits near the
    front-right x-y edge, whose cells take the taper's x = blen redirect."""
    import torch
    case = dict(CASES["golden"], nt=nt, ntstep=nt, sx=3, sy=17, sz=5)
    ve = oracle.extend_init_borders(layered_model(case), case["blen"], "abc")
    v2 = oracle.v2dt2(ve, case["dt"])
    base = rtmb.FLAG_FAST_FMA if form == "fma" else 0
    out = []
    for flags in (base, base | rtmb.FLAG_NO_TAPER_STORE):
        ctx = ctx_for(case, flags=flags)
        ctx.load_v2dt2(dev(v2, cuda), from_host=False)
        rec = torch.zeros(rec_shape(case), dtype=torch.float32, device=cuda)
        ctx.model_shot(case["sx"], case["sy"], case["sz"], rec)
        out.append(host(rec))
    assert nt < 3 or np.any(out[0] != 0)
    assert np.array_equal(out[0], out[1])
    if form == "exact":
        ref, rc = oracle.model_shot(oracle_params(case), v2)
        assert rc == 0 and bitexact(out[0], ref)


@pytest.mark.parametrize("extra", [0, rtmb.FLAG_IMG_FULL_Z], ids=["img", "img_full_z"])
@pytest.mark.parametrize("form", ["exact", "fma"])
def test_hbc_tapered_storage_matches_raw_fields(cuda, oracle, form, extra):
    """HBC migration keeps the source wavefield tapered in HBM except its last two levels (the
    snapshots of the backward pass) and the receiver wavefield tapered throughout: the image equals
    the taper-on-load form's bit for bit, also over the tapered top slab (RTMB_FLAG_IMG_FULL_Z)."""
    case = CASES["mid"]
    p = oracle_params(case)
    rec, _ = oracle.model_shot(p, oracle.v2dt2(oracle.extend_init_borders(layered_model(case), case["blen"], "abc"),
                                               case["dt"]))
    v2 = oracle.v2dt2(oracle.extend_init_borders(layered_model(case), case["blen"], "hbc", seed=4), case["dt"])
    base = (rtmb.FLAG_FAST_FMA if form == "fma" else 0) | extra
    a, _ = migrate_gpu(case, v2, rec, "hbc", cuda, flags=base)
    b, _ = migrate_gpu(case, v2, rec, "hbc", cuda, flags=base | rtmb.FLAG_NO_TAPER_STORE)
    assert np.abs(a).max() > 0
    assert np.array_equal(a, b)


def test_model_matches_reference_golden(cuda, golden):
    """GPU record vs the reference program's own .seism output."""
    import rtmb as R
    case = CASES["golden"]
    v2 = R.v2dt2(R.prepare_velocity(layered_model(case), case["blen"], "abc"), case["dt"])
    got = model_gpu(case, v2, cuda)
    assert bitexact(got, golden["model_abc"]["rec"])


@pytest.mark.parametrize("bc", ["hbc", "rbc"])
def test_migration_matches_reference_golden(cuda, golden, bc):
    """GPU image vs the reference program's own RTMIMG output (same extended velocity)."""
    case = CASES["golden"]
    g = golden[f"mig_{bc}"]
    _, fin = migrate_gpu(case, rtmb.v2dt2(g["vpe"], case["dt"]), g["rec"], bc, cuda)
    assert bitexact(fin, g["img"])


@pytest.mark.parametrize("flags", [0, rtmb.FLAG_NO_TMA], ids=["tma", "plain"])
@pytest.mark.parametrize("bc", ["hbc", "rbc"])
@pytest.mark.parametrize("cname", ["odd", "mid"])
def test_migration_bitexact(cuda, oracle, cname, bc, flags):
    case = CASES[cname]
    p = oracle_params(case)
    ve = oracle.extend_init_borders(layered_model(case), case["blen"], bc, seed=case["seed"])
    v2 = oracle.v2dt2(ve, case["dt"])
    rec, _ = oracle.model_shot(p, oracle.v2dt2(oracle.extend_init_borders(layered_model(case), case["blen"], "abc"),
                                               case["dt"]))
    ref_img, rc = oracle.migrate(p, v2, rec, bc)
    assert rc == 0
    img, _ = migrate_gpu(case, v2, rec, bc, cuda, flags=flags)
    assert bitexact(img, ref_img), rel_l2(img, ref_img)


@pytest.mark.parametrize("bc", ["hbc", "rbc"])
def test_fma_form_within_tolerance(cuda, oracle, bc):
    case = CASES["mid"]
    p = oracle_params(case)
    v2m = oracle.v2dt2(oracle.extend_init_borders(layered_model(case), case["blen"], "abc"), case["dt"])
    ref_rec, _ = oracle.model_shot(p, v2m)
    got_rec = model_gpu(case, v2m, cuda, flags=rtmb.FLAG_FAST_FMA)
    assert rel_l2(got_rec, ref_rec) <= 1e-5
    v2 = oracle.v2dt2(oracle.extend_init_borders(layered_model(case), case["blen"], bc, seed=1), case["dt"])
    ref_img, _ = oracle.migrate(p, v2, ref_rec, bc)
    img, _ = migrate_gpu(case, v2, ref_rec, bc, cuda, flags=rtmb.FLAG_FAST_FMA)
    assert rel_l2(img, ref_img) <= 1e-4


def test_host_buffer_forms(cuda, oracle):
    case = CASES["odd"]
    p = oracle_params(case)
    v2 = oracle.v2dt2(oracle.extend_init_borders(layered_model(case), case["blen"], "hbc", seed=2), case["dt"])
    ctx = ctx_for(case, "hbc")
    ctx.load_v2dt2(v2, from_host=True)
    rec = np.zeros(rec_shape(case), np.float32)
    ctx.model_shot_host(case["sx"], case["sy"], case["sz"], rec)
    ref_rec, _ = oracle.model_shot(p, v2)
    assert bitexact(rec, ref_rec)
    img = np.zeros(ctx.padded_shape, np.float32)
    ctx.migrate_shot_host(case["sx"], case["sy"], case["sz"], rec, img)
    ref_img, _ = oracle.migrate(p, v2, rec, "hbc")
    assert bitexact(img, ref_img)


def test_driver_errors(cuda):
    case = CASES["golden"]
    ctx = ctx_for(case)
    import torch
    rec = torch.zeros(rec_shape(case), device=cuda)
    with pytest.raises(rtmb.RtmbError) as e:
        ctx.model_shot(0, 0, 0, rec)          # no velocity loaded
    assert e.value.code == rtmb.RTMB_EINVAL
    ctx.load_v2dt2(np.full(ctx.padded_shape, 0.02, np.float32), from_host=True)
    with pytest.raises(rtmb.RtmbError) as e:
        ctx.model_shot(case["nx"], 0, 0, rec)  # source outside the model
    assert e.value.code == rtmb.RTMB_EINVAL
    bad = np.full(ctx.padded_shape, 0.02, np.float32)
    bad[20, 18, 20] = np.nan
    ctx.load_v2dt2(bad, from_host=True)
    with pytest.raises(rtmb.RtmbError) as e:
        ctx.model_shot(case["sx"], case["sy"], case["sz"], rec)
    assert e.value.code == rtmb.RTMB_ENAN


@pytest.mark.parametrize("bc", ["hbc", "rbc"])
def test_graph_replay_matches_eager(cuda, oracle, bc):
    """RTMB_FLAG_USE_GRAPH: the captured-and-replayed shots (the second one through an in-place
    update of the executable graph) give the eager results bit for bit."""
    import torch
    case = CASES["golden"]
    ve = oracle.extend_init_borders(layered_model(case), case["blen"], bc, seed=7)
    v2 = oracle.v2dt2(ve, case["dt"])
    shots = [(case["sx"], case["sy"], case["sz"]), (case["sx"] - 3, case["sy"] + 2, case["sz"] + 1)]
    out = {}
    for flags in (0, rtmb.FLAG_USE_GRAPH):
        ctx = ctx_for(case, bc, flags)
        ctx.load_v2dt2(v2, from_host=True)
        res = []
        for (sx, sy, sz) in shots:
            rec = torch.zeros(rec_shape(case), dtype=torch.float32, device=cuda)
            ctx.model_shot(sx, sy, sz, rec)
            img = torch.zeros(ctx.padded_shape, dtype=torch.float32, device=cuda)
            ctx.migrate_shot(sx, sy, sz, rec, img)
            ctx.sync()
            res += [host(rec), host(img)]
        out[flags] = (res, ctx.launches)
    for a, b in zip(out[0][0], out[rtmb.FLAG_USE_GRAPH][0]):
        assert bitexact(a, b)
    assert out[0][1] == out[rtmb.FLAG_USE_GRAPH][1]  # same kernels, counted the same way


def test_autotune_picks_a_chunk_and_keeps_results(cuda, oracle):
    """rtmb_autotune times the step kernel for several x-chunk lengths and keeps the fastest; the
    chunk only changes how planes are split across CTAs, never a result."""
    import torch
    case = CASES["mid"]
    ve = oracle.extend_init_borders(layered_model(case), case["blen"], "abc")
    v2 = oracle.v2dt2(ve, case["dt"])
    ctx = ctx_for(case, "hbc")
    ctx.load_v2dt2(v2, from_host=True)
    rec0 = torch.zeros(rec_shape(case), dtype=torch.float32, device=cuda)
    ctx.model_shot(case["sx"], case["sy"], case["sz"], rec0)
    chunk, ms = ctx.autotune()
    assert chunk in (8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256) and ms > 0
    rec1 = torch.zeros_like(rec0)
    ctx.model_shot(case["sx"], case["sy"], case["sz"], rec1)
    ctx.sync()
    assert bitexact(host(rec0), host(rec1))


@pytest.mark.parametrize("bc", ["hbc", "rbc"])
def test_dual_backward_step_matches_two_launches(cuda, oracle, bc):
    """In both FP32 forms the RBC backward source and receiver steps run as one dual-wavefield launch
    by default; it gives the two-launch result (RTMB_FLAG_NO_DUAL) bit for bit.  HBC migration keeps
    two launches."""
    import torch
    case = CASES["mid"]
    p = oracle_params(case)
    rec, _ = oracle.model_shot(p, oracle.v2dt2(oracle.extend_init_borders(layered_model(case), case["blen"], "abc"),
                                               case["dt"]))
    v2 = oracle.v2dt2(oracle.extend_init_borders(layered_model(case), case["blen"], bc, seed=7), case["dt"])
    out = {}
    for flags in (rtmb.FLAG_FAST_FMA, rtmb.FLAG_FAST_FMA | rtmb.FLAG_NO_DUAL, 0, rtmb.FLAG_NO_DUAL):
        ctx = ctx_for(case, bc, flags)
        ctx.load_v2dt2(v2, from_host=True)
        img = torch.zeros(ctx.padded_shape, dtype=torch.float32, device=cuda)
        ctx.profile(True)
        ctx.migrate_shot(case["sx"], case["sy"], case["sz"], dev(rec, cuda), img)
        ctx.sync()
        out[flags] = (host(img), ctx.profile_read()["backward_dual"]["launches"])
    fma, two, exact, exact_two = (out[rtmb.FLAG_FAST_FMA], out[rtmb.FLAG_FAST_FMA | rtmb.FLAG_NO_DUAL], out[0],
                                  out[rtmb.FLAG_NO_DUAL])
    n_dual = case["nt"] - 2 if bc == "rbc" else 0
    assert fma[1] == n_dual and two[1] == 0 and exact[1] == n_dual and exact_two[1] == 0
    assert bitexact(fma[0], two[0])
    assert bitexact(exact[0], exact_two[0])
