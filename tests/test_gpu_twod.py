"""2D models (nx = 1): the reference's rtmStep2D (the plane x = blen, the y and z terms only) in
every driver and in the per-operator step, against the CPU oracle (pinned to the reference in
test_oracle_pin.py) and against the reference's own output files (tests/golden/twod.npz).

Exact form: BIT-EXACT.  FMA form: record rel-L2 <= 1e-5, image rel-L2 <= 1e-4."""
import numpy as np
import pytest

import rtmb
from rtm_cases import CASES, bitexact, layered_model, lib_input, oracle_params, rel_l2

pytestmark = pytest.mark.gpu


def dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


def case2d(cname="golden"):
    return dict(CASES[cname], nx=1, sx=0, rsx=0, rcx=1, rdx=1)


def rec_shape(case):
    return (case["nt"] // case["ntstep"], case["rcx"], case["rcy"], case["ntstep"])


def ctx_for(case, bc="hbc", flags=0):
    return rtmb.Context(rtmb.Params.from_input(lib_input(case, bc), flags=flags, device=0))


def model(case, v2, cuda, flags=0):
    import torch
    ctx = ctx_for(case, "hbc", flags)
    ctx.load_v2dt2(v2, from_host=True)
    rec = torch.zeros(rec_shape(case), dtype=torch.float32, device=cuda)
    ctx.model_shot(case["sx"], case["sy"], case["sz"], rec)
    ctx.sync()
    return rec.cpu().numpy()


def migrate(case, v2, rec, bc, cuda, flags=0):
    import torch
    ctx = ctx_for(case, bc, flags)
    ctx.load_v2dt2(v2, from_host=True)
    img = torch.zeros(ctx.padded_shape, dtype=torch.float32, device=cuda)
    ctx.migrate_shot(case["sx"], case["sy"], case["sz"], dev(rec, cuda), img)
    ctx.sync()
    return img.cpu().numpy()


@pytest.mark.parametrize("flags", [0, rtmb.FLAG_NO_TAPER_STORE, rtmb.FLAG_NO_TMA], ids=["tma", "tma_raw", "plain"])
@pytest.mark.parametrize("cname", ["golden", "odd"])
def test_twod_model_and_migration_bitexact(cuda, oracle, cname, flags):
    case = case2d(cname)
    p = oracle_params(case)
    v2m = oracle.v2dt2(oracle.extend_init_borders(layered_model(case), case["blen"], "abc"), case["dt"])
    ref, rc = oracle.model_shot(p, v2m)
    assert rc == 0 and np.abs(ref).max() > 0
    assert bitexact(model(case, v2m, cuda, flags), ref)
    for bc in ("hbc", "rbc"):
        v2 = oracle.v2dt2(oracle.extend_init_borders(layered_model(case), case["blen"], bc, seed=3), case["dt"])
        want, rc = oracle.migrate(p, v2, ref, bc)
        assert rc == 0 and np.abs(want).max() > 0
        assert bitexact(migrate(case, v2, ref, bc, cuda, flags), want), bc


def test_twod_matches_reference_files(cuda, oracle, golden):
    g = golden["twod"]
    case = case2d()
    v2m = oracle.v2dt2(oracle.extend_init_borders(layered_model(case), case["blen"], "abc"), case["dt"])
    assert bitexact(model(case, v2m, cuda), g["rec"])
    for bc in ("hbc", "rbc"):
        img = migrate(case, oracle.v2dt2(g[f"vpe_{bc}"], case["dt"]), g["rec"], bc, cuda)
        fin = oracle.filter_remove(img, case["blen"], case["dx"], case["dy"], case["dz"])
        assert bitexact(fin, g[f"img_{bc}"]), bc
    import torch
    ctx = ctx_for(case, "hbc")
    ctx.load_v2dt2(oracle.v2dt2(g["vpe_fmig"], case["dt"]), from_host=True)
    img = torch.zeros(ctx.padded_shape, dtype=torch.float32, device=cuda)
    ctx.migrate_shot_fmig(case["sx"], case["sy"], case["sz"], dev(g["rec"], cuda), img, float(g["fmin"]),
                          float(g["fmax"]))
    ctx.sync()
    fin = oracle.filter_remove(img.cpu().numpy(), case["blen"], case["dx"], case["dy"], case["dz"])
    assert bitexact(fin, g["img_fmig"])


def test_twod_fma_within_tolerance(cuda, oracle):
    case = case2d()
    p = oracle_params(case)
    v2m = oracle.v2dt2(oracle.extend_init_borders(layered_model(case), case["blen"], "abc"), case["dt"])
    ref, _ = oracle.model_shot(p, v2m)
    got = model(case, v2m, cuda, rtmb.FLAG_FAST_FMA)
    assert rel_l2(got, ref) <= 1e-5, rel_l2(got, ref)
    v2 = oracle.v2dt2(oracle.extend_init_borders(layered_model(case), case["blen"], "rbc", seed=3), case["dt"])
    want, _ = oracle.migrate(p, v2, ref, "rbc")
    img = migrate(case, v2, ref, "rbc", cuda, rtmb.FLAG_FAST_FMA)
    assert rel_l2(img, want) <= 1e-4, rel_l2(img, want)


@pytest.mark.parametrize("flags", [0, rtmb.FLAG_NO_TMA], ids=["tma", "plain"])
def test_twod_per_operator_step(cuda, oracle, flags):
    """rtmb_step on a 2D context is the reference's rtmStep2D: the plane x = blen, bit-exact, and
    nothing else written."""
    g_case = dict(case2d(), ny=14, nz=20, blen=6)
    rng = np.random.default_rng(9)
    shp = (1 + 2 * g_case["blen"], g_case["ny"] + 2 * g_case["blen"], g_case["nz"] + 2 * g_case["blen"])
    P = rng.standard_normal(shp).astype(np.float32)
    PP = rng.standard_normal(shp).astype(np.float32)
    V = (rng.random(shp) * 0.1).astype(np.float32)
    ctx = ctx_for(g_case, "hbc", flags)
    c = oracle.stencil_coefs(8, g_case["dx"], g_case["dy"], g_case["dz"])
    want, _ = oracle.step2d(8, c, P, PP, V, g_case["blen"])
    pp = dev(PP, cuda)
    ctx.step(dev(P, cuda), pp, dev(V, cuda))
    ctx.sync()
    assert bitexact(pp.cpu().numpy(), want)


def test_twod_rejected_where_unsupported(cuda, oracle):
    import torch
    case = case2d()
    ctx = ctx_for(case, "hbc")
    v2m = oracle.v2dt2(oracle.extend_init_borders(layered_model(case), case["blen"], "abc"), case["dt"])
    ctx.load_v2dt2(v2m, from_host=True)
    rec = torch.zeros(rec_shape(case), dtype=torch.float64, device=cuda)
    with pytest.raises(rtmb.RtmbError) as e:
        ctx.model_shot_f64(case["sx"], case["sy"], case["sz"], rec)
    assert e.value.code == rtmb.RTMB_EINVAL
