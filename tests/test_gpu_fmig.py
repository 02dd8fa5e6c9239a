"""Frequency-domain RTM (fmig) on the GPU against the CPU oracle (pinned to the reference program
in test_oracle_pin.py) and against the reference's own golden image.

Exact form: image BIT-EXACT, one pass over all frequencies (the reference CPU build's order) and
in groups of frequencies (the oracle run with the same groups).  FMA form: image rel-L2 <= 1e-4."""
import numpy as np
import pytest

import rtmb
from rtm_cases import CASES, bitexact, layered_model, lib_input, oracle_params, rel_l2

pytestmark = pytest.mark.gpu

BANDS = {"golden": (5.0, 40.0), "odd": (2.0, 30.0), "mid": (3.0, 24.0)}


def dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


def setup(oracle, cname):
    case = CASES[cname]
    p = oracle_params(case)
    v2m = oracle.v2dt2(oracle.extend_init_borders(layered_model(case), case["blen"], "abc"), case["dt"])
    rec, rc = oracle.model_shot(p, v2m)
    assert rc == 0
    v2 = oracle.v2dt2(oracle.extend_init_borders(layered_model(case), case["blen"], "hbc", seed=11), case["dt"])
    return case, p, v2, rec


def fmig_gpu(case, v2, rec, band, cuda, flags=0, nwstep=0):
    import torch
    ctx = rtmb.Context(rtmb.Params.from_input(lib_input(case, "hbc"), flags=flags, device=0))
    ctx.load_v2dt2(v2, from_host=True)
    img = torch.full(ctx.padded_shape, 7.0, dtype=torch.float32, device=cuda)  # overwritten
    ctx.migrate_shot_fmig(case["sx"], case["sy"], case["sz"], dev(rec, cuda), img, band[0], band[1], nwstep)
    ctx.sync()
    return img.cpu().numpy(), ctx


@pytest.mark.parametrize("cname", ["golden", "odd", "mid"])
def test_fmig_exact_bitexact(cuda, oracle, cname):
    case, p, v2, rec = setup(oracle, cname)
    band = BANDS[cname]
    ref, rc = oracle.migrate_fmig(p, v2, rec, *band)
    assert rc == 0 and np.abs(ref).max() > 0
    got, _ = fmig_gpu(case, v2, rec, band, cuda)
    assert bitexact(got, ref), rel_l2(got, ref)


def test_fmig_groups_bitexact(cuda, oracle):
    """nwstep = 1 and 3 re-run the time loop per group; the oracle with the same groups agrees."""
    case, p, v2, rec = setup(oracle, "golden")
    band = BANDS["golden"]
    for nws in (1, 3):
        ref, _ = oracle.migrate_fmig(p, v2, rec, *band, nws)
        got, _ = fmig_gpu(case, v2, rec, band, cuda, nwstep=nws)
        assert bitexact(got, ref), (nws, rel_l2(got, ref))


def test_fmig_matches_reference_golden(cuda, oracle, golden):
    case = CASES["golden"]
    g = golden["mig_fmig"]
    v2 = oracle.v2dt2(g["vpe"], case["dt"])
    got, _ = fmig_gpu(case, v2, g["rec"], (float(g["fmin"]), float(g["fmax"])), cuda)
    fin = oracle.filter_remove(got, case["blen"], case["dx"], case["dy"], case["dz"])
    assert bitexact(fin, g["img"])


@pytest.mark.parametrize("cname", ["golden", "mid"])
def test_fmig_fma_within_tolerance(cuda, oracle, cname):
    case, p, v2, rec = setup(oracle, cname)
    band = BANDS[cname]
    ref, _ = oracle.migrate_fmig(p, v2, rec, *band)
    got, ctx = fmig_gpu(case, v2, rec, band, cuda, flags=rtmb.FLAG_FAST_FMA)
    assert rel_l2(got, ref) <= 1e-4, rel_l2(got, ref)


def test_fmig_graph_and_profile(cuda, oracle):
    """The graph-captured time loop gives the eager result; the profile counts one DFT launch per
    time step and two wavefield steps."""
    case, p, v2, rec = setup(oracle, "golden")
    band = BANDS["golden"]
    eager, ctx = fmig_gpu(case, v2, rec, band, cuda)
    graph, _ = fmig_gpu(case, v2, rec, band, cuda, flags=rtmb.FLAG_USE_GRAPH)
    assert bitexact(graph, eager)
    import torch
    ctx.profile(True)
    img = torch.zeros(ctx.padded_shape, dtype=torch.float32, device=cuda)
    ctx.migrate_shot_fmig(case["sx"], case["sy"], case["sz"], dev(rec, cuda), img, *band)
    pr = ctx.profile_read()
    assert pr["fmig_freq"]["launches"] == case["nt"]
    assert pr["fmig_step"]["launches"] == 2 * case["nt"]


def test_fmig_errors(cuda, oracle):
    import torch
    case, p, v2, rec = setup(oracle, "golden")
    ctx = rtmb.Context(rtmb.Params.from_input(lib_input(case, "hbc"), device=0))
    ctx.load_v2dt2(v2, from_host=True)
    img = torch.zeros(ctx.padded_shape, dtype=torch.float32, device=cuda)
    r = dev(rec, cuda)
    for fmin, fmax in ((30.0, 30.0), (40.0, 5.0), (5.0, 6.0)):  # empty band; below one df
        with pytest.raises(rtmb.RtmbError) as e:
            ctx.migrate_shot_fmig(case["sx"], case["sy"], case["sz"], r, img, fmin, fmax)
        assert e.value.code == rtmb.RTMB_EINVAL


def test_fmig_per_operator_sequence_matches_driver(cuda, oracle):
    """The platform operators an adapter binds (rtmStepMultipleWave, the taper, the source, the
    receivers, rtmUpdateFreqContributions, rtmFreqDomainImageCondition), called through the C ABI
    in the reference's order, give the fused driver's image bit for bit."""
    import torch
    case, p, v2, rec = setup(oracle, "golden")
    band = BANDS["golden"]
    want, ctx = fmig_gpu(case, v2, rec, band, cuda)
    w2, kre, kim = (dev(a, cuda) for a in rtmb.fmig_tables(case["dt"], case["nt"], *band))
    nw = w2.numel()
    v = dev(v2, cuda)
    shp = ctx.padded_shape
    Ps, PPs, Pr, PPr = (torch.zeros(shp, dtype=torch.float32, device=cuda) for _ in range(4))
    fq = [torch.zeros((nw, case["nx"], case["ny"], case["nz"]), dtype=torch.float32, device=cuda) for _ in range(4)]
    img = torch.zeros(shp, dtype=torch.float32, device=cuda)
    r = dev(rec, cuda)
    nt, ntstep = case["nt"], case["ntstep"]
    for st in range(nt):
        rt = nt - 1 - st
        ctx.step_multiwave(Ps, PPs, Pr, PPr, v)
        for f in (Ps, PPs, Pr, PPr):
            ctx.taper_all(f)
        ctx.apply_source(PPs, case["sx"], case["sy"], case["sz"], st)
        ctx.restore_receivers(PPr, r[rt // ntstep], rt % ntstep)
        for iw in range(nw):
            ctx.fmig_update_freq(st, iw, iw, PPs, PPr, *fq, kre, kim)
            ctx.fmig_image_condition(iw, iw, w2, img, *fq)
        Ps, PPs = PPs, Ps
        Pr, PPr = PPr, Pr
    ctx.sync()
    assert bitexact(img.cpu().numpy(), want)
